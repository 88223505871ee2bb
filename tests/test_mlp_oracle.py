"""CPU pinning of the bracket-network oracle (oracle/mlp_oracle.hpp) and of
the learned-bracket c2p in the oracle.

The network has no counterpart in the reference, so its oracle is pinned
independently: the FP64 gradient by central finite differences, the
BF16-emulating forward by a torch re-implementation with torch's own
bfloat16 rounding, the features by a numpy restatement of the Kastaun
scalars (kastaun_c2p.hh:306-337).  The bracket contract (results do not
depend on where the Brent solve starts, only iteration counts do) is
checked on the oracle's c2p with brackets built from the plain roots."""
import numpy as np
import torch

import _oracle
from grace_b200 import abi, params, workloads
from parity import prim_tol, state_residual

H = 64


def random_params(seed):
    rng = np.random.default_rng(seed)
    P = np.zeros(abi.MLP_NUM_PARAMS, np.float32)
    nf = abi.MLP_IN
    o = 0
    W1 = np.zeros((H, 16), np.float32)
    W1[:, :nf] = rng.uniform(-1.1, 1.1, (H, nf))
    W1[:, nf:2 * nf] = W1[:, :nf]
    P[o:o + H * 16] = W1.ravel(); o += H * 16
    P[o:o + H] = rng.uniform(-0.1, 0.1, H); o += H
    for _ in range(2):
        P[o:o + H * H] = rng.uniform(-0.3, 0.3, H * H); o += H * H
        P[o:o + H] = rng.uniform(-0.1, 0.1, H); o += H
    P[o:o + H] = rng.uniform(-0.3, 0.3, H); o += H
    P[o] = 0.05; o += 1
    assert o == abi.MLP_NUM_WEIGHTS
    P[o:o + nf] = [-6.0, -1.0, 0.5, -2.0, 0.3, -3.0]
    P[o + nf:o + 2 * nf] = [2.5, 2.0, 1.0, 2.5, 0.3, 1.5]
    P[o + 2 * nf], P[o + 2 * nf + 1], P[o + 2 * nf + 2] = 1e-3, 2e-2, 0.05
    return P


def feats_targets(n, seed):
    cons, _ = workloads.c2p_states(n, seed=seed)
    f = _oracle.mlp_features(params.c2p_bench(), cons)
    rng = np.random.default_rng(seed + 1)
    t = np.abs(1e-3 + 2e-2 * rng.standard_normal(n)).astype(np.float32)
    return cons, f, t


def test_features_match_numpy_restatement():
    P = params.c2p_bench()
    cons, _ = workloads.c2p_states(4000, seed=31)
    f = _oracle.mlp_features(P, cons)
    D = cons[0]
    q = cons[4] / D
    r = cons[1:4] / D
    Bt = cons[7:10] / np.sqrt(D)
    r2 = np.sum(r * r, axis=0)
    b2 = np.sum(Bt * Bt, axis=0)
    rb = np.sum(r * Bt, axis=0)
    ref = np.stack([np.log10(D), np.log10(np.maximum(q, 1e-30)), 0.5 * np.log10(r2 + 1e-30),
                    np.log10(b2 + 1e-30), np.clip(rb * rb / (r2 * b2 + 1e-300), 0, 1)])
    assert np.max(np.abs(f[:5] - ref)) < 2e-5
    # log mu0 bounds the plain root from above (kastaun_c2p.hh:355-372)
    n = cons.shape[1]
    z = np.zeros(n)
    _, _, _, _, _, mu, _ = _oracle.c2p_batch_guess(P, cons, z, z)
    ok = mu > 0
    assert ok.mean() > 0.99
    assert np.all(f[5][ok] >= np.log(mu[ok]) - 1e-6)


def _torch_forward(P, feat):
    """Independent forward with torch's bfloat16 rounding (FP64 sums)."""
    bf = lambda x: torch.as_tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64)
    o = 0
    W1 = bf(P[o:o + H * 16].reshape(H, 16)); o += H * 16
    b1 = torch.as_tensor(P[o:o + H], dtype=torch.float64); o += H
    W2 = bf(P[o:o + H * H].reshape(H, H)); o += H * H
    b2 = torch.as_tensor(P[o:o + H], dtype=torch.float64); o += H
    W3 = bf(P[o:o + H * H].reshape(H, H)); o += H * H
    b3 = torch.as_tensor(P[o:o + H], dtype=torch.float64); o += H
    w4 = torch.as_tensor(P[o:o + H], dtype=torch.float64); o += H
    b4 = float(P[o]); o += 1
    nf = abi.MLP_IN
    fmu, fsd, tmu, tsd = P[o:o + nf], P[o + nf:o + 2 * nf], P[o + 2 * nf], P[o + 2 * nf + 1]
    xn = (torch.as_tensor(feat.T, dtype=torch.float32) - torch.as_tensor(fmu)) / torch.as_tensor(fsd)
    x = torch.zeros(feat.shape[1], 16, dtype=torch.float64)
    hi = xn.to(torch.bfloat16).to(torch.float32)
    x[:, :nf] = hi.to(torch.float64)
    x[:, nf:2 * nf] = (xn - hi).to(torch.bfloat16).to(torch.float64)
    act = lambda a: bf(torch.relu(a).to(torch.float32))
    h1 = act(x @ W1.T + b1)
    h2 = act(h1 @ W2.T + b2)
    h3 = act(h2 @ W3.T + b3)
    return (h3 @ w4 + b4).numpy() * float(tsd) + float(tmu)


def test_forward_matches_torch_bf16():
    P = random_params(3)
    _, f, _ = feats_targets(3000, 32)
    y = _oracle.mlp_forward(P, f, emulate=True)
    yt = _torch_forward(P, f)
    # same rounding points; only FP64 summation order differs, which can
    # move a value across a BF16 rounding boundary in rare cases
    d = np.abs(y - yt)
    assert np.mean(d < 1e-10) > 0.99
    assert np.max(d) < 1e-2


def test_gradient_matches_finite_differences():
    P = random_params(4)
    _, f, t = feats_targets(256, 33)
    loss, g = _oracle.mlp_loss_grad(P, f, t, emulate=False)
    assert np.isfinite(loss) and loss > 0
    rng = np.random.default_rng(5)
    idx = np.concatenate([rng.integers(0, abi.MLP_NUM_WEIGHTS, 40),
                          [abi.MLP_NUM_WEIGHTS - 1, 16 * 64 + 3, 0, 1, 2, 3, 4]])
    for i in idx:
        h = 1e-5 * max(1.0, abs(float(P[i])))
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        hp = float(Pp[i]) - float(P[i])
        hm = float(P[i]) - float(Pm[i])
        lp, _ = _oracle.mlp_loss_grad(Pp, f, t, emulate=False)
        lm, _ = _oracle.mlp_loss_grad(Pm, f, t, emulate=False)
        fd = (lp - lm) / (hp + hm)
        assert abs(fd - g[i]) <= 1e-4 * abs(g[i]) + 1e-8, (i, fd, g[i])
    # without BF16 emulation the remainder inputs are zero: no gradient there
    W1g = g[:64 * 16].reshape(64, 16)
    assert np.all(W1g[:, abi.MLP_IN:] == 0.0)
    _, ge = _oracle.mlp_loss_grad(P, f, t, emulate=True)
    assert np.all(ge[:64 * 16].reshape(64, 16)[:, 2 * abi.MLP_IN:] == 0.0)


def test_bf16_gradient_is_close_to_fp64():
    P = random_params(6)
    _, f, t = feats_targets(2048, 34)
    l0, g0 = _oracle.mlp_loss_grad(P, f, t, emulate=False)
    l1, g1 = _oracle.mlp_loss_grad(P, f, t, emulate=True)
    assert abs(l1 - l0) < 0.05 * l0
    assert np.linalg.norm(g1 - g0) < 0.1 * np.linalg.norm(g0)


def test_oracle_bracket_changes_iterations_not_results():
    """Oracle c2p started from brackets around the plain root: the same
    primitives within the c2p tolerance whatever the width; fewer Brent
    iterations only once the bracket is narrower than ~1e-5 relative (the
    plain top mu0 is within 5e-5 of the root for half of these states, so
    Brent from [0, mu0] already needs ~5 iterations); from a bracket that
    misses the root, the plain path, bit-identical."""
    P = params.c2p_bench()
    cons, _ = workloads.c2p_states(20000, seed=35)
    n = cons.shape[1]
    none = np.zeros(n)
    pr0, co0, e0, it0, gu0, mu0, _ = _oracle.c2p_batch_guess(P, cons, none, none)
    assert not gu0.any()
    pr_plain, _, e_plain, _, it_plain, _ = _oracle.c2p_batch(P, cons)
    assert np.array_equal(pr0, pr_plain) and np.array_equal(e0, e_plain) and np.array_equal(it0, it_plain)
    ok = mu0 > 0
    mean_iters = {}
    for w in (1e-2, 1e-3, 1e-6):
        lo = np.where(ok, mu0 * np.exp(-w), 0.0)
        hi = np.where(ok, mu0 * np.exp(w), 0.0)
        pr1, _, e1, it1, gu1, mu1, _ = _oracle.c2p_batch_guess(P, cons, lo, hi)
        assert gu1[ok].mean() > 0.999
        same = e1 == e0
        assert same.mean() > 0.999
        res = state_residual(pr1[:, same], pr0[:, same])
        assert np.all(res < prim_tol(pr0)[same]), res.max()
        mean_iters[w] = it1[gu1 == 1].mean()
    plain = it0[ok].mean()
    assert 4.0 < plain < 6.0
    assert mean_iters[1e-6] < plain - 1.0
    assert mean_iters[1e-2] > mean_iters[1e-3] > mean_iters[1e-6]
    # brackets entirely above the root: no sign change -> plain path
    lo2 = np.where(ok, mu0 * 1.5, 0.0)
    hi2 = np.where(ok, mu0 * 1.6, 0.0)
    pr2, _, e2, it2, gu2, _, _ = _oracle.c2p_batch_guess(P, cons, lo2, hi2)
    assert not gu2.any()
    assert np.array_equal(pr2, pr0) and np.array_equal(it2, it0)


def test_plain_solver_window_exceeds_flat_1e12():
    """The acceptance bound of a learned bracket against the plain c2p.
    Brent stops within 2 eps |mu| + 1e-15 of the root in mu
    (kastaun_c2p.hh:372, rootfinding.hh:73-231): an absolute window, so a
    state with small mu (hot or magnetised) has a relative window up to
    1e-15 / mu in mu, and W = (1 - v^2)^(-1/2) amplifies it by ~W^2 in the
    primitives.  The plain solver itself, started from any other valid
    bracket around the root, moves the primitives of about 17 % of the c2p
    workload's states by more than 1e-12 (up to ~1e-9 at W ~ 50), with every
    state within 1e-12 x max(1, W^2): a flat 1e-12 is not a property of the
    plain path, the W^2-scaled bound is, and the learned bracket is held to
    that bound (same error bits, residual <= 1e-12 max(1, W^2))."""
    from parity import prim_tol, state_residual
    P = params.c2p_bench()
    n = 1 << 16
    cons, _ = workloads.c2p_states(n, seed=5)
    z = np.zeros(n)
    pr0, _, err0, _, _, mu0, _ = _oracle.c2p_batch_guess(P, cons, z, z)
    assert np.all(mu0 > 0)
    # the same plain solve from the bracket [0.9 mu, mu0]: same function,
    # same tolerance, another start
    pr1, _, err1, _, used, mu1, _ = _oracle.c2p_batch_guess(P, cons, 0.9 * mu0, np.full(n, 1e300))
    assert used.mean() == 1.0 and np.array_equal(err0, err1)
    r = state_residual(pr1, pr0)
    assert 0.05 < np.mean(r > 1e-12) < 0.5 and r.max() > 1e-10
    assert np.all(r <= prim_tol(pr0))
