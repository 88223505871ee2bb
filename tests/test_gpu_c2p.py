"""GPU c2p (through the C ABI) against the CPU oracle."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import GRMHDEquationsSystem
from parity import PRIM_TOL, prim_tol, state_residual

pytestmark = pytest.mark.gpu


def _compare(P, cons, metric=None, mode=abi.MODE_PLAIN):
    dev = torch.device("cuda:0")
    sysg = GRMHDEquationsSystem(P)
    sysg.set_mode(mode)
    c_d = torch.from_numpy(np.ascontiguousarray(cons)).to(dev)
    m_d = torch.from_numpy(np.ascontiguousarray(metric)).to(dev) if metric is not None else None
    n = cons.shape[1]
    err_d = torch.zeros(n, dtype=torch.int32, device=dev)
    co_d = torch.zeros_like(c_d)
    pr_g = sysg.conservs_to_prims(c_d, m_d, cons_out=co_d, err=err_d).cpu().numpy()
    err_g = err_d.cpu().numpy().view(np.uint32)
    pr_o, co_o, err_o, _, _, _ = _oracle.c2p_batch(P, cons, metric)
    return pr_g, co_d.cpu().numpy(), err_g, pr_o, co_o, err_o


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
@pytest.mark.parametrize("preset", ["c2p_bench", "blast"])
def test_c2p_batch_matches_oracle(preset, mode):
    """Plain mode: the reference's operations; tuned mode: the tuned c2p
    arithmetic (same functions up to rounding), both within the W^2-aware
    1e-12 bound of the oracle."""
    P = getattr(params, preset)()
    cons, _ = workloads.c2p_states(50000, seed=11)
    pr_g, co_g, err_g, pr_o, co_o, err_o = _compare(P, cons, mode=mode)
    assert (err_g == err_o).mean() > 0.999
    same = err_g == err_o
    tol = prim_tol(pr_o)[same]
    res = state_residual(pr_g[:, same], pr_o[:, same])
    assert np.all(res < tol), res.max()
    rho_rel = np.abs(pr_g[abi.P_RHO][same] - pr_o[abi.P_RHO][same]) / pr_o[abi.P_RHO][same]
    assert np.all(rho_rel < tol), rho_rel.max()
    assert np.mean(rho_rel < PRIM_TOL) > 0.95


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_c2p_without_entropy_backup_matches_oracle(mode):
    """use_ent_backup = 0 (grmhd.c2p.use_entropy_backup off): the states whose
    Kastaun result is distrusted keep it instead of the entropy-based solve
    (the tuned mode's deferred second pass then has nothing to do), against
    the oracle with the same switch."""
    P = params.c2p_bench()
    P.use_ent_backup = 0
    cons, _ = workloads.c2p_states(50000, seed=12)
    pr_g, co_g, err_g, pr_o, co_o, err_o = _compare(P, cons, mode=mode)
    assert (err_g == err_o).mean() > 0.999
    same = err_g == err_o
    res = state_residual(pr_g[:, same], pr_o[:, same])
    assert np.all(res < prim_tol(pr_o)[same]), res.max()
    # the switch matters on this workload: with the backup on, a fifth of the
    # states (the magnetically dominated ones) come out of the other solve,
    # different beyond 1e-12
    pr_b = _oracle.c2p_batch(params.c2p_bench(), cons)[0]
    assert np.mean(state_residual(pr_b, pr_o) > 1e-12) > 0.1


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_c2p_velocity_limit_matches_oracle(mode):
    """max_w = 10 (grmhd.c2p.max_lorentz_factor): limit_primitives rescales
    the velocity of the 80 % of the workload's states that would move
    faster (c2p.cpp:63-115), flagged in the error bits; against the oracle
    with the same limit."""
    P = params.c2p_bench()
    P.max_w = 10.0
    cons, _ = workloads.c2p_states(50000, seed=13)
    pr_g, co_g, err_g, pr_o, co_o, err_o = _compare(P, cons, mode=mode)
    assert (err_g == err_o).mean() > 0.999
    same = err_g == err_o
    # the limiter rescales the solved state, so the solver's window is that
    # of the unlimited state: the W^2-aware bound of the unlimited solve
    pr_u, _, err_u, _, _, _ = _oracle.c2p_batch(params.c2p_bench(), cons)
    res = state_residual(pr_g[:, same], pr_o[:, same])
    assert np.all(res < prim_tol(pr_u)[same]), res.max()
    W = np.sqrt(1.0 + np.sum(pr_g[abi.P_ZX:abi.P_ZZ + 1] ** 2, axis=0))
    assert W.max() < 10.0
    assert np.mean(err_o != err_u) > 0.5


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
@pytest.mark.parametrize("knob", ["temp_fl", "eps_max"])
def test_c2p_floors_and_ceilings_match_oracle(knob, mode):
    """The temperature floor (grmhd.atmosphere.temp_fl: the floored states'
    temperature reset and pressure recomputed, c2p.cpp:356-370) and the eps
    ceiling (eos.eps_maximum: the upper eps bound of the EOS range that
    limit_conservatives and the solves use, and the entropy backup's result
    accepted only below it, c2p.cpp:303) set where they act
    on about 30 % of the workload's states, against the oracle with the same
    setting."""
    cons, _ = workloads.c2p_states(50000, seed=14)
    base = _oracle.c2p_batch(params.c2p_bench(), cons)
    P = params.c2p_bench()
    if knob == "temp_fl":
        P.temp_fl = float(np.quantile(base[0][abi.P_TEMP], 0.3))
    else:
        P.eos.eps_max = float(np.quantile(base[0][abi.P_EPS], 0.7))
    pr_g, co_g, err_g, pr_o, co_o, err_o = _compare(P, cons, mode=mode)
    assert np.mean(err_o != base[2]) > 0.2  # the knob acts
    assert (err_g == err_o).mean() > 0.999
    same = err_g == err_o
    res = state_residual(pr_g[:, same], pr_o[:, same])
    assert np.all(res < prim_tol(base[0])[same]), res.max()
    assert np.all(np.isfinite(pr_g[:12]))


def test_c2p_curved_metric_matches_oracle():
    """Schwarzschild in Cartesian Kerr-Schild at R=4 (the curved-metric sweep
    of test/test_c2p.cpp:359-455): primitives -> cons on that metric -> c2p."""
    import ctypes
    P = params.c2p_bench()
    _, prims = workloads.c2p_states(8192, seed=12)
    n = prims.shape[1]
    H = 1.0 / 4.0
    fac = 1 + 2 * H
    metric = np.zeros((10, n))
    metric[0] = fac
    metric[3] = metric[5] = 1.0
    metric[6] = 2 * H / fac
    metric[9] = 1 / np.sqrt(fac)
    L = _oracle.lib("orc")
    cons = np.zeros((10, n))
    L.orc_prims_to_conservs(ctypes.byref(P), n, _oracle.p(np.ascontiguousarray(prims)), _oracle.p(metric),
                            _oracle.p(cons))
    cons[7:10] = prims[abi.P_BX:abi.P_BZ + 1] * np.sqrt(fac)
    pr_g, _, err_g, pr_o, _, err_o = _compare(P, cons, metric)
    same = err_g == err_o
    assert same.mean() > 0.99
    rel = np.abs(pr_g[abi.P_RHO][same] - pr_o[abi.P_RHO][same]) / pr_o[abi.P_RHO][same]
    assert np.all(rel < prim_tol(pr_o)[same])


def test_c2p_edge_cases():
    """Negative density, zero momentum, tau below the floor, NaN-free output."""
    P = params.c2p_bench()
    cons, _ = workloads.c2p_states(64, seed=13)
    cons[0, 0] = -1e-8           # D < 0 -> atmosphere
    cons[1:4, 1] = 0.0           # zero momentum
    cons[4, 2] = -1.0            # tau far below the floor -> limit_conservatives
    cons[0, 3] = 1e-20           # below the atmosphere threshold
    pr_g, co_g, err_g, pr_o, co_o, err_o = _compare(P, cons)
    assert np.array_equal(err_g, err_o)
    assert np.all(np.isfinite(pr_g[:12]))
    assert err_g[0] & (1 << 20) and err_g[3] & (1 << 20)  # C2P_ATMO_RESET
    rel = np.abs(pr_g[abi.P_RHO] - pr_o[abi.P_RHO]) / pr_o[abi.P_RHO]
    assert np.all(rel < prim_tol(pr_o))
