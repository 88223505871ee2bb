"""FMR restriction into coarse buffers (grb_restrict_to_coarse) and
prolongation into ghost zones (grb_prolong_to_ghosts) on the GPU
against the oracle (oracle/amr_oracle.hpp, itself pinned to the reference's
operators): bit for bit, both variable lists, every Morton child position,
the three face arrays, every ghost element kind; and div B of the restricted
and of the prolonged face fields."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem

pytestmark = pytest.mark.gpu

N, G = 16, 4
NN = N + 2 * G


def test_restrict_to_coarse_matches_oracle_bitwise():
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(31)
    nq, ncb = 16, 16
    st = rng.standard_normal((nq, abi.N_EVOL_VARS, NN, NN, NN))
    fb = [rng.standard_normal((nq, NN, NN, NN + 1)), rng.standard_normal((nq, NN, NN + 1, NN)),
          rng.standard_normal((nq, NN + 1, NN, NN))]
    src_q = np.arange(nq, dtype=np.int64)
    dst_q = rng.permutation(ncb)[:nq].astype(np.int64)
    child = (np.arange(nq) % 8).astype(np.uint8)
    vlo, vhi = [0, 5, 6, 13], [1, 2, 3, 4]
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(N, N, N, G, nq, np.ones((nq, 3)), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    fine = Fields(T(st), T(fb[0]), T(fb[1]), T(fb[2]))
    cb = Fields(torch.zeros((ncb, abi.N_EVOL_VARS, NN, NN, NN), dtype=torch.float64, device=dev),
                *[torch.zeros((ncb,) + x.shape[1:], dtype=torch.float64, device=dev) for x in fb])
    g.restrict_to_coarse(fine, cb, T(src_q), T(dst_q), T(child), vlo, vhi)
    torch.cuda.synchronize()
    # oracle
    ost = np.zeros((ncb, abi.N_EVOL_VARS, NN, NN, NN))
    _oracle.restrict_cells("orc", N, G, abi.N_EVOL_VARS, st, ost, src_q, dst_q, child, vlo, vhi)
    np.testing.assert_array_equal(cb.state.cpu().numpy(), ost)
    for d in range(3):
        of = np.zeros((ncb,) + fb[d].shape[1:])
        _oracle.restrict_faces(d, N, G, np.ascontiguousarray(fb[d]), of, src_q, dst_q)
        np.testing.assert_array_equal((cb.bx, cb.by, cb.bz)[d].cpu().numpy(), of)
    assert g.status().device_flags == 0


@pytest.mark.parametrize("n", [4, 6, 8])
def test_restrict_small_blocks_match_oracle(n):
    """The 5-point restriction on small blocks: with 4 cells along z one
    thread per coarse cell, from 6 on the z-column walk, both bit for bit."""
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(40 + n)
    nq = 8
    M = n + 2 * G
    st = rng.standard_normal((nq, abi.N_EVOL_VARS, M, M, M))
    q = np.arange(nq, dtype=np.int64)
    child = np.arange(nq).astype(np.uint8)
    vlo, vhi = [0, 4], [1, 2, 3, 7, 20]
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(n, n, n, G, nq, np.ones((nq, 3)), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    fine = Fields(T(st), None, None, None)
    cb = Fields(torch.zeros_like(fine.state), None, None, None)
    g.restrict_to_coarse(fine, cb, T(q), T(q), T(child), vlo, vhi, faces=False)
    torch.cuda.synchronize()
    ost = np.zeros_like(st)
    _oracle.restrict_cells("orc", n, G, abi.N_EVOL_VARS, st, ost, q, q, child, vlo, vhi)
    np.testing.assert_array_equal(cb.state.cpu().numpy(), ost)


def test_restricted_face_field_is_divergence_free():
    """A discretely divergence-free fine face field (curl of an edge vector
    potential) restricts to a divergence-free coarse one."""
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(8)
    Ax, Ay, Az = [rng.standard_normal((NN + 1, NN + 1, NN + 1)) for _ in range(3)]
    bx = (Az[:NN, 1:, :] - Az[:NN, :NN, :]) - (Ay[1:, :NN, :] - Ay[:NN, :NN, :])
    by = (Ax[1:, :, :NN] - Ax[:NN, :, :NN]) - (Az[:NN, :, 1:] - Az[:NN, :, :NN])
    bz = (Ay[:, :NN, 1:] - Ay[:, :NN, :NN]) - (Ax[:, 1:, :NN] - Ax[:, :NN, :NN])
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(N, N, N, G, 1, np.ones((1, 3)), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)[None]).to(dev)
    st = torch.zeros((1, abi.N_EVOL_VARS, NN, NN, NN), dtype=torch.float64, device=dev)
    fine = Fields(st, T(bx), T(by), T(bz))
    cb = Fields(st.clone(), *[torch.zeros_like(x) for x in (fine.bx, fine.by, fine.bz)])
    q = torch.zeros(1, dtype=torch.int64, device=dev)
    g.restrict_to_coarse(fine, cb, q, q)
    cx, cy, cz = (x[0].cpu().numpy() for x in (cb.bx, cb.by, cb.bz))
    h, s = N // 2, slice(G, G + N // 2)
    div = (cx[s, s, G + 1:G + h + 1] - cx[s, s, s]) + (cy[s, G + 1:G + h + 1, s] - cy[s, s, s]) + \
          (cz[G + 1:G + h + 1, s, s] - cz[s, s, s])
    assert np.max(np.abs(div)) < 1e-13


NELEM = {0: 6, 1: 12, 2: 8}
FSH = [(NN, NN, NN + 1), (NN, NN + 1, NN), (NN + 1, NN, NN)]


@pytest.mark.parametrize("n", [16, 8, 4])
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_prolong_to_ghosts_matches_oracle_bitwise(kind, n):
    """grb_prolong_to_ghosts against the oracle (pinned to the reference's
    prolong_op / div_free_prolong_op): every element of the kind on several
    quadrants, both variable lists, face B with random fine-neighbour
    flags, bit for bit."""
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(60 + kind + n)
    nq, ncb = 6, 8
    NN = n + 2 * G
    FSH = [(NN, NN, NN + 1), (NN, NN + 1, NN), (NN + 1, NN, NN)]
    st0 = rng.standard_normal((nq, abi.N_EVOL_VARS, NN, NN, NN))
    fb0 = [rng.standard_normal((nq,) + s) for s in FSH]
    cst = rng.standard_normal((ncb, abi.N_EVOL_VARS, NN, NN, NN))
    cfb = [rng.standard_normal((ncb,) + s) for s in FSH]
    fq = np.repeat(np.arange(nq), NELEM[kind]).astype(np.int64)
    el = np.tile(np.arange(NELEM[kind]), nq).astype(np.uint8)
    perm = rng.permutation(len(fq))
    fq, el = fq[perm], el[perm]
    cq = rng.permutation(ncb)[:nq][fq].astype(np.int64)
    hf = rng.integers(0, 2, size=(len(fq), 3, 2)).astype(np.int8)
    vlo, vhi = [0, 5, 6, 13], [1, 2, 3, 4, 22]
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(n, n, n, G, nq, np.ones((nq, 3)), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    fine = Fields(T(st0), *[T(x) for x in fb0])
    cb = Fields(T(cst), *[T(x) for x in cfb])
    g.prolong_to_ghosts(fine, cb, kind, T(fq), T(cq), T(el), T(hf), vlo, vhi)
    torch.cuda.synchronize()
    ost = st0.copy()
    _oracle.prolong_cells("orc", kind, n, G, abi.N_EVOL_VARS, ost, cst, fq, cq, el, vlo, vhi)
    ofb = [x.copy() for x in fb0]
    _oracle.prolong_faces("orc", kind, n, G, ofb, cfb, fq, cq, el, hf)
    np.testing.assert_array_equal(fine.state.cpu().numpy(), ost)
    for d in range(3):
        np.testing.assert_array_equal((fine.bx, fine.by, fine.bz)[d].cpu().numpy(), ofb[d])
    assert (ost != st0).any() and all((a != b).any() for a, b in zip(ofb, fb0))
    assert g.status().device_flags == 0


def test_prolonged_ghost_faces_are_divergence_free():
    """Faces, edges and corners of a quadrant prolonged from a divergence-free
    coarse face field (no fine neighbours): every fine ghost cell's div B at
    round-off."""
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(9)
    Ax = rng.standard_normal((NN + 1, NN + 1, NN))
    Ay = rng.standard_normal((NN + 1, NN, NN + 1))
    Az = rng.standard_normal((NN, NN + 1, NN + 1))
    cbx = (Az[:, 1:, :] - Az[:, :-1, :]) - (Ay[1:] - Ay[:-1])
    cby = (Ax[1:] - Ax[:-1]) - (Az[:, :, 1:] - Az[:, :, :-1])
    cbz = (Ay[:, :, 1:] - Ay[:, :, :-1]) - (Ax[:, 1:, :] - Ax[:, :-1, :])
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(N, N, N, G, 1, np.ones((1, 3)), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    st = torch.zeros((1, abi.N_EVOL_VARS, NN, NN, NN), dtype=torch.float64, device=dev)
    fine = Fields(st, *[torch.full((1,) + s, float("nan"), dtype=torch.float64, device=dev) for s in FSH])
    cb = Fields(st.clone(), T(cbx[None]), T(cby[None]), T(cbz[None]))
    for kind in (0, 1, 2):
        el = torch.arange(NELEM[kind], dtype=torch.uint8, device=dev)
        z = torch.zeros(NELEM[kind], dtype=torch.int64, device=dev)
        hf = torch.zeros((NELEM[kind], 3, 2), dtype=torch.int8, device=dev)
        g.prolong_to_ghosts(fine, cb, kind, z, z, el, hf)
    bx, by, bz = (x[0].cpu().numpy() for x in (fine.bx, fine.by, fine.bz))
    div = (bx[:, :, 1:] - bx[:, :, :-1]) + (by[:, 1:, :] - by[:, :-1, :]) + (bz[1:] - bz[:-1])
    ghost = np.ones((NN, NN, NN), bool)
    ghost[G:G + N, G:G + N, G:G + N] = False
    assert np.isfinite(div[ghost]).all()
    assert np.abs(div[ghost]).max() <= 1e-13 * max(np.abs(cbx).max(), np.abs(cby).max(), np.abs(cbz).max())


def test_fmr_operators_replay_in_a_cuda_graph():
    """Restriction into coarse buffers and prolongation into all 26 ghost
    elements launch only kernels and allocate nothing, so they can sit in
    the captured step between the stage and the aux pass: captured once,
    replayed on new data, they give the eager results bit for bit."""
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(77)
    nq = 8
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(N, N, N, G, nq, np.ones((nq, 3)), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    shp = [(nq, abi.N_EVOL_VARS, NN, NN, NN)] + [(nq,) + s for s in FSH]
    fine = Fields(*[torch.empty(s, dtype=torch.float64, device=dev) for s in shp])
    cb = Fields(*[torch.empty(s, dtype=torch.float64, device=dev) for s in shp])
    q = torch.arange(nq, dtype=torch.int64, device=dev)
    child = (q % 8).to(torch.uint8)
    lists = []
    for kind in (0, 1, 2):
        ne = NELEM[kind]
        lists.append((kind, q.repeat_interleave(ne), torch.arange(ne, dtype=torch.uint8, device=dev).repeat(nq),
                      torch.zeros((nq * ne, 3, 2), dtype=torch.int8, device=dev)))
    lo, hi = [0, 5, 6], [1, 2, 3, 4]

    def fmr():
        g.restrict_to_coarse(fine, cb, q, q, child, lo, hi)
        for kind, fq, el, hf in lists:
            g.prolong_to_ghosts(fine, cb, kind, fq, fq, el, hf, lo, hi)

    def load(seed):
        r = np.random.default_rng(seed)
        for t, s in zip((fine.state, fine.bx, fine.by, fine.bz, cb.state, cb.bx, cb.by, cb.bz), shp + shp):
            t.copy_(T(r.standard_normal(s)))

    load(1)
    fmr()  # first calls outside the capture
    load(2)
    fmr()
    torch.cuda.synchronize()
    eager = [x.clone() for x in (fine.state, fine.bx, fine.by, fine.bz, cb.state)]
    graph = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(graph, stream=s):
            fmr()
    torch.cuda.current_stream().wait_stream(s)
    load(2)
    graph.replay()
    torch.cuda.synchronize()
    for a, b in zip((fine.state, fine.bx, fine.by, fine.bz, cb.state), eager):
        assert torch.equal(a, b)
    assert g.status().device_flags == 0
