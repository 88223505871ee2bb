"""The scratch-free stage entry point, grb_advance_substep_static.

Some callers cannot call cudaMalloc — a host code whose GPU memory is
owned up front by a pooling allocator, or a plugin host that forbids a
library to allocate device memory after start-up.  For them the library
exports a variant of the stage whose scratch lives in a fixed file-scope
device array.  This test calls it through the C ABI on two consecutive
stages and checks the new state against the handle-based
grb_advance_substep on the same inputs (same kernels: within the 1e-10
stage tolerance, in practice bit for bit), with the Gardiner-Stone EMF and
FOFC and with the UCT EMF (whose chunks hold the face velocities instead of
the face and cell-centred E).  The grid has more blocks than one pass over
the static array holds, so the chunked path is exercised.  One 16^3 block
(the benchmark's block size) is also compared with the CPU oracle.
The file sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import ctypes

import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import _lib, abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem
from parity import cons_rel_err, interior

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _static_stage(lib, P, blocks, dt, dtfact, new, old, aux):
    g = blocks.c()
    nf, of = new.c(), old.c()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.grb_advance_substep_static(ctypes.byref(P), ctypes.byref(g), 0.0, dt, dtfact,
                                          ctypes.byref(nf), ctypes.byref(of),
                                          ctypes.c_void_p(aux.data_ptr()), s)


@pytest.mark.parametrize("emf", [abi.EMF_GS, abi.EMF_UCT])
def test_static_scratch_stage_matches_handle_stage(emf):
    lib = _lib.load()
    dev = torch.device("cuda:0")
    P = params.blast()
    if emf == abi.EMF_GS:
        P.max_sigma = 100.0  # keeps FOFC busy on this setup (see test_gpu_stage)
    else:
        P.emf, P.fofc_enable = abi.EMF_UCT, 0  # FOFC needs the GS EMF
    su, (st, bx, by, bz, aux) = workloads.blast(nb=(4, 4, 4), n=(8, 8, 8))
    # 64 blocks of 8^3 need ~83 MB (GS) / ~92 MB (UCT) of scratch: more than
    # one pass of the array
    per_block = 8 * (17 ** 3) * ((21 + 6 + 3) if emf == abi.EMF_GS else (21 + 12 + 3))
    assert su.nq * per_block > abi.STATIC_SCRATCH_BYTES
    blocks = Blocks(8, 8, 8, 4, su.nq, su.idx(), device=dev)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    ref = GRMHDEquationsSystem(P)
    ref.reserve(blocks)
    base = Fields(T(st), T(bx), T(by), T(bz))
    aux_d = T(aux)
    ref.fill_ghosts_brick(base, su.nb, su.periodic)
    ref.compute_auxiliary_quantities(base, aux_d)
    dt = 0.25 / su.idx()[0, 0]
    # two consecutive stages: u1 = u0 + dt L(u0), then 3/4 u0 + 1/4 u1 + 1/4 dt L(u1)
    a_old, b_old = base.clone(), base.clone()
    aux_a, aux_b = aux_d.clone(), aux_d.clone()
    for dtfact in (1.0, 0.25):
        a_new, b_new = a_old.clone(), b_old.clone()
        ref.advance_substep(0.0, dt, dtfact, a_new, a_old, aux_a)
        rc = _static_stage(lib, P, blocks, dt, dtfact, b_new, b_old, aux_b)
        assert rc == abi.OK
        torch.cuda.synchronize()
        ga = a_new.state.cpu().numpy()[:, :7]
        gb = b_new.state.cpu().numpy()[:, :7]
        e = cons_rel_err(interior(gb, 4), interior(ga, 4))
        assert e.max() < TOL, e
        for x, y in ((a_new.bx, b_new.bx), (a_new.by, b_new.by), (a_new.bz, b_new.bz)):
            d = (x - y).abs().max().item() / max(x.abs().max().item(), 1e-300)
            assert d < TOL
        # next stage starts from the states just produced
        for f, au in ((a_new, aux_a), (b_new, aux_b)):
            ref.fill_ghosts_brick(f, su.nb, su.periodic)
            ref.compute_auxiliary_quantities(f, au)
        a_old, b_old = a_new, b_new


def test_static_scratch_stage_on_a_16cubed_block_matches_oracle():
    """One substep of one 16^3 block of the blast wave (GS + FOFC) through the
    scratch-free entry point, twice in a row on the same inputs (the array
    keeps the first call's contents: the second must not depend on them),
    against the CPU oracle's advance_substep.  The input is the state after
    one RK3 step of the oracle, where FOFC recomputes ~1200 faces."""
    lib = _lib.load()
    dev = torch.device("cuda:0")
    P = params.blast()
    P.max_sigma = 100.0
    su, f = workloads.blast(nb=(1, 1, 1), n=(16, 16, 16), lo=(-1.5,) * 3, hi=(1.5,) * 3)
    old = [x.copy() for x in f[:4]]
    aux = f[4].copy()
    S = _oracle.Stage(P, 16, 16, 16, 4, 1)
    _oracle.fill_ghosts("orc", su, old)
    S.compute_aux(su.idx().copy(), old, aux)
    dt = 0.25 / su.idx()[0, 0]
    sp, spp = [x.copy() for x in old], [x.copy() for x in old]
    _oracle.rk3_step(S, su, dt, old, sp, spp, aux)
    new_h = [x.copy() for x in old]
    S.advance_substep(su.idx().copy(), dt, 1.0, new_h, old, aux)
    assert S.fofc_counts()[0] > 0
    blocks = Blocks(16, 16, 16, 4, 1, su.idx(), device=dev)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    o = Fields(*[T(x) for x in old])
    aux_d = T(aux)
    for _ in range(2):
        n = o.clone()
        assert _static_stage(lib, P, blocks, dt, 1.0, n, o, aux_d) == abi.OK
        torch.cuda.synchronize()
        e = cons_rel_err(interior(n.state.cpu().numpy()[:, :7], 4), interior(new_h[0][:, :7], 4))
        assert e.max() < TOL, e
        for x, y in zip((n.bx, n.by, n.bz), new_h[1:]):
            d = np.max(np.abs(x.cpu().numpy() - y)) / max(np.max(np.abs(y)), 1e-300)
            assert d < TOL


def test_static_scratch_rejects_oversized_blocks():
    lib = _lib.load()
    P = params.blast()
    dev = torch.device("cuda:0")
    n = 64  # one 64^3 block with 4 ghosts needs ~93 MB of scratch
    idx = torch.ones(3, dtype=torch.float64, device=dev)
    g = abi.Grid(n, n, n, 4, 1, idx.data_ptr(), None)
    dummy = torch.zeros(8, dtype=torch.float64, device=dev)
    f = abi.Fields(dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr())
    rc = lib.grb_advance_substep_static(ctypes.byref(P), ctypes.byref(g), 0.0, 1e-3, 1.0,
                                        ctypes.byref(f), ctypes.byref(f),
                                        ctypes.c_void_p(dummy.data_ptr()), None)
    assert rc == abi.ERR_INVALID
