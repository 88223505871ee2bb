"""The -fmad=false build of the library (libgrace_b200_exact.so: every
multiply and add rounded on its own, as the CPU oracle is compiled with
-ffp-contract=off) against the oracle.  With the two sides rounding alike,
the c2p's error bits and the stage's C2P_ERR flags and FOFC counts must
agree on every state and cell: a flag that flips here is a logic
difference, not an FMA contraction.  The remaining value differences come
from the math functions (pow, log, exp of CUDA and of the C library may
differ in the last bit)."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem
from parity import cons_rel_err, interior, prim_tol, state_residual

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("preset", ["c2p_bench", "blast"])
def test_exact_build_c2p_error_bits_match_oracle_everywhere(preset):
    P = getattr(params, preset)()
    cons, _ = workloads.c2p_states(50000, seed=11)
    dev = torch.device("cuda:0")
    g = GRMHDEquationsSystem(P, variant="exact")
    c_d = torch.from_numpy(np.ascontiguousarray(cons)).to(dev)
    err_d = torch.zeros(cons.shape[1], dtype=torch.int32, device=dev)
    pr_g = g.conservs_to_prims(c_d, err=err_d).cpu().numpy()
    err_g = err_d.cpu().numpy().view(np.uint32)
    pr_o, _, err_o, _, _, _ = _oracle.c2p_batch(P, cons)
    bad = np.flatnonzero(err_g != err_o)
    assert bad.size == 0, [(int(i), hex(err_g[i]), hex(err_o[i])) for i in bad[:10]]
    res = state_residual(pr_g, pr_o)
    assert np.all(res < prim_tol(pr_o)), res.max()
    same = np.all(pr_g[:12] == pr_o[:12], axis=0)
    print(f"{preset}: {same.mean():.4f} of the states bit for bit, max residual {res.max():.2e}")


@pytest.mark.parametrize("name", ["blast", "balsara"])
def test_exact_build_stage_flags_match_oracle_everywhere(name):
    """One SSP-RK3 step in the plain mode of the exact build: C2P_ERR on
    every cell of every block and the FOFC counts equal the oracle's."""
    if name == "blast":
        P = params.blast()
        P.max_sigma = 100.0  # FOFC busy (see test_gpu_stage)
        su, f = workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
        dt = 0.25 / su.idx()[0, 0]
    else:
        P = params.balsara1()
        su, f = workloads.balsara1(nb=(4, 1, 1), n=(8, 8, 8))
        dt = 0.4 / su.idx()[0, 0]
    dev = torch.device("cuda:0")
    g = GRMHDEquationsSystem(P, variant="exact")
    g.reserve(Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    st, bx, by, bz, aux = f
    state = Fields(T(st), T(bx), T(by), T(bz))
    aux_d = T(aux)
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)
    bc(state)
    g.compute_auxiliary_quantities(state, aux_d)
    sp, spp = state.clone(), state.clone()
    g.rk3_step(dt, state, sp, spp, aux_d, bc)
    torch.cuda.synchronize()
    ga = aux_d.cpu().numpy()
    # oracle
    ost = [x.copy() for x in (st, bx, by, bz)]
    oa = aux.copy()
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq)
    _oracle.fill_ghosts("orc", su, ost)
    S.compute_aux(su.idx().copy(), ost, oa)
    osp = [x.copy() for x in ost]
    ospp = [x.copy() for x in ost]
    _oracle.rk3_step(S, su, dt, ost, osp, ospp, oa)
    np.testing.assert_array_equal(ga[:, abi.C2P_ERR], oa[:, abi.C2P_ERR])
    st_ = g.status()
    assert (st_.fofc_faces, st_.fofc_edges) == S.fofc_counts()
    e = cons_rel_err(interior(state.state.cpu().numpy()[:, :7], su.ngz), interior(ost[0][:, :7], su.ngz))
    assert e.max() < 1e-10, e
    print(f"{name}: exact build, max state-normalised difference {e.max():.2e}")
