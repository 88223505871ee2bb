"""Balsara-1 to its final time on the GPU against the reference's own
numerics on the CPU (oracle/_ref: the reference's EOS, c2p, reconstruction,
Riemann and EMF kernels in the restated loops), with the adaptive time
step of evolve_impl (find_stable_timestep after every step, CFL 0.4).
Criterion: density L1 difference at t_end <= 1e-8 relative.  Reduced to
256 x 16 x 16 cells (16 blocks of 16^3) so that the CPU side takes seconds."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem

pytestmark = pytest.mark.gpu

T_END, CFL = 0.4, 0.4


def _run_gpu(P, su, f, mode):
    dev = torch.device("cuda:0")
    st, bx, by, bz, aux = f
    blocks = Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev)
    g = GRMHDEquationsSystem(P)
    g.reserve(blocks)
    g.set_mode(mode)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(T(st), T(bx), T(by), T(bz))
    aux_d = T(aux)
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)
    bc(state)
    g.compute_auxiliary_quantities(state, aux_d)
    sp, spp = state.clone(), state.clone()
    if mode == abi.MODE_TUNED:
        g.autotune(sp, state, aux_d)
    dx = T(1.0 / su.idx())
    dt_d = torch.zeros(1, dtype=torch.float64, device=dev)
    g.find_stable_timestep(state, aux_d, dx, CFL, dt_d)
    t, steps = 0.0, 0
    while t < T_END - 1e-15:
        dt = min(dt_d.item(), T_END - t)
        g.rk3_step(dt, state, sp, spp, aux_d, bc, next_dt=(dx, CFL, dt_d))
        t += dt
        steps += 1
    torch.cuda.synchronize()
    assert g.status().device_flags == 0
    return aux_d.cpu().numpy(), steps


def _run_ref(P, su, f):
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq, "ref")
    state = [st, bx, by, bz]
    _oracle.fill_ghosts("ref", su, state)
    S.compute_aux(su.idx().copy(), state, aux)
    sp = [x.copy() for x in state]
    spp = [x.copy() for x in state]
    dx = np.ascontiguousarray(1.0 / su.idx())
    dtn = S.find_stable_timestep(state, aux, dx, CFL)
    t, steps = 0.0, 0
    while t < T_END - 1e-15:
        dt = min(dtn, T_END - t)
        _oracle.rk3_step(S, su, dt, state, sp, spp, aux, "ref")
        dtn = S.find_stable_timestep(state, aux, dx, CFL)
        t += dt
        steps += 1
    return aux, steps


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_balsara1_density_l1_at_t_end(mode):
    if _oracle.lib("ref") is None:
        pytest.skip("pinning build oracle/_ref not present")
    P = params.balsara1()
    su, f = workloads.balsara1(nb=(16, 1, 1), n=(16, 16, 16))
    ag, ng = _run_gpu(P, su, f, mode)
    ar, nr = _run_ref(P, su, f)
    assert ng == nr
    g = su.ngz
    rg = ag[:, abi.RHO, g:-g, g:-g, g:-g]
    rr = ar[:, abi.RHO, g:-g, g:-g, g:-g]
    l1 = np.sum(np.abs(rg - rr)) / np.sum(np.abs(rr))
    print(f"Balsara-1 t={T_END}: {ng} steps, density L1 rel {l1:.3e}")
    assert l1 <= 1e-8, l1
    # the shock tube evolved: the density range spans the fan
    assert rr.max() > 0.9 and rr.min() < 0.2


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_balsara1_configured_size_density_l1_against_reference_fixture(mode):
    """Balsara-1 at its configured size, 1024 x 16 x 16 cells (64 blocks of
    16^3), to t = 0.4 on the GPU against the reference's own numerics run to
    the same time (tests/golden/balsara1024_ref.npz, made by
    tests/golden/make_balsara1024.py with the pinning build: 1006 steps; the
    reference's density does not vary across the periodic y, z directions,
    to the bit, so one x-line stands for the whole field): the same step
    count and density L1 difference <= 1e-8 relative."""
    import os
    fx = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "balsara1024_ref.npz"))
    assert float(fx["transverse_spread"]) == 0.0
    P = params.balsara1()
    su, f = workloads.balsara1(nb=(64, 1, 1), n=(16, 16, 16))
    ag, ng = _run_gpu(P, su, f, mode)
    assert ng == int(fx["steps"])
    g = su.ngz
    rg = ag[:, abi.RHO, g:-g, g:-g, g:-g]                    # (64, nz, ny, nx)
    line = fx["rho_line"].reshape(64, 1, 1, 16)
    l1 = np.sum(np.abs(rg - line)) / np.sum(np.abs(np.broadcast_to(line, rg.shape)))
    print(f"Balsara-1 1024x16x16 t=0.4: {ng} steps, density L1 rel {l1:.3e}")
    assert l1 <= 1e-8, l1
