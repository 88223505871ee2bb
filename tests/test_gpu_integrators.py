"""The other explicit time integrators of evolve_impl on the GPU (forward
Euler, midpoint RK2 and the four-stage low-storage rk4 branch,
evolve.cpp:173-189 and 226-332, GRMHDEquationsSystem.euler_step /
rk2_step / rk4_step) against the oracle stepped in the same order: one
step of the blast wave on a 2^3 brick of 8^3 blocks, plain and tuned, the
state within the step tolerance, div B at round-off."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem
from parity import cons_rel_err, interior

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10


def _oracle_step(name, S, su, dt, st, aux):
    idx = su.idx()
    bc = lambda f: _oracle.fill_ghosts("orc", su, f)
    sub = lambda new, old, fact: S.advance_substep(idx.copy(), dt, fact, new, old, aux)
    auxp = lambda f: S.compute_aux(idx.copy(), f, aux)
    sp = [x.copy() for x in st]
    S.reset_diag(aux)
    if name == "euler":
        sub(st, sp, 1.0); bc(st); auxp(st)
    elif name == "rk2":
        sub(sp, st, 0.5); bc(sp); auxp(sp)
        sub(st, sp, 1.0); bc(st); auxp(st)
    else:
        s1, s2, s3 = st, sp, [x.copy() for x in st]
        (d1, g11, g21, b1), (d2, g12, g22, b2), (d3, g13, g23, b3), (d4, g14, g24, b4) = \
            GRMHDEquationsSystem.RK4_COEFFS
        S.linop(s3, s1, s2, g11, g21); sub(s3, s1, b1); bc(s3); auxp(s3)
        S.linop(s2, s2, s3, 1.0, d2); S.linop(s1, s3, s2, g12, g22); sub(s1, s3, b2); bc(s1); auxp(s1)
        S.linop(s2, s2, s1, 1.0, d3); S.linop(s3, s1, s2, g13, g23); sub(s3, s1, b3); bc(s3); auxp(s3)
        S.linop(s1, s3, s2, g14, g24); sub(s1, s3, b4); bc(s1); auxp(s1)
    return st


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
@pytest.mark.parametrize("name", ["euler", "rk2", "rk4"])
def test_integrator_step_matches_oracle(name, mode):
    P = params.blast()
    su, f = workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
    dt = 0.25 / su.idx()[0, 0]
    # oracle
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq)
    ost = [st, bx, by, bz]
    _oracle.fill_ghosts("orc", su, ost)
    S.compute_aux(su.idx().copy(), ost, aux)
    ost = _oracle_step(name, S, su, dt, ost, aux)
    # GPU
    dev = torch.device("cuda:0")
    g = GRMHDEquationsSystem(P)
    g.reserve(Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev))
    g.set_mode(mode)
    if mode == abi.MODE_TUNED:
        g.set_tuning(1, 1, 1, 1)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(*[T(x) for x in f[:4]])
    gaux = T(f[4])
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)
    bc(state)
    g.compute_auxiliary_quantities(state, gaux)
    sp = state.clone()
    if name == "euler":
        g.euler_step(dt, state, sp, gaux, bc)
    elif name == "rk2":
        g.rk2_step(dt, state, sp, gaux, bc)
    else:
        g.rk4_step(dt, state, sp, state.clone(), gaux, bc)
    torch.cuda.synchronize()
    gs = [x.cpu().numpy() for x in (state.state, state.bx, state.by, state.bz)]
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(ost[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], ost[1:]):
        assert np.max(np.abs(a - b)) <= STEP_TOL * np.max(np.abs(b))
    ga = gaux.cpu().numpy()
    bmax = max(np.max(np.abs(x)) for x in gs[1:])
    assert np.max(np.abs(interior(ga[:, abi.BDIV], su.ngz))) * su.dx[0] < 1e-13 * bmax
    assert torch.equal(sp.state, state.state)
    assert g.status().device_flags == 0
