"""Boundary mass outflux (grb_accumulate_boundary_outflow, the reference's
boundary_outflow_t::accumulate) on the GPU: after each substep, the outflux
it accumulates equals minus the change of the total rest mass sum(D) dV that
the same substep's flux update made (the update is a telescoping flux
difference, so the two agree to round-off), plain and tuned."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_outflow_equals_mass_lost_by_the_update(mode):
    dev = torch.device("cuda:0")
    su, f = workloads.blast_drifting()
    P = params.blast()
    st, bx, by, bz, aux = f
    g = GRMHDEquationsSystem(P)
    g.reserve(Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev))
    g.set_mode(mode)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(T(st), T(bx), T(by), T(bz))
    aux_d = T(aux)
    g.fill_ghosts_brick(state, su.nb, su.periodic)
    g.compute_auxiliary_quantities(state, aux_d)
    if mode == abi.MODE_TUNED:
        g.set_tuning(1, 1, 1, 1)
    quad, face = su.outer_faces()
    assert len(quad) == 24  # 8 blocks x 3 outer faces
    dxs = T(np.tile(su.dx, (su.nq, 1)))
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    dt = 0.25 * su.dx[0]
    dV = float(np.prod(su.dx))
    G, n = su.ngz, su.n[0]
    mass = lambda fl: float(fl.state[:, abi.DENS, G:G + n, G:G + n, G:G + n].sum()) * dV
    total = 0.0
    for dtfact in (1.0, 0.25, 2.0 / 3.0):
        new = state.clone()
        m0 = mass(new)
        g.advance_substep(0.0, dt, dtfact, new, state, aux_d)
        before = float(out)
        g.accumulate_boundary_outflow(T(quad), T(face), dxs, dt, dtfact, out)
        torch.cuda.synchronize()
        flux_out = float(out) - before
        dm = mass(new) - m0
        assert abs(flux_out) > 1e-3 * m0 * dtfact * dt  # mass really crosses the boundary
        assert abs(dm + flux_out) <= 1e-12 * m0
        total += flux_out
    assert abs(float(out) - total) <= 1e-15 * abs(total) + 1e-300
    assert g.status().device_flags == 0


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_outflow_matches_oracle(mode):
    """One substep of the drifting blast wave on the GPU and in the oracle:
    the accumulated outflux against the oracle's sum over its own face
    fluxes (the restated accumulate), within 1e-11 relative."""
    dev = torch.device("cuda:0")
    su, f = workloads.blast_drifting()
    P = params.blast()
    st, bx, by, bz, aux = f
    dt, dtfact = 0.25 * su.dx[0], 1.0
    quad, face = su.outer_faces()
    dxs = np.tile(su.dx, (su.nq, 1))
    # oracle
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq)
    old = [x.copy() for x in (st, bx, by, bz)]
    aux_h = aux.copy()
    _oracle.fill_ghosts("orc", su, old)
    S.compute_aux(su.idx().copy(), old, aux_h)
    new = [x.copy() for x in old]
    S.advance_substep(su.idx().copy(), dt, dtfact, new, old, aux_h)
    want = S.boundary_outflow(quad, face, dxs, dt, dtfact)
    # GPU
    g = GRMHDEquationsSystem(P)
    g.reserve(Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev))
    g.set_mode(mode)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(T(st), T(bx), T(by), T(bz))
    aux_d = T(aux)
    g.fill_ghosts_brick(state, su.nb, su.periodic)
    g.compute_auxiliary_quantities(state, aux_d)
    if mode == abi.MODE_TUNED:
        g.set_tuning(1, 1, 1, 1)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    nw = state.clone()
    g.advance_substep(0.0, dt, dtfact, nw, state, aux_d)
    g.accumulate_boundary_outflow(T(quad), T(face), T(dxs), dt, dtfact, out)
    torch.cuda.synchronize()
    assert abs(want) > 0
    assert abs(float(out) - want) <= 1e-11 * abs(want)
