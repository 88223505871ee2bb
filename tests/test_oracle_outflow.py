"""The oracle's restated outflow accumulation (boundary_outflow_t::
accumulate): on the oracle's own substep it equals minus the change of the
total rest mass (the update is a telescoping flux difference), and it is
the same sum over the pinning build's fluxes (the reference's numerics)."""
import os

import numpy as np
import pytest

import _oracle
from grace_b200 import abi, params, workloads


def _substep(which):
    su, (st, bx, by, bz, aux) = workloads.blast_drifting()
    P = params.blast()
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq, which)
    old = [x.copy() for x in (st, bx, by, bz)]
    _oracle.fill_ghosts(which, su, old)
    S.compute_aux(su.idx().copy(), old, aux)
    new = [x.copy() for x in old]
    dt = 0.25 * su.dx[0]
    S.advance_substep(su.idx().copy(), dt, 1.0, new, old, aux)
    quad, face = su.outer_faces()
    out = S.boundary_outflow(quad, face, np.tile(su.dx, (su.nq, 1)), dt, 1.0)
    G, n = su.ngz, su.n[0]
    dV = float(np.prod(su.dx))
    mass = lambda s: float(s[:, abi.DENS, G:G + n, G:G + n, G:G + n].sum()) * dV
    return out, mass(old[0]), mass(new[0])


def test_oracle_outflow_balances_the_mass_change():
    out, m0, m1 = _substep("orc")
    assert abs(out) > 1e-6 * m0
    assert abs((m1 - m0) + out) <= 1e-12 * m0


@pytest.mark.skipif(not os.path.exists(_oracle.REF), reason="pinning build absent")
def test_outflow_on_the_reference_numerics():
    a = _substep("orc")[0]
    b = _substep("ref")[0]
    assert abs(a - b) <= 1e-13 * abs(b)
