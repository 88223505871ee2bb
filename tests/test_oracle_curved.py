"""Curved-metric Cowling stage on the CPU: the oracle's restated loops and
geometric sources against the same loops on the reference's own kernels
(oracle/_ref), one SSP-RK3 step on Schwarzschild in Kerr-Schild coordinates
(tests/curved.py)."""
import numpy as np
import pytest

import _oracle
from curved import curved_setup
from grace_b200 import abi
from parity import cons_rel_err, interior


@pytest.mark.parametrize("emf", [abi.EMF_GS, abi.EMF_UCT])
def test_curved_step_restated_vs_reference_numerics(emf):
    if _oracle.lib("ref") is None:
        pytest.skip("pinning build oracle/_ref not present")
    P, su, f = curved_setup(emf=emf, fofc=1 if emf == abi.EMF_GS else 0)
    out = {}
    for which in ("orc", "ref"):
        st, bx, by, bz, aux = [x.copy() for x in f]
        S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq, which)
        state = [st, bx, by, bz]
        _oracle.fill_ghosts(which, su, state)
        S.compute_aux(su.idx().copy(), state, aux)
        sp = [x.copy() for x in state]
        spp = [x.copy() for x in state]
        _oracle.rk3_step(S, su, 0.25 / su.idx()[0, 0], state, sp, spp, aux, which)
        out[which] = (state, aux)
    (so, ao), (sr, ar) = out["orc"], out["ref"]
    e = cons_rel_err(interior(so[0][:, :7], su.ngz), interior(sr[0][:, :7], su.ngz))
    assert e.max() < 1e-12, e
    # the step moved the matter (sources and fluxes active)
    e0 = cons_rel_err(interior(so[0][:, :7], su.ngz), interior(f[0][:, :7], su.ngz))
    assert e0.max() > 1e-6
    for a, b in zip(so[1:], sr[1:]):
        assert np.max(np.abs(a - b)) <= 1e-12 * max(np.max(np.abs(b)), 1e-300)
