"""The LLF light-cone floor (rusanov_use_c_limit, grmhd.hh:855-883) in the
oracle: on the blast wave with the limit above the background density the
floor changes the step, so the GPU parity test of the LLF stage with the
floor exercises it (CPU only)."""
import numpy as np

import _oracle
from grace_b200 import abi, params, workloads
from parity import cons_rel_err, interior


def _step(P, su, f, dt):
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq)
    state = [st, bx, by, bz]
    _oracle.fill_ghosts("orc", su, state)
    S.compute_aux(su.idx().copy(), state, aux)
    sp = [x.copy() for x in state]
    spp = [x.copy() for x in state]
    _oracle.rk3_step(S, su, dt, state, sp, spp, aux)
    return state


def test_llf_floor_changes_the_step():
    P = params.blast()
    P.riemann = abi.RIEMANN_LLF
    su, f = workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
    dt = 0.25 / su.idx()[0, 0]
    a = _step(P, su, f, dt)
    P.rusanov_use_c_limit = 1e-3
    b = _step(P, su, f, dt)
    e = cons_rel_err(interior(a[0][:, :7], 4), interior(b[0][:, :7], 4))
    assert e.max() > 1e-8
    # HLLE and LLF differ too
    P.riemann = abi.RIEMANN_HLL
    P.rusanov_use_c_limit = 0.0
    c = _step(P, su, f, dt)
    assert cons_rel_err(interior(a[0][:, :7], 4), interior(c[0][:, :7], 4)).max() > 1e-8
    assert np.all(np.isfinite(a[0]))
