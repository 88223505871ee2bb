"""Refluxing in the oracle (CPU), on the two-level FMR case of fmr_case.py.

The reference's own refluxing (src/evolution/refluxing.cpp) needs the p4est
ghost layer and MPI, so it is not compiled in place; its properties are what
pins the restatement, as the reference's test_flux_reflux.cpp and
test_ct_flux_conservation.cpp check them:
  * with the coarse fluxes on hanging faces replaced by the fine ones, the
    total mass over the leaves of a periodic hierarchy is conserved to
    round-off through a substep (and is not without refluxing);
  * with the edge EMFs of the interface made to agree, every coarse face on
    an interface keeps the mean of the 4 fine faces it covers (the magnetic
    flux through the interface is the same from both sides) through a
    substep (and does not without refluxing).
"""
import numpy as np

import _oracle
from fmr_case import hanging_face_mismatch, interior_mass, two_level_case


def _substep(reflux):
    H, P, f = two_level_case()
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, H.n, H.n, H.n, H.ngz, H.nq)
    R = H.reflux_lists()
    if reflux:
        S.set_reflux(R)
    idx = H.idx()
    old = [st, bx, by, bz]
    S.compute_aux(idx.copy(), old, aux)
    new = [x.copy() for x in old]
    dt = 0.25 / idx[:, 0].max()
    S.advance_substep(idx.copy(), dt, 1.0, new, old, aux)
    return H, R, old, new


def test_reflux_conserves_mass_and_interface_flux():
    H, R, old, new = _substep(True)
    m0, m1 = interior_mass(H, old[0]), interior_mass(H, new[0])
    assert abs(m1 - m0) <= 1e-14 * m0, (m0, m1)
    assert hanging_face_mismatch(H, R, old) == 0.0  # uniform field to start
    assert hanging_face_mismatch(H, R, new) < 1e-14


def test_without_reflux_the_interfaces_leak():
    H, R, old, new = _substep(False)
    m0, m1 = interior_mass(H, old[0]), interior_mass(H, new[0])
    assert abs(m1 - m0) > 1e-10 * m0
    assert hanging_face_mismatch(H, R, new) > 1e-10


def test_reflux_lists_of_the_two_level_case():
    """6 hanging faces (each face of the refined block), 12 hanging edges
    along its edges (one fine side, three coarse sides) and 12 middle lines
    (one coarse side with its offset, two fine sides), 30 same-level faces
    and 18 same-level edges."""
    H, _, _ = two_level_case()
    R = H.reflux_lists()
    assert len(R["face_coarse_q"]) == 6 and len(R["same_face_q"]) == 60
    ns = R["edge_nsides"]
    assert list(ns).count(4) == 12 and list(ns).count(3) == 12
    fine = R["edge_is_fine"].reshape(-1, 4)
    assert np.all(fine[ns == 4].sum(1) == 1) and np.all(fine[ns == 3].sum(1) == 2)
    off = R["edge_off"].reshape(-1, 4, 2)
    assert np.all(off[ns == 3][:, 0].sum(1) == 1) and np.all(off[ns == 4] == 0)
    assert len(R["same_edge_nsides"]) == 18
