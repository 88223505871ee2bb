"""Refluxing on the GPU (grb_set_reflux) against the oracle on the two-level
FMR case of fmr_case.py: one substep with the hanging-face fluxes and the
interface EMFs corrected, plain and tuned; the state within the step
tolerance of the oracle's, the leaves' total mass conserved to round-off,
and every coarse face on an interface equal to the mean of the 4 fine faces
it covers."""
import numpy as np
import pytest
import torch

import _oracle
from fmr_case import hanging_face_mismatch, interior_mass, two_level_case
from grace_b200 import abi
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem
from parity import cons_rel_err, interior

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_reflux_substep_matches_oracle_and_conserves(mode):
    H, P, f = two_level_case()
    R = H.reflux_lists()
    idx = H.idx()
    dt = 0.25 / idx[:, 0].max()
    # oracle
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, H.n, H.n, H.n, H.ngz, H.nq)
    S.set_reflux(R)
    old = [st, bx, by, bz]
    S.compute_aux(idx.copy(), old, aux)
    onew = [x.copy() for x in old]
    S.advance_substep(idx.copy(), dt, 1.0, onew, old, aux)
    # GPU
    dev = torch.device("cuda:0")
    g = GRMHDEquationsSystem(P)
    g.reserve(Blocks(H.n, H.n, H.n, H.ngz, H.nq, idx, device=dev))
    g.set_mode(mode)
    if mode == abi.MODE_TUNED:
        g.set_tuning(1, 1, 1, 1)
    g.set_reflux(R)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    gold = Fields(*[T(x) for x in f[:4]])
    aux_d = T(f[4])
    g.compute_auxiliary_quantities(gold, aux_d)
    gnew = gold.clone()
    g.advance_substep(0.0, dt, 1.0, gnew, gold, aux_d)
    torch.cuda.synchronize()
    gs = [x.cpu().numpy() for x in (gnew.state, gnew.bx, gnew.by, gnew.bz)]
    e = cons_rel_err(interior(gs[0][:, :7], H.ngz), interior(onew[0][:, :7], H.ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], onew[1:]):
        assert np.max(np.abs(a - b)) < STEP_TOL * np.max(np.abs(b))
    m0, m1 = interior_mass(H, f[0]), interior_mass(H, gs[0])
    assert abs(m1 - m0) <= 1e-14 * m0, (m0, m1)
    assert hanging_face_mismatch(H, R, gs) < 1e-14
    assert g.status().device_flags == 0
    # refluxing off again: the interfaces leak as in the oracle without it
    g.set_reflux(None)
    gnew2 = gold.clone()
    g.advance_substep(0.0, dt, 1.0, gnew2, gold, aux_d)
    torch.cuda.synchronize()
    assert abs(interior_mass(H, gnew2.state.cpu().numpy()) - m0) > 1e-10 * m0
