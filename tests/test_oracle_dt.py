"""The oracle's restated find_stable_timestep_impl against the same loop
driven by the reference's own EOS and characteristic-speed kernels
(oracle/_ref, built where the GRACE sources are present)."""
import numpy as np
import pytest

import _oracle
from grace_b200 import params, workloads


@pytest.mark.parametrize("name", ["blast", "balsara"])
def test_find_stable_timestep_matches_reference_numerics(name):
    if _oracle.lib("ref") is None:
        pytest.skip("pinning build oracle/_ref not present")
    if name == "blast":
        P, (su, f) = params.blast(), workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
    else:
        P, (su, f) = params.balsara1(), workloads.balsara1(nb=(4, 1, 1), n=(8, 8, 8))
    out = {}
    for which in ("orc", "ref"):
        st, bx, by, bz, aux = [x.copy() for x in f]
        S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq, which)
        state = [st, bx, by, bz]
        _oracle.fill_ghosts(which, su, state)
        S.compute_aux(su.idx().copy(), state, aux)
        out[which] = S.find_stable_timestep(state, aux, np.ascontiguousarray(1.0 / su.idx()), 0.4)
    assert out["orc"] == out["ref"]
    assert 0.0 < out["orc"] < 1.0
