"""Ghost fill of a brick of blocks (grb_fill_ghosts_brick) against the
oracle's (phys_bc_kernels.hh / copy_kernels.hh restated): every ghost cell
and face of the 7 HRSC variables and the three face-B arrays bit for bit,
for every combination of periodic and outflow axes, on the run-based path
(ghost width 4, interior extents multiples of 4) and the per-cell one."""
import itertools

import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [8, 6])
@pytest.mark.parametrize("periodic", list(itertools.product([False, True], repeat=3)))
def test_fill_ghosts_brick_matches_oracle(n, periodic):
    dev = torch.device("cuda:0")
    su = workloads.BrickSetup((2, 3, 2), (n, n, n), (0.0, 0.0, 0.0), (1.0, 1.5, 1.0), 4, periodic)
    rng = np.random.default_rng(n + 2 * sum(periodic))
    st, bx, by, bz, _ = su.empty()
    arrays = [rng.standard_normal(a.shape) for a in (st, bx, by, bz)]
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(Blocks(n, n, n, su.ngz, su.nq, su.idx(), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    f = Fields(*[T(a) for a in arrays])
    g.fill_ghosts_brick(f, su.nb, su.periodic)
    torch.cuda.synchronize()
    want = [a.copy() for a in arrays]
    _oracle.fill_ghosts("orc", su, want)
    got = [x.cpu().numpy() for x in (f.state, f.bx, f.by, f.bz)]
    # the cell arrays: the 7 HRSC variables are exchanged, the static metric is not
    np.testing.assert_array_equal(got[0][:, :abi.N_HRSC], want[0][:, :abi.N_HRSC])
    for a, b in zip(got[1:], want[1:]):
        np.testing.assert_array_equal(a, b)
