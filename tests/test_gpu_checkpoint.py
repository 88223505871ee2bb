"""Restart from a checkpoint on the GPU: two SSP-RK3 steps of the blast
wave, a checkpoint, two more steps; against loading the checkpoint into
fresh arrays, refilling the ghost zones and recomputing the primitives (as
GRACE does after loading) and stepping twice: the same bits in every array,
plain and tuned (the uninterrupted run refills and recomputes at the same
point, which is what a restart changes)."""
import numpy as np
import pytest
import torch

from grace_b200 import abi, params, workloads
from grace_b200.checkpoint import load_checkpoint, save_checkpoint
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_restart_continues_bit_for_bit(mode, tmp_path):
    su, f = workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
    dev = torch.device("cuda:0")
    blocks = Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev)
    g = GRMHDEquationsSystem(params.blast())
    g.reserve(blocks)
    g.set_mode(mode)
    if mode == abi.MODE_TUNED:
        g.set_tuning(1, 1, 1, 1)
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(*[T(x) for x in f[:4]])
    aux = T(f[4])
    bc(state)
    g.compute_auxiliary_quantities(state, aux)
    sp, spp = state.clone(), state.clone()
    dt = 0.25 / su.idx()[0, 0]

    def restart_point(st, sp_, ax):
        bc(st)
        g.compute_auxiliary_quantities(st, ax)
        g.linop_apply(sp_, st, None, 1.0, 0.0)

    for _ in range(2):
        g.rk3_step(dt, state, sp, spp, aux, bc)
    path = save_checkpoint(str(tmp_path), state, time=2 * dt, iteration=2, extents=((-6, 6),) * 3)
    # uninterrupted
    restart_point(state, sp, aux)
    for _ in range(2):
        g.rk3_step(dt, state, sp, spp, aux, bc)
    # restarted into fresh arrays
    r = blocks.new_fields()
    raux = torch.zeros_like(aux)
    t, it, _, _ = load_checkpoint(path, r)
    assert it == 2 and t == 2 * dt
    rsp, rspp = r.clone(), r.clone()
    restart_point(r, rsp, raux)
    for _ in range(2):
        g.rk3_step(dt, r, rsp, rspp, raux, bc)
    torch.cuda.synchronize()
    for a, b in zip((state.state, state.bx, state.by, state.bz), (r.state, r.bx, r.by, r.bz)):
        assert torch.equal(a, b)
    assert g.status().device_flags == 0
