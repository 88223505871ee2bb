"""Two ranks over gloo (CPU): the blast wave on a 4x2x2 brick split into two
x-slabs of blocks, each rank advancing its own blocks with the oracle and
exchanging x-halos between stages, reproduces the single-rank RK3 step bit
for bit, with outflow and with periodic x boundaries (with two ranks both
x-neighbours are the same rank).  Covers the host-side partitioning logic
of N>1 runs."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import _oracle
from grace_b200 import abi, params, workloads
from _slab import exchange_x_halos, split_columns


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


NB = (4, 2, 2)
N = 8
G = 4


def _periodic(su, periodic_x):
    """The same brick with periodic x boundaries when asked."""
    if not periodic_x:
        return su
    return workloads.BrickSetup(su.nb, su.n, su.lo, su.hi, su.ngz, (True, False, False))


def _single(periodic_x=False):
    P = params.blast()
    su, f = workloads.blast(nb=NB, n=(N,) * 3)
    su = _periodic(su, periodic_x)
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, N, N, N, G, su.nq)
    state = [st, bx, by, bz]
    _oracle.fill_ghosts("orc", su, state)
    S.compute_aux(su.idx().copy(), state, aux)
    sp = [x.copy() for x in state]
    spp = [x.copy() for x in state]
    _oracle.rk3_step(S, su, 0.25 / su.idx()[0, 0], state, sp, spp, aux)
    return state


def _view(a, nbx):
    # (nq, ...) with q x-fastest -> (nbz, nby, nbx, nv, NZ, NY, NXa)
    sh = a.shape
    nv = sh[1] if a.ndim == 5 else 1
    return a.reshape(NB[2], NB[1], nbx, nv, *sh[-3:])


def _worker(rank, world, port, out_q, periodic_x=False):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    x0, x1 = split_columns(NB[0], world, rank)
    nbl = x1 - x0
    P = params.blast()
    su, f = workloads.blast(nb=NB, n=(N,) * 3)
    # this rank's blocks: columns x0..x1-1 of every (y, z) row
    qs = [q for q in range(su.nq) if x0 <= q % NB[0] < x1]
    loc = [x[qs].copy() for x in f]
    st, bx, by, bz, aux = loc
    sub = workloads.BrickSetup((nbl, NB[1], NB[2]), (N,) * 3, (-6 + 12 * x0 / NB[0], -6, -6),
                               (-6 + 12 * x1 / NB[0], 6, 6), G, (False, False, False))
    S = _oracle.Stage(P, N, N, N, G, len(qs))
    idx = su.idx()[qs].copy()

    def bc(fields):
        _oracle.fill_ghosts("orc", sub, fields)  # local sweeps (outflow at the rank edges)
        arrs = [(_view(fields[0], nbl)[:, :, :, :abi.N_HRSC], False), (_view(fields[1], nbl), True),
                (_view(fields[2], nbl), False), (_view(fields[3], nbl), False)]
        hrsc = arrs[0][0].copy()
        arrs[0] = (hrsc, False)
        exchange_x_halos(arrs, G, N, nbl, periodic_x, dist, rank, world)
        # the exchanged x-slabs span the neighbour's full y, z extent (its
        # own y and z ghosts included), so edges and corners are right too
        _view(fields[0], nbl)[:, :, :, :abi.N_HRSC] = hrsc

    state = [st, bx, by, bz]
    bc(state)
    S.compute_aux(idx, state, aux)
    sp = [x.copy() for x in state]
    spp = [x.copy() for x in state]
    dt = 0.25 / su.idx()[0, 0]
    S.reset_diag(aux)
    S.advance_substep(idx, dt, 1.0, sp, state, aux)
    bc(sp)
    S.compute_aux(idx, sp, aux)
    S.linop(spp, state, sp, 0.75, 0.25)
    S.advance_substep(idx, dt, 0.25, spp, sp, aux)
    bc(spp)
    S.compute_aux(idx, spp, aux)
    S.linop(state, state, spp, 1.0 / 3, 2.0 / 3.0)
    S.advance_substep(idx, dt, 2.0 / 3.0, state, spp, aux)
    bc(state)
    S.compute_aux(idx, state, aux)
    out_q.put((rank, qs, state[0][:, :7].copy()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("periodic_x", [False, True])
def test_two_rank_slab_split_matches_single_rank(periodic_x):
    ref = _single(periodic_x)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q, periodic_x)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = G
    for rank, qs, st in got:
        a = st[:, :, g:-g, g:-g, g:-g]
        b = ref[0][qs][:, :7, g:-g, g:-g, g:-g]
        bad = [int(np.sum(a[:, v] != b[:, v])) for v in range(7)]
        assert sum(bad) == 0, (rank, bad)


def test_one_rank_periodic_wrap_matches_brick_fill():
    """world == 1 with periodic x: the rank wraps its own edge columns (no
    message), and the x-ghosts equal the oracle's periodic brick fill."""
    su, f = workloads.blast(nb=NB, n=(N,) * 3)
    ref = [x.copy() for x in f[:4]]
    _oracle.fill_ghosts("orc", _periodic(su, True), ref)
    got = [x.copy() for x in f[:4]]
    _oracle.fill_ghosts("orc", su, got)  # outflow everywhere first
    arrs = [(_view(got[0], NB[0])[:, :, :, :abi.N_HRSC], False), (_view(got[1], NB[0]), True),
            (_view(got[2], NB[0]), False), (_view(got[3], NB[0]), False)]
    hrsc = arrs[0][0].copy()
    arrs[0] = (hrsc, False)
    exchange_x_halos(arrs, G, N, NB[0], True, None, 0, 1)
    _view(got[0], NB[0])[:, :, :, :abi.N_HRSC] = hrsc
    assert np.array_equal(got[0][:, :abi.N_HRSC], ref[0][:, :abi.N_HRSC])
    for a, b in zip(got[1:], ref[1:]):
        assert np.array_equal(a, b)
