"""Block partitioning across ranks and the host-side halo exchange of a
brick of same-level blocks (GRACE's MPI domain decomposition of the p4est
forest, src/amr forest.cpp:158-165, reduced to a 1-D slab split along x).

Rank r owns the contiguous x-range of block columns [x0, x1); the x-ghosts
at the rank boundary come from the neighbouring rank through
torch.distributed point-to-point messages (one send and one receive per
side), everything else from the rank's own blocks.  Works with the gloo
backend on host arrays (tests) and with NCCL on device tensors.
"""
import numpy as np


def split_columns(nbx, world, rank):
    """Contiguous x-columns of blocks owned by `rank`."""
    base, extra = divmod(nbx, world)
    x0 = rank * base + min(rank, extra)
    return x0, x0 + base + (1 if rank < extra else 0)


def exchange_x_halos(arrays, g, nx, nb_local, periodic_x, dist, rank, world):
    """Exchange the x-ghost layers of the rank-boundary blocks.

    arrays: list of (array, stag) with array shaped (nbz, nby, nbx_local,
    nv, NZ, NY, NXa) — blocks ordered x-fastest — and stag True for the
    x-staggered face array (NXa = NX+1).  Only the lowest and highest block
    columns of the rank talk to the neighbours; interior columns and the
    domain edges are filled locally beforehand.  Sends the interior layers
    [g, 2g) (low side) and [nx, nx+g) (high side) of the edge columns; for
    the x-staggered array the low-side source is [g+1, 2g+1) and the high
    ghosts are [nx+g+1, nx+2g+1) (the faces g and nx+g belong to the block)."""
    import torch
    left = rank - 1 if rank > 0 else (world - 1 if periodic_x else None)
    right = rank + 1 if rank < world - 1 else (0 if periodic_x else None)
    reqs = []
    recv = []
    for arr, stag in arrays:
        s0 = 1 if stag else 0
        lo_src = arr[:, :, 0, :, :, :, g + s0:2 * g + s0]
        hi_src = arr[:, :, nb_local - 1, :, :, :, nx:nx + g]
        if left is not None:
            buf = torch.from_numpy(np.ascontiguousarray(lo_src))
            reqs.append(dist.isend(buf, left))
            rb = torch.empty_like(buf)
            reqs.append(dist.irecv(rb, left))
            recv.append((arr, 0, rb, stag, "lo"))
        if right is not None:
            buf = torch.from_numpy(np.ascontiguousarray(hi_src))
            reqs.append(dist.isend(buf, right))
            rb = torch.empty_like(buf)
            reqs.append(dist.irecv(rb, right))
            recv.append((arr, nb_local - 1, rb, stag, "hi"))
    for r in reqs:
        r.wait()
    for arr, col, rb, stag, side in recv:
        if side == "lo":
            arr[:, :, col, :, :, :, 0:g] = rb.numpy()
        else:
            o = nx + g + (1 if stag else 0)
            arr[:, :, col, :, :, :, o:o + g] = rb.numpy()
