"""Block partitioning across ranks and the host-side halo exchange of a
brick of same-level blocks (GRACE's MPI domain decomposition of the p4est
forest, src/amr forest.cpp:158-165, reduced to a 1-D slab split along x).
Test infrastructure for the multi-rank CPU tests: host (numpy) arrays over
torch.distributed point-to-point messages (gloo).

Rank r owns the contiguous x-range of block columns [x0, x1); the x-ghosts
at the rank boundary come from the neighbouring rank (one send and one
receive per side), everything else from the rank's own blocks.
"""
import numpy as np

# Message tags by travel direction: a message sent to the left neighbour
# (the sender's low-side interior, which fills the receiver's high ghosts)
# and one sent to the right neighbour (the sender's high-side interior,
# which fills the receiver's low ghosts).  With two ranks and periodic x both
# neighbours are the same rank, so the tag is what tells the two apart.
TAG_LEFTWARD = 0
TAG_RIGHTWARD = 1


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
    ghosts are [nx+g+1, nx+2g+1) (the faces g and nx+g belong to the block).
    One rank with periodic x wraps its own columns locally (no message)."""
    def lo_src(arr, stag):
        s0 = 1 if stag else 0
        return arr[:, :, 0, :, :, :, g + s0:2 * g + s0]

    def hi_src(arr):
        return arr[:, :, nb_local - 1, :, :, :, nx:nx + g]

    def put(arr, stag, side, data):
        if side == "lo":
            arr[:, :, 0, :, :, :, 0:g] = data
        else:
            o = nx + g + (1 if stag else 0)
            arr[:, :, nb_local - 1, :, :, :, o:o + g] = data

    if world == 1:
        if periodic_x:
            for arr, stag in arrays:
                lo, hi = lo_src(arr, stag).copy(), hi_src(arr).copy()
                put(arr, stag, "lo", hi)
                put(arr, stag, "hi", lo)
        return

    import torch
    left = rank - 1 if rank > 0 else (world - 1 if periodic_x else None)
    right = rank + 1 if rank < world - 1 else (0 if periodic_x else None)
    reqs = []
    recv = []
    for arr, stag in arrays:
        if left is not None:
            buf = torch.from_numpy(np.ascontiguousarray(lo_src(arr, stag)))
            reqs.append(dist.isend(buf, left, tag=TAG_LEFTWARD))
            rb = torch.empty_like(buf)
            # the left neighbour's high side, sent rightward
            reqs.append(dist.irecv(rb, left, tag=TAG_RIGHTWARD))
            recv.append((arr, rb, stag, "lo"))
        if right is not None:
            buf = torch.from_numpy(np.ascontiguousarray(hi_src(arr)))
            reqs.append(dist.isend(buf, right, tag=TAG_RIGHTWARD))
            rb = torch.empty_like(buf)
            # the right neighbour's low side, sent leftward
            reqs.append(dist.irecv(rb, right, tag=TAG_LEFTWARD))
            recv.append((arr, rb, stag, "hi"))
    for r in reqs:
        r.wait()
    for arr, rb, stag, side in recv:
        put(arr, stag, side, rb.numpy())
