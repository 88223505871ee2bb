"""Interior copies between pinned host memory and the device
(grb_copy_evolved_interior, grb_copy_evolved_packed): exact round trips,
ghost zones untouched, upload + ghost fill equal to copying whole arrays;
the block-range brick fill and the host step pipelined over runs of blocks
(rk3_step_host) equal to their whole-grid, sequential forms bit for bit."""
import numpy as np
import pytest
import torch

from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem

pytestmark = pytest.mark.gpu


def _system(su, P):
    dev = torch.device("cuda:0")
    blocks = Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev)
    g = GRMHDEquationsSystem(P)
    g.reserve(blocks)
    return g, dev


def _interior_masks(su, whole_rows=False):
    """Interior cells / faces of the cell array and the three face arrays;
    whole_rows: the rows of the interior (y, z) range at every x."""
    g = su.ngz
    nx, ny, nz = su.n
    NX, NY, NZ = nx + 2 * g, ny + 2 * g, nz + 2 * g

    def m(shape, stag):
        out = np.zeros(shape, dtype=bool)
        hi = [nz + g, ny + g, nx + g]
        if stag is not None:
            hi[stag] += 1
        out[g:hi[0], g:hi[1], (0 if whole_rows else g):(shape[2] if whole_rows else hi[2])] = True
        return out
    return (m((NZ, NY, NX), None), m((NZ, NY, NX + 1), 2), m((NZ, NY + 1, NX), 1),
            m((NZ + 1, NY, NX), 0))


@pytest.mark.parametrize("nvars", [abi.N_HRSC, abi.N_EVOL_VARS])
def test_interior_round_trip_is_exact(nvars):
    su, f = workloads.blast(nb=(2, 2, 1), n=(8, 8, 8))
    g, dev = _system(su, params.blast())
    rng = np.random.default_rng(7)
    st, bx, by, bz = [np.ascontiguousarray(x) for x in f[:4]]
    dstate = Fields(*[torch.from_numpy(x).to(dev) for x in (st, bx, by, bz)])
    host = Fields(torch.from_numpy(rng.standard_normal((su.nq, nvars) + st.shape[2:])).pin_memory(),
                  *[torch.from_numpy(rng.standard_normal(x.shape)).pin_memory() for x in (bx, by, bz)])
    before = [x.cpu().numpy().copy() for x in (dstate.state, dstate.bx, dstate.by, dstate.bz)]
    g.copy_evolved_interior(host, dstate, to_device=True)
    torch.cuda.synchronize()
    after = [x.cpu().numpy() for x in (dstate.state, dstate.bx, dstate.by, dstate.bz)]
    masks = _interior_masks(su)
    hs = host.state.numpy()
    # cells: HRSC vars take the host interior, everything else is unchanged
    for v in range(abi.N_EVOL_VARS):
        a, b = after[0][:, v], before[0][:, v]
        if v < abi.N_HRSC:
            np.testing.assert_array_equal(a[:, masks[0]], hs[:, v][:, masks[0]])
            np.testing.assert_array_equal(a[:, ~masks[0]], b[:, ~masks[0]])
        else:
            np.testing.assert_array_equal(a, b)
    for a, b, h, m in zip(after[1:], before[1:], (host.bx, host.by, host.bz), masks[1:]):
        np.testing.assert_array_equal(a[:, m], h.numpy()[:, m])
        np.testing.assert_array_equal(a[:, ~m], b[:, ~m])
    # and back into zeroed host arrays: the interior rows at every x
    back = Fields(torch.zeros_like(host.state).pin_memory(), *[torch.zeros_like(x).pin_memory()
                                                              for x in (host.bx, host.by, host.bz)])
    g.copy_evolved_interior(back, dstate, to_device=False)
    torch.cuda.synchronize()
    rows = _interior_masks(su, whole_rows=True)
    bs = back.state.numpy()
    for v in range(nvars):
        exp = after[0][:, v] if v < abi.N_HRSC else np.zeros_like(bs[:, v])
        np.testing.assert_array_equal(bs[:, v][:, rows[0]], exp[:, rows[0]])
        assert not bs[:, v][:, ~rows[0]].any()
    for b, a, m in zip((back.bx, back.by, back.bz), after[1:], rows[1:]):
        np.testing.assert_array_equal(b.numpy()[:, m], a[:, m])
        assert not b.numpy()[:, ~m].any()


def test_upload_and_ghost_fill_equals_whole_copy():
    """The e2e leg's upload (interior copy, then the ghost fill) gives the
    device state, ghosts included, of copying the whole arrays."""
    su, f = workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
    g, dev = _system(su, params.blast())
    st, bx, by, bz = [np.ascontiguousarray(x) for x in f[:4]]
    ref = Fields(*[torch.from_numpy(x).to(dev) for x in (st, bx, by, bz)])
    g.fill_ghosts_brick(ref, su.nb, su.periodic)
    host = Fields(*[x.cpu().pin_memory() for x in (ref.state[:, :abi.N_HRSC].contiguous(), ref.bx, ref.by,
                                                   ref.bz)])
    up = Fields(ref.state.clone(), *[torch.full_like(x, np.nan) for x in (ref.bx, ref.by, ref.bz)])
    up.state[:, :abi.N_HRSC] = np.nan
    g.copy_evolved_interior(host, up, to_device=True)
    g.fill_ghosts_brick(up, su.nb, su.periodic)
    torch.cuda.synchronize()
    for a, b in zip((up.state, up.bx, up.by, up.bz), (ref.state, ref.bx, ref.by, ref.bz)):
        assert torch.equal(a, b)


def test_unpinned_host_arrays_are_rejected():
    su, f = workloads.blast(nb=(1, 1, 1), n=(8, 8, 8))
    g, dev = _system(su, params.blast())
    st, bx, by, bz = [np.ascontiguousarray(x) for x in f[:4]]
    dstate = Fields(*[torch.from_numpy(x).to(dev) for x in (st, bx, by, bz)])
    host = Fields(*[torch.from_numpy(x.copy()) for x in (st, bx, by, bz)])
    with pytest.raises(ValueError):
        g.copy_evolved_interior(host, dstate, to_device=True)


def test_packed_round_trip_is_exact():
    """grb_copy_evolved_packed: the packed host arrays hold exactly the
    interior of the device arrays (download), an upload writes exactly the
    interior back and leaves ghosts and the non-evolved variables alone."""
    su, f = workloads.blast(nb=(2, 2, 1), n=(8, 8, 8))
    g, dev = _system(su, params.blast())
    st, bx, by, bz = [np.ascontiguousarray(x) for x in f[:4]]
    d = Fields(*[torch.from_numpy(x).to(dev) for x in (st, bx, by, bz)])
    host = g.packed_host_fields()
    g.copy_evolved_packed(host, d, to_device=False)
    torch.cuda.synchronize()
    G = su.ngz
    nx, ny, nz = su.n
    np.testing.assert_array_equal(host.state.numpy(), st[:, :abi.N_HRSC, G:G + nz, G:G + ny, G:G + nx])
    np.testing.assert_array_equal(host.bx.numpy(), bx[:, G:G + nz, G:G + ny, G:G + nx + 1])
    np.testing.assert_array_equal(host.by.numpy(), by[:, G:G + nz, G:G + ny + 1, G:G + nx])
    np.testing.assert_array_equal(host.bz.numpy(), bz[:, G:G + nz + 1, G:G + ny, G:G + nx])
    rng = np.random.default_rng(3)
    for h in (host.state, host.bx, host.by, host.bz):
        h.copy_(torch.from_numpy(rng.standard_normal(tuple(h.shape))))
    before = [x.cpu().numpy().copy() for x in (d.state, d.bx, d.by, d.bz)]
    g.copy_evolved_packed(host, d, to_device=True)
    torch.cuda.synchronize()
    after = [x.cpu().numpy() for x in (d.state, d.bx, d.by, d.bz)]
    exp = [before[0].copy(), before[1].copy(), before[2].copy(), before[3].copy()]
    exp[0][:, :abi.N_HRSC, G:G + nz, G:G + ny, G:G + nx] = host.state.numpy()
    exp[1][:, G:G + nz, G:G + ny, G:G + nx + 1] = host.bx.numpy()
    exp[2][:, G:G + nz, G:G + ny + 1, G:G + nx] = host.by.numpy()
    exp[3][:, G:G + nz + 1, G:G + ny, G:G + nx] = host.bz.numpy()
    for a, b in zip(after, exp):
        np.testing.assert_array_equal(a, b)


def test_packed_copy_by_array_on_two_streams():
    """Face B downloaded on a second stream and the cell variables on the
    current one (the e2e leg's overlap) give the one-call download."""
    su, f = workloads.blast(nb=(2, 1, 1), n=(8, 8, 8))
    g, dev = _system(su, params.blast())
    d = Fields(*[torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in f[:4]])
    ref, split = g.packed_host_fields(), g.packed_host_fields()
    for h in (split.state, split.bx, split.by, split.bz):
        h.zero_()
    g.copy_evolved_packed(ref, d, to_device=False)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g.copy_evolved_packed(split, d, to_device=False, stream=side, arrays=(False, True, True, True))
    g.copy_evolved_packed(split, d, to_device=False, arrays=(True, False, False, False))
    torch.cuda.synchronize()
    for a, b in zip((split.state, split.bx, split.by, split.bz), (ref.state, ref.bx, ref.by, ref.bz)):
        assert torch.equal(a, b)


@pytest.mark.parametrize("periodic", [False, True])
def test_block_range_fill_equals_whole_fill(periodic):
    """grb_fill_ghosts_brick_range over consecutive runs of blocks fills
    every ghost exactly as one whole-brick fill."""
    su, f = workloads.blast(nb=(2, 3, 4), n=(8, 8, 8))
    g, dev = _system(su, params.blast())
    rng = np.random.default_rng(11)
    d = Fields(*[torch.from_numpy(rng.standard_normal(x.shape)).to(dev) for x in f[:4]])
    ref = d.clone()
    per = (periodic,) * 3
    g.fill_ghosts_brick(ref, su.nb, per)
    for q0, q1 in ((0, 5), (5, 6), (6, 17), (17, su.nq)):
        g.fill_ghosts_brick(d, su.nb, per, blocks=(q0, q1))
    torch.cuda.synchronize()
    for a, b in zip((d.state, d.bx, d.by, d.bz), (ref.state, ref.bx, ref.by, ref.bz)):
        assert torch.equal(a, b)


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_pipelined_host_step_matches_sequential(mode):
    """GRMHDEquationsSystem.rk3_step_host (upload, fill, primitives, step and
    download pipelined over runs of z-slabs on three streams; also chained,
    each step's uploads overlapping the previous step's tail) gives the bits
    of the sequential host round trip, two steps in a row, in the host
    arrays and in every device array; tuned: the static-metric cache found
    at each run's first block, ranges trimmed to the next stage."""
    from grace_b200.host import brick_runs
    su, f = workloads.blast(nb=(2, 2, 5), n=(8, 8, 8))
    P = params.blast()
    if mode == abi.MODE_TUNED:
        P.ranges = abi.RANGES_NEXT_STAGE
    g, dev = _system(su, P)
    g.set_mode(mode)
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    st0 = Fields(*[T(x) for x in f[:4]])
    bc(st0)
    aux0 = T(f[4])
    g.compute_auxiliary_quantities(st0, aux0)
    if mode == abi.MODE_TUNED:
        g.set_static_metric(st0)
        g.set_tuning(1, 1, 1, 1)
    dt = 0.25 / su.idx()[0, 0]
    runs, deps = brick_runs(su.nb, su.periodic, 3)
    assert len(runs) == 3
    fill_run = lambda fl, s, stream: g.fill_ghosts_brick(fl, su.nb, su.periodic, stream=stream, blocks=runs[s])
    out = []
    io = (torch.cuda.Stream(), torch.cuda.Stream())
    for piped in (False, True, "chained"):
        state, aux = st0.clone(), aux0.clone()
        sp, spp = state.clone(), state.clone()
        host = g.packed_host_fields()
        g.copy_evolved_packed(host, state, to_device=False)
        prev = None
        for _ in range(2):
            if piped == "chained":
                # each step's uploads wait only for the previous step's
                # download of the same run
                prev = g.rk3_step_host(dt, host, state, sp, spp, aux, bc, runs, fill_run, deps, streams=io,
                                       after=prev, wait=False)
            elif piped:
                g.rk3_step_host(dt, host, state, sp, spp, aux, bc, runs, fill_run, deps)
            else:
                g.copy_evolved_packed(host, state, to_device=True)
                bc(state)
                g.compute_auxiliary_quantities(state, aux)
                # rk3_step's entry condition: state_p equals state (whose
                # conserved variables the primitives pass may have rewritten)
                g.linop_apply(sp, state, None, 1.0, 0.0)
                g.rk3_step(dt, state, sp, spp, aux, bc)
                g.copy_evolved_packed(host, state, to_device=False)
        torch.cuda.current_stream().wait_stream(io[1])
        torch.cuda.synchronize()
        out.append([x.clone() for x in (host.state, host.bx, host.by, host.bz, state.state, state.bx, state.by,
                                         state.bz, sp.state, sp.bx, sp.by, sp.bz, aux)])
    assert not torch.equal(out[0][0], torch.from_numpy(f[0][:, :abi.N_HRSC, 4:12, 4:12, 4:12].copy()))
    for other in out[1:]:
        for k, (a, b) in enumerate(zip(out[0], other)):
            assert torch.equal(a, b), k
    assert g.status().device_flags == 0


@pytest.mark.parametrize("alias", [None, "B", "D"])
def test_three_term_linop_matches_numpy(alias):
    """grb_linop_apply3: A = b B + c C + d D over every cell and face of all
    23 variables, the sums left to right; in the -fmad=false build bit for
    bit against the same double-precision expression on the host, in the
    default build (products contracted into FMAs) to 1e-15 of the terms'
    magnitude; also with A aliasing B or D (the reference's integrators
    combine in place)."""
    su, f = workloads.blast(nb=(2, 1, 1), n=(8, 8, 8))
    dev = torch.device("cuda:0")
    blocks = Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev)
    ge = GRMHDEquationsSystem(params.blast(), variant="exact")
    ge.reserve(blocks)
    g, _ = _system(su, params.blast())
    rng = np.random.default_rng(21)
    mk = lambda: Fields(*[torch.from_numpy(rng.standard_normal(x.shape)).to(dev) for x in f[:4]])
    b, c, d = 0.5, -1.0 / 3.0, 2.0 / 7.0
    for sysg, exact in ((ge, True), (g, False)):
        B, C, D = mk(), mk(), mk()
        A = B if alias == "B" else D if alias == "D" else mk()
        host = [[x.cpu().numpy() for x in (F.state, F.bx, F.by, F.bz)] for F in (B, C, D)]
        exp = [b * xb + c * xc + d * xd for xb, xc, xd in zip(*host)]
        scale = [np.abs(b * xb) + np.abs(c * xc) + np.abs(d * xd) for xb, xc, xd in zip(*host)]
        sysg.linop_apply3(A, B, C, D, b, c, d)
        torch.cuda.synchronize()
        for a, e, sc in zip((A.state, A.bx, A.by, A.bz), exp, scale):
            if exact:
                np.testing.assert_array_equal(a.cpu().numpy(), e)
            else:
                assert np.all(np.abs(a.cpu().numpy() - e) <= 1e-15 * sc)
