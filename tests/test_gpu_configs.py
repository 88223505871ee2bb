"""The FMR configurations on the GPU against the oracle: the magnetised TOV
star on its five-level hierarchy (grace_b200.workloads.tov_hierarchy,
32/224/224/224/256 blocks per level) and the Fishbone-Moncrief torus in
Kerr-Schild on its four-level one (torus_hierarchy, 32/224/184/576), with
8^3 blocks, through one SSP-RK3 step of the
stage with refluxing (grb_set_reflux) and the gather-map ghost fill between
stages (grb_fill_ghosts_gather); the oracle runs the same step with the
same descriptor lists and the host fill of the same maps (the TOV star
also with the benchmark's 16^3 blocks).  The device gather fill itself
matches the host fill bit for bit."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem
from parity import cons_rel_err, interior

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10


def _oracle_rk3(S, H, idx, dt, state, aux):
    bc = lambda f: H.fill_ghosts(*f)
    sp = [x.copy() for x in state]
    spp = [x.copy() for x in state]
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


def _case(name, n=8):
    if name == "tov":
        H = workloads.tov_hierarchy(n)
        (st, bx, by, bz, aux), _ = workloads.magnetised_tov(H)
        return H, params.tov(), (st, bx, by, bz, aux)
    H = workloads.torus_hierarchy(n)
    return H, params.torus(), workloads.fm_torus(H)


# 8^3 blocks in both modes; the TOV star also at the benchmark's 16^3 blocks
# in tuned mode (3.9 M cells, about two minutes of oracle time)
@pytest.mark.parametrize("name,mode,n", [("tov", abi.MODE_PLAIN, 8), ("tov", abi.MODE_TUNED, 8),
                                         ("torus", abi.MODE_PLAIN, 8), ("torus", abi.MODE_TUNED, 8),
                                         ("tov", abi.MODE_TUNED, 16)])
def test_fmr_config_rk3_step_matches_oracle(name, mode, n):
    H, P, (st, bx, by, bz, aux) = _case(name, n)
    H.fill_ghosts(st, bx, by, bz)
    R = H.reflux_lists()
    maps = H.gather_maps()
    idx = H.idx()
    dt = 0.25 / idx[:, 0].max()
    # oracle
    ost = [x.copy() for x in (st, bx, by, bz)]
    oaux = aux.copy()
    S = _oracle.Stage(P, H.n, H.n, H.n, H.ngz, H.nq)
    S.set_reflux(R)
    S.compute_aux(idx.copy(), ost, oaux)
    _oracle_rk3(S, H, idx.copy(), dt, ost, oaux)
    # GPU
    dev = torch.device("cuda:0")
    Pg = abi.Params.from_buffer_copy(P)
    if mode == abi.MODE_TUNED:
        Pg.ranges = abi.RANGES_NEXT_STAGE
    g = GRMHDEquationsSystem(Pg)
    g.reserve(Blocks(H.n, H.n, H.n, H.ngz, H.nq, idx, device=dev))
    g.set_mode(mode)
    g.set_reflux(R)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(T(st), T(bx), T(by), T(bz))
    aux_d = T(aux)
    bc = lambda f: g.fill_ghosts_gather(f, maps)
    g.compute_auxiliary_quantities(state, aux_d)
    sp, spp = state.clone(), state.clone()
    if mode == abi.MODE_TUNED:
        g.set_static_metric(state)
        g.set_tuning(1, 1, 1, 1)
    g.rk3_step(dt, state, sp, spp, aux_d, bc)
    torch.cuda.synchronize()
    gs = [x.cpu().numpy() for x in (state.state, state.bx, state.by, state.bz)]
    # Parity metric of these configurations: each variable's largest error
    # relative to its largest magnitude, and the state-normalised per-cell
    # error where rho > 1e-4 rho_max.  Their densities span 8 orders of
    # magnitude: an atmosphere cell's conserved variables change by the
    # fluxes of its dense neighbours, so its per-cell relative error carries
    # the neighbours' rounding amplified by the contrast (the oracle and the
    # reference's own numerics, two CPU builds of the same operations,
    # already differ there by up to 1e-7 per cell, and by under 3e-12
    # relative to each field's magnitude).
    A, B = interior(gs[0][:, :7], H.ngz), interior(ost[0][:, :7], H.ngz)
    for v in range(7):
        assert np.max(np.abs(A[:, v] - B[:, v])) <= STEP_TOL * np.max(np.abs(B[:, v])), v
    rho = interior(oaux[:, abi.RHO], H.ngz)
    dense = (rho > 1e-4 * rho.max())[:, None]
    e = cons_rel_err(np.where(dense, A, 1.0), np.where(dense, B, 1.0))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], ost[1:]):
        assert np.max(np.abs(a - b)) < STEP_TOL * np.max(np.abs(b))
    ga = aux_d.cpu().numpy()
    gi, oi = interior(ga, H.ngz), interior(oaux, H.ngz)
    d1 = dense[:, 0]
    for v in (abi.RHO, abi.PRESS):
        r = np.max(np.abs(gi[:, v][d1] - oi[:, v][d1]) / np.abs(oi[:, v][d1]))
        assert r < STEP_TOL, (v, r)
    np.testing.assert_array_equal(gi[:, abi.C2P_ERR], oi[:, abi.C2P_ERR])
    # div B stays at round-off in every block
    bmax = max(np.max(np.abs(x)) for x in gs[1:])
    dx = H.spacings()
    assert np.max(np.abs(gi[:, abi.BDIV]) * dx[:, 0, None, None, None]) < 1e-12 * bmax
    assert g.status().device_flags == 0


def test_gather_fill_matches_host_fill():
    """grb_fill_ghosts_gather on random data equals the host fill of the
    same maps bit for bit (both accumulate the 8 slots in order, each
    product and sum rounded on its own)."""
    H = workloads.tov_hierarchy(8)
    rng = np.random.default_rng(3)
    NN = H.n + 2 * H.ngz
    st = rng.standard_normal((H.nq, abi.N_EVOL_VARS, NN, NN, NN))
    bx = rng.standard_normal((H.nq, NN, NN, NN + 1))
    by = rng.standard_normal((H.nq, NN, NN + 1, NN))
    bz = rng.standard_normal((H.nq, NN + 1, NN, NN))
    dev = torch.device("cuda:0")
    g = GRMHDEquationsSystem(params.tov())
    g.reserve(Blocks(H.n, H.n, H.n, H.ngz, H.nq, H.idx(), device=dev))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    f = Fields(T(st), T(bx), T(by), T(bz))
    g.fill_ghosts_gather(f, H.gather_maps())
    torch.cuda.synchronize()
    H.fill_ghosts(st, bx, by, bz)
    for a, b in zip((f.state, f.bx, f.by, f.bz), (st, bx, by, bz)):
        assert np.array_equal(a.cpu().numpy(), b)


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_fmr_host_step_pipeline_matches_sequential(mode):
    """rk3_step_host on the TOV hierarchy (refluxing, gather fill): runs of
    blocks filled by their part of the gather maps, the substeps on the
    whole grid, two chained steps; the same bits as the sequential host
    round trip in the host arrays and every device array."""
    from grace_b200.host import gather_runs
    H, P, (st, bx, by, bz, aux) = _case("tov")
    H.fill_ghosts(st, bx, by, bz)
    R, maps, idx = H.reflux_lists(), H.gather_maps(), H.idx()
    dt = 0.25 / idx[:, 0].max()
    dev = torch.device("cuda:0")
    Pg = abi.Params.from_buffer_copy(P)
    if mode == abi.MODE_TUNED:
        Pg.ranges = abi.RANGES_NEXT_STAGE
    g = GRMHDEquationsSystem(Pg)
    blocks = Blocks(H.n, H.n, H.n, H.ngz, H.nq, idx, device=dev)
    g.reserve(blocks)
    g.set_mode(mode)
    g.set_reflux(R)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    st0 = Fields(T(st), T(bx), T(by), T(bz))
    aux0 = T(aux)
    g.compute_auxiliary_quantities(st0, aux0)
    if mode == abi.MODE_TUNED:
        g.set_static_metric(st0)
        g.set_tuning(1, 1, 1, 1)
    bc = lambda fl: g.fill_ghosts_gather(fl, maps)
    runs, run_maps, deps = gather_runs(maps, blocks, 5)
    fill_run = lambda fl, s, stream: g.fill_ghosts_gather(fl, run_maps[s], stream=stream)
    io = (torch.cuda.Stream(), torch.cuda.Stream())
    out = []
    for piped in (False, True):
        state, a = st0.clone(), aux0.clone()
        sp, spp = state.clone(), state.clone()
        host = g.packed_host_fields()
        g.copy_evolved_packed(host, state, to_device=False)
        prev = None
        for _ in range(2):
            if piped:
                prev = g.rk3_step_host(dt, host, state, sp, spp, a, bc, runs, fill_run, deps, streams=io, after=prev,
                                       wait=False, whole_grid_substeps=True)
            else:
                g.copy_evolved_packed(host, state, to_device=True)
                bc(state)
                g.compute_auxiliary_quantities(state, a)
                g.linop_apply(sp, state, None, 1.0, 0.0)
                g.rk3_step(dt, state, sp, spp, a, bc)
                g.copy_evolved_packed(host, state, to_device=False)
        torch.cuda.current_stream().wait_stream(io[1])
        torch.cuda.synchronize()
        out.append([x.clone() for x in (host.state, host.bx, host.by, host.bz, state.state, state.bx, state.by,
                                         state.bz, sp.state, a)])
    for k, (x, y) in enumerate(zip(*out)):
        assert torch.equal(x, y), k
    assert g.status().device_flags == 0
