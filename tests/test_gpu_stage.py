"""GPU GRMHD stage (through the C ABI) against the CPU oracle on small grids."""
import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem
from parity import cons_rel_err, interior, tuned_aux_mask

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10   # state-normalised relative error after one RK3 step


def _setup(name):
    if name == "blast":
        P = params.blast()
        su, f = workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
        cfl = 0.25
    else:
        P = params.balsara1()
        su, f = workloads.balsara1(nb=(4, 1, 1), n=(8, 8, 8))
        cfl = 0.4
    return P, su, f, cfl / su.idx()[0, 0]


def _gpu_run(P, su, f, dt, nsteps, mode=abi.MODE_PLAIN, tuning=None, static_metric=False,
             ranges=abi.RANGES_NEXT_STAGE):
    """nsteps SSP-RK3 steps on the GPU.  Tuned runs use the aux and linop
    ranges of the benchmark (the next stage's cells only) unless `ranges`
    says otherwise."""
    dev = torch.device("cuda:0")
    st, bx, by, bz, aux = f
    blocks = Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev)
    P = abi.Params.from_buffer_copy(P)
    P.ranges = ranges
    g = GRMHDEquationsSystem(P)
    g.reserve(blocks)
    g.set_mode(mode)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(T(st), T(bx), T(by), T(bz))
    aux_d = T(aux)
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)
    bc(state)
    g.compute_auxiliary_quantities(state, aux_d)
    sp, spp = state.clone(), state.clone()
    if static_metric:
        g.set_static_metric(state)
    if mode == abi.MODE_TUNED:
        if tuning is None:
            g.autotune(sp, state, aux_d)
        else:
            g.set_tuning(*tuning)
    for _ in range(nsteps):
        g.rk3_step(dt, state, sp, spp, aux_d, bc)
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in (state.state, state.bx, state.by, state.bz)], aux_d.cpu().numpy(), g


def _aux_sel(P, su, mode, ranges=abi.RANGES_NEXT_STAGE):
    """Index of the aux cells maintained by this mode (all cells, or the
    tuned pass's list with the GS EMF and the next stage's ranges), for
    arrays (nq, NZ, NY, NX)."""
    if mode == abi.MODE_TUNED and P.emf == abi.EMF_GS and ranges == abi.RANGES_NEXT_STAGE:
        return (slice(None), tuned_aux_mask(su))
    return (slice(None),)


def _oracle_run(P, su, f, dt, nsteps):
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq)
    state = [st, bx, by, bz]
    _oracle.fill_ghosts("orc", su, state)
    S.compute_aux(su.idx().copy(), state, aux)
    sp = [x.copy() for x in state]
    spp = [x.copy() for x in state]
    for _ in range(nsteps):
        _oracle.rk3_step(S, su, dt, state, sp, spp, aux)
    return state, aux, S


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
@pytest.mark.parametrize("name", ["blast", "balsara"])
def test_one_rk3_step_matches_oracle(name, mode):
    P, su, f, dt = _setup(name)
    gs, ga, g = _gpu_run(P, su, f, dt, 1, mode)
    os_, oa, S = _oracle_run(P, su, f, dt, 1)
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(os_[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], os_[1:]):
        d = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert d < STEP_TOL
    # aux primitives of the new state (the cells this mode maintains)
    sel = _aux_sel(P, su, mode)
    for v in (abi.RHO, abi.PRESS, abi.EPS):
        r = np.max(np.abs(ga[:, v][sel] - oa[:, v][sel]) / np.abs(oa[:, v][sel]))
        assert r < STEP_TOL, (v, r)
    np.testing.assert_array_equal(ga[:, abi.C2P_ERR][sel], oa[:, abi.C2P_ERR][sel])


@pytest.mark.parametrize("flux", [0, 1, 2])
@pytest.mark.parametrize("name", ["blast", "balsara"])
def test_tuned_flux_candidates_match_oracle(name, flux):
    """Each tuned flux candidate (global loads; TMA-staged shared-memory
    tiles of 128 threads at 4 CTAs/SM and of 256 threads at 2) gives one RK3
    step within the step tolerance
    of the oracle, GS (blast) and UCT (Balsara-1) transverse ranges."""
    P, su, f, dt = _setup(name)
    gs, ga, g = _gpu_run(P, su, f, dt, 1, abi.MODE_TUNED, tuning=(flux, 0, 0, 0))
    assert g.tuning()["flux"]["min_ctas_per_sm"] == [4, 104, 102][flux]
    os_, oa, S = _oracle_run(P, su, f, dt, 1)
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(os_[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], os_[1:]):
        d = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert d < STEP_TOL
    assert g.status().device_flags == 0


@pytest.mark.parametrize("flux", [0, 1])
@pytest.mark.parametrize("recon", [abi.RECON_MC2, abi.RECON_MINMOD, abi.RECON_DONOR])
def test_tuned_flux_reconstructions_match_oracle(recon, flux):
    """The per-cell reconstruction of the TMA-staged flux kernel (both face
    values of a cell at once) and the per-face one of the global-load
    kernel, for the limiter and donor schemes, within the step tolerance of
    the oracle on the blast wave."""
    P, su, f, dt = _setup("blast")
    P.recon = recon
    gs, ga, g = _gpu_run(P, su, f, dt, 1, abi.MODE_TUNED, tuning=(flux, 0, 0, 0))
    os_, oa, S = _oracle_run(P, su, f, dt, 1)
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(os_[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], os_[1:]):
        d = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert d < STEP_TOL
    assert g.status().device_flags == 0


@pytest.mark.parametrize("aux", [3, 4, 5])
@pytest.mark.parametrize("name", ["blast", "balsara"])
def test_aux_work_queue_matches_oracle(name, aux):
    """The work-queue form of the aux pass (one wave of CTAs pulling 128-cell
    tiles from a device counter) at each register cap: one RK3 step within
    the step tolerance of the oracle, and its fused dt reduction equal to the
    separate pass to rounding."""
    P, su, f, dt = _setup(name)
    gs, ga, g = _gpu_run(P, su, f, dt, 1, abi.MODE_TUNED, tuning=(1, 0, 0, aux))
    assert g.tuning()["aux"]["min_ctas_per_sm"] == [103, 104, 105][aux - 3]
    os_, oa, S = _oracle_run(P, su, f, dt, 1)
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(os_[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e
    sel = _aux_sel(P, su, abi.MODE_TUNED)
    for v in (abi.RHO, abi.PRESS, abi.EPS):
        r = np.max(np.abs(ga[:, v][sel] - oa[:, v][sel]) / np.abs(oa[:, v][sel]))
        assert r < STEP_TOL, (v, r)
    np.testing.assert_array_equal(ga[:, abi.C2P_ERR][sel], oa[:, abi.C2P_ERR][sel])
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    state = Fields(*[T(x) for x in gs])
    aux_d = T(ga)
    dx = T(1.0 / su.idx())
    d1 = torch.zeros(1, dtype=torch.float64, device=dev)
    d2 = torch.zeros(1, dtype=torch.float64, device=dev)
    g.compute_auxiliary_quantities_dt(state, aux_d, dx, 0.4, d1)
    g.find_stable_timestep(state, aux_d, dx, 0.4, d2)
    torch.cuda.synchronize()
    assert abs(d1.item() - d2.item()) <= 1e-14 * d2.item()
    assert g.status().device_flags == 0


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_div_b_and_conservation_blast(mode):
    P, su, f, dt = _setup("blast")
    gs, ga, g = _gpu_run(P, su, f, dt, 3, mode)
    bd = interior(ga[:, abi.BDIV], su.ngz)
    assert np.max(np.abs(bd)) < 1e-13


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_fofc_flags_match_oracle(mode):
    P, su, f, dt = _setup("blast")
    # With the schema-default magnetisation ceiling (max_sigma = 100) the
    # blast background sits on the clamp, the dry-run c2p reports "floored"
    # and FOFC recomputes several hundred faces per stage.
    P.max_sigma = 100.0
    gs, ga, g = _gpu_run(P, su, f, dt, 1, mode)
    os_, oa, S = _oracle_run(P, su, f, dt, 1)
    st = g.status()
    assert st.fofc_faces > 0
    assert (st.fofc_faces, st.fofc_edges) == S.fofc_counts()
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(os_[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e


@pytest.mark.parametrize("name", ["blast", "balsara"])
def test_one_rk3_step_matches_reference_fixture(name):
    """GPU against the reference's own per-cell numerics (tests/golden)."""
    import os
    P, su, f, dt = _setup(name)
    gs, ga, g = _gpu_run(P, su, f, dt, 1)
    ref = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "stage_ref.npz"))
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), ref[f"{name}_cons"])
    assert e.max() < STEP_TOL, e


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_graph_replay_matches_eager(mode):
    """Three SSP-RK3 steps, the last two replayed from one captured CUDA
    graph, are bit-identical to three eagerly launched steps, FOFC included.
    Both runs start from the same initial data on the same handle, so the
    library's scratch (the GS cell-centred E of the last aux pass) is
    reproduced too."""
    P, su, f, dt = _setup("blast")
    P.max_sigma = 100.0  # the schema default: the magnetisation clamp fires and FOFC is exercised
    dev = torch.device("cuda:0")
    blocks = Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev)
    g = GRMHDEquationsSystem(P)
    g.reserve(blocks)
    g.set_mode(mode)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    st, bx, by, bz, aux = f
    init = Fields(T(st), T(bx), T(by), T(bz))
    init_aux = T(aux)
    state, aux_d = init.clone(), init_aux.clone()
    sp, spp = init.clone(), init.clone()
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)

    def start():
        state.copy_(init)
        aux_d.copy_(init_aux)
        bc(state)
        g.compute_auxiliary_quantities(state, aux_d)
        sp.copy_(state)
        spp.copy_(state)

    start()
    if mode == abi.MODE_TUNED:
        g.autotune(sp, state, aux_d)
    start()
    for _ in range(3):
        g.rk3_step(dt, state, sp, spp, aux_d, bc)
    torch.cuda.synchronize()
    eager = [x.cpu().numpy() for x in (state.state, state.bx, state.by, state.bz, aux_d)]
    start()
    g.rk3_step(dt, state, sp, spp, aux_d, bc)   # first-call set-up outside the capture
    graph, per_step = g.capture_rk3_step(dt, state, sp, spp, aux_d, bc)
    assert per_step > 20
    graph.replay()
    graph.replay()
    torch.cuda.synchronize()
    replayed = [x.cpu().numpy() for x in (state.state, state.bx, state.by, state.bz, aux_d)]
    for x, y in zip(eager, replayed):
        assert np.array_equal(x, y, equal_nan=True)
    assert g.status().device_flags == 0


@pytest.mark.parametrize("name", ["blast", "balsara"])
@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_timestep_reduction(name, mode):
    """find_stable_timestep on the GPU, fused into the aux pass and as a
    separate pass, against the oracle's find_stable_timestep_impl on the
    same arrays; the fused aux pass gives the plain pass's aux and state.
    The two aux kernels are separate compiled instantiations (and, tuned,
    under different register caps), so they agree to rounding, not bit for
    bit."""
    P, su, f, dt = _setup(name)
    (st, bx, by, bz), aux, g = _gpu_run(P, su, f, dt, 1, mode)
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dx = np.ascontiguousarray(1.0 / su.idx())
    cfl = 0.4
    state = Fields(T(st), T(bx), T(by), T(bz))
    aux_a, aux_b = T(aux), T(aux)
    state_b = state.clone()
    dt_f = torch.zeros(1, dtype=torch.float64, device=dev)
    dt_s = torch.zeros(1, dtype=torch.float64, device=dev)
    g.compute_auxiliary_quantities(state, aux_a)
    g.compute_auxiliary_quantities_dt(state_b, aux_b, T(dx), cfl, dt_f)
    g.find_stable_timestep(state_b, aux_b, T(dx), cfl, dt_s)
    torch.cuda.synchronize()
    a, b = aux_a.cpu().numpy(), aux_b.cpu().numpy()
    da = np.abs(a - b) / np.maximum(np.abs(a), 1e-300)
    assert np.max(da[np.isfinite(da)]) < 1e-12, np.max(da)
    sa, sb = state.state.cpu().numpy(), state_b.state.cpu().numpy()
    assert np.max(np.abs(sa - sb) / np.maximum(np.abs(sa), 1e-300)) < 1e-12
    assert abs(dt_f.item() - dt_s.item()) <= 1e-14 * dt_s.item()
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq)
    host = [state_b.state.cpu().numpy(), None, None, None]
    dt_o = S.find_stable_timestep(host, aux_b.cpu().numpy(), dx, cfl)
    assert abs(dt_f.item() - dt_o) <= 1e-13 * dt_o, (dt_f.item(), dt_o)
    assert 0.0 < dt_o < 1.0


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
@pytest.mark.parametrize("emf", [abi.EMF_GS, abi.EMF_UCT])
def test_curved_metric_step_matches_oracle(emf, mode):
    """One SSP-RK3 step on Schwarzschild in Kerr-Schild coordinates
    (tests/curved.py): metric derivatives, extrinsic curvature and the
    curved geometric sources through the whole stage, hybrid EOS; div B
    stays at round-off."""
    from curved import curved_setup
    P, su, f = curved_setup(emf=emf, fofc=1 if emf == abi.EMF_GS else 0)
    dt = 0.25 / su.idx()[0, 0]
    gs, ga, g = _gpu_run(P, su, f, dt, 1, mode)
    os_, oa, S = _oracle_run(P, su, f, dt, 1)
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(os_[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], os_[1:]):
        d = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert d < STEP_TOL
    bmax = max(np.max(np.abs(x)) for x in gs[1:])
    assert np.max(np.abs(interior(ga[:, abi.BDIV], su.ngz))) * su.dx[0] < 1e-13 * bmax
    assert g.status().device_flags == 0


@pytest.mark.parametrize("tuning", [None, (0, 0, 0, 0), (1, 0, 0, 0)])
def test_curved_excision_donor_faces_match_oracle(tuning):
    """Excision by lapse on the curved setup: with alp_ex = 0.8 the cells
    with x below ~3.56 are excised by the c2p and every face next to one is
    a donor face (first-order states, grmhd.hh getflux); plain mode and both
    tuned flux kernels against the oracle."""
    from curved import curved_setup
    P, su, f = curved_setup(emf=abi.EMF_GS, fofc=1)
    P.alp_ex = 0.8
    alp = f[0][:, abi.ALP]
    assert alp.min() < 0.8 < alp.max()
    dt = 0.25 / su.idx()[0, 0]
    mode = abi.MODE_PLAIN if tuning is None else abi.MODE_TUNED
    gs, ga, g = _gpu_run(P, su, f, dt, 1, mode, tuning=tuning)
    os_, oa, S = _oracle_run(P, su, f, dt, 1)
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(os_[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], os_[1:]):
        d = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert d < STEP_TOL
    assert g.status().device_flags == 0


@pytest.mark.parametrize("update", [0, 1, 2])
@pytest.mark.parametrize("case", ["blast", "curved"])
def test_static_metric_cache_gives_identical_steps(case, update):
    """The tuned update reading the static-metric cache (grb_set_static_metric)
    gives the steps of the tuned update that differentiates the metric
    itself, at each register cap: the derivatives are the same bits (the
    stencil is evaluated without contraction), the rest of the update the
    same arithmetic in another kernel instantiation, so the two agree to a
    few ulp (1e-12 state-normalised after two RK3 steps); on the curved setup
    the cached steps also match the oracle."""
    if case == "blast":
        P, su, f, dt = _setup("blast")
    else:
        from curved import curved_setup
        P, su, f = curved_setup(emf=abi.EMF_GS, fofc=1)
        dt = 0.25 / su.idx()[0, 0]
    gs0, ga0, _ = _gpu_run(P, su, f, dt, 2, abi.MODE_TUNED, tuning=(1, 0, update, 0))
    gs1, ga1, g = _gpu_run(P, su, f, dt, 2, abi.MODE_TUNED, tuning=(1, 0, update, 0), static_metric=True)
    e = cons_rel_err(interior(gs1[0][:, :7], su.ngz), interior(gs0[0][:, :7], su.ngz))
    assert e.max() < 1e-12, e.max()
    for a, b in zip(gs1[1:], gs0[1:]):
        assert np.max(np.abs(a - b)) <= 1e-12 * max(np.max(np.abs(b)), 1e-300)
    np.testing.assert_array_equal(ga1[:, abi.C2P_ERR], ga0[:, abi.C2P_ERR])
    assert g.status().device_flags == 0
    if case == "curved":
        os_, oa, S = _oracle_run(P, su, f, dt, 2)
        e = cons_rel_err(interior(gs1[0][:, :7], su.ngz), interior(os_[0][:, :7], su.ngz))
        assert e.max() < STEP_TOL, e
    g.set_static_metric(None)


def _two_level_blast():
    """Two levels of the blast wave in one block array: the [-6, 6]^3 brick
    (dx 0.75) and a finer [-3, 3]^3 brick (dx 0.375), 8 blocks of 8^3 each,
    as an FMR hierarchy hands its blocks of every level to one launch.
    Returns the concatenated arrays, per-block idx and the two setups."""
    lv = [workloads.blast(nb=(2, 2, 2), n=(8, 8, 8)),
          workloads.blast(nb=(2, 2, 2), n=(8, 8, 8), lo=(-3, -3, -3), hi=(3, 3, 3))]
    sus = [x[0] for x in lv]
    f = [np.ascontiguousarray(np.concatenate([x[1][a] for x in lv])) for a in range(5)]
    idx = np.concatenate([s.idx() for s in sus])
    return sus, f, idx


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_two_level_blocks_in_one_launch_match_oracle(mode):
    """Blocks of two refinement levels (different spacings) advanced by the
    same launches: every kernel takes its spacing per block.  Ghosts are
    filled per level; one RK3 step at the fine level's CFL against the
    oracle, and the stable dt reduced over both levels with dx(0, q)."""
    P = params.blast()
    sus, f, idx = _two_level_blast()
    nq = sum(s.nq for s in sus)
    dt = 0.25 / idx[:, 0].max()
    ngz, n = sus[0].ngz, sus[0].n
    cut = [0, sus[0].nq, nq]
    # GPU: one system for the stage, one per level for its ghost fill
    dev = torch.device("cuda:0")
    g = GRMHDEquationsSystem(P)
    g.reserve(Blocks(n[0], n[1], n[2], ngz, nq, idx, device=dev))
    g.set_mode(mode)
    lvl = []
    for s in sus:
        gl = GRMHDEquationsSystem(P)
        gl.reserve(Blocks(n[0], n[1], n[2], ngz, s.nq, s.idx(), device=dev))
        lvl.append(gl)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    def bc(fl):
        for t, (s, gl) in enumerate(zip(sus, lvl)):
            a, b = cut[t], cut[t + 1]
            gl.fill_ghosts_brick(Fields(fl.state[a:b], fl.bx[a:b], fl.by[a:b], fl.bz[a:b]), s.nb, s.periodic)

    state = Fields(T(f[0]), T(f[1]), T(f[2]), T(f[3]))
    aux = T(f[4])
    bc(state)
    g.compute_auxiliary_quantities(state, aux)
    sp, spp = state.clone(), state.clone()
    if mode == abi.MODE_TUNED:
        g.set_static_metric(state)
        g.autotune(sp, state, aux)
    g.rk3_step(dt, state, sp, spp, aux, bc)
    dx = torch.from_numpy(np.ascontiguousarray(1.0 / idx)).to(dev)  # dx(d, q) at [3 q + d]
    dtd = torch.zeros(1, dtype=torch.float64, device=dev)
    g.find_stable_timestep(state, aux, dx, 0.25, dtd)
    torch.cuda.synchronize()
    gs = [x.cpu().numpy() for x in (state.state, state.bx, state.by, state.bz)]
    # oracle: the same hierarchy on the CPU
    st_, bx_, by_, bz_, ax_ = [x.copy() for x in f]
    S = _oracle.Stage(P, n[0], n[1], n[2], ngz, nq)
    ost = [st_, bx_, by_, bz_]

    def obc(fl):
        for t, s in enumerate(sus):
            a, b = cut[t], cut[t + 1]
            _oracle.fill_ghosts("orc", s, [x[a:b] for x in fl])

    obc(ost)
    S.compute_aux(idx.copy(), ost, ax_)
    osp = [x.copy() for x in ost]
    ospp = [x.copy() for x in ost]
    i2 = idx.copy()
    S.reset_diag(ax_)
    S.advance_substep(i2, dt, 1.0, osp, ost, ax_)
    obc(osp)
    S.compute_aux(i2, osp, ax_)
    S.linop(ospp, ost, osp, 0.75, 0.25)
    S.advance_substep(i2, dt, 0.25, ospp, osp, ax_)
    obc(ospp)
    S.compute_aux(i2, ospp, ax_)
    S.linop(ost, ost, ospp, 1.0 / 3, 2.0 / 3.0)
    S.advance_substep(i2, dt, 2.0 / 3.0, ost, ospp, ax_)
    obc(ost)
    S.compute_aux(i2, ost, ax_)
    e = cons_rel_err(interior(gs[0][:, :7], ngz), interior(ost[0][:, :7], ngz))
    assert e.max() < STEP_TOL, e.max()
    for a, b in zip(gs[1:], ost[1:]):
        assert np.max(np.abs(a - b)) < STEP_TOL * max(np.max(np.abs(b)), 1e-300)
    dto = S.find_stable_timestep(ost, ax_, np.ascontiguousarray(1.0 / idx), 0.25)
    assert abs(dtd.item() - dto) <= 1e-12 * dto, (dtd.item(), dto)
    assert g.status().device_flags == 0


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_curved_radius_excision_matches_oracle(mode):
    """Excision by radius (excision_criterion: radius) on the curved setup:
    the c2p excises the cells whose centre, from the block coordinates
    (grb_grid.coords: the centre of cell (0, 0, 0) of each block), lies
    within r_ex = 3.6 of the origin (the brick spans r = 3 .. 5.2); one
    SSP-RK3 step against the oracle given the same coordinates."""
    from curved import curved_setup
    P, su, f = curved_setup(emf=abi.EMF_GS, fofc=1)
    P.excise_by_radius = 1
    P.r_ex = 3.6
    crd = su.coords()
    X = su.cell_centres()
    r = np.sqrt(np.sum(X ** 2, axis=1))
    assert r.min() < P.r_ex < r.max()
    dt = 0.25 / su.idx()[0, 0]
    idx = su.idx()
    # oracle, coordinates passed to every substep and aux pass
    st, bx, by, bz, aux = [x.copy() for x in f]
    S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq)
    state = [st, bx, by, bz]
    bc_o = lambda fl: _oracle.fill_ghosts("orc", su, fl)
    bc_o(state)
    S.compute_aux(idx.copy(), state, aux, crd)
    sp = [x.copy() for x in state]
    spp = [x.copy() for x in state]
    S.reset_diag(aux)
    S.advance_substep(idx.copy(), dt, 1.0, sp, state, aux, crd)
    bc_o(sp)
    S.compute_aux(idx.copy(), sp, aux, crd)
    S.linop(spp, state, sp, 0.75, 0.25)
    S.advance_substep(idx.copy(), dt, 0.25, spp, sp, aux, crd)
    bc_o(spp)
    S.compute_aux(idx.copy(), spp, aux, crd)
    S.linop(state, state, spp, 1.0 / 3, 2.0 / 3.0)
    S.advance_substep(idx.copy(), dt, 2.0 / 3.0, state, spp, aux, crd)
    bc_o(state)
    S.compute_aux(idx.copy(), state, aux, crd)
    # GPU, the same coordinates in the grid
    dev = torch.device("cuda:0")
    blocks = Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, idx, coords=crd, device=dev)
    g = GRMHDEquationsSystem(P)
    g.reserve(blocks)
    g.set_mode(mode)
    if mode == abi.MODE_TUNED:
        g.set_tuning(1, 1, 1, 1)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    gst = Fields(*[T(x) for x in f[:4]])
    gaux = T(f[4])
    bc = lambda fl: g.fill_ghosts_brick(fl, su.nb, su.periodic)
    bc(gst)
    g.compute_auxiliary_quantities(gst, gaux)
    gsp, gspp = gst.clone(), gst.clone()
    g.rk3_step(dt, gst, gsp, gspp, gaux, bc)
    torch.cuda.synchronize()
    gs = [x.cpu().numpy() for x in (gst.state, gst.bx, gst.by, gst.bz)]
    ga = gaux.cpu().numpy()
    e = cons_rel_err(interior(gs[0][:, :7], su.ngz), interior(state[0][:, :7], su.ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], state[1:]):
        assert np.max(np.abs(a - b)) < STEP_TOL * np.max(np.abs(b))
    # the excised cells carry the excision flag in both, the same cells
    sel = (slice(None),) + tuple(slice(su.ngz, -su.ngz) for _ in range(3))
    np.testing.assert_array_equal(ga[:, abi.C2P_ERR][sel], aux[:, abi.C2P_ERR][sel])
    assert g.status().device_flags == 0
