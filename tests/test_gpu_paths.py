"""GPU parity of the paths the other stage tests do not reach, each against
the CPU oracle through the C ABI:

* the benchmarked configuration itself: 16^3 blocks with 4 ghosts, WENO-Z +
  HLLE + Gardiner-Stone + FOFC in tuned mode with the aux pass and linop on
  the next stage's cells, the static-metric cache, the TMA-staged flux
  tiles, the per-block aux cell list and the compacted FOFC face list;
* the LLF (Rusanov) Riemann solver of the stage, with and without the
  light-cone floor rusanov_use_c_limit (grmhd.hh:855-883), and under the
  UCT EMF;
* the compacted FOFC list's overflow path (more tagged faces than the list
  holds: the whole-box recompute);
* a three-piece piecewise-polytropic cold EOS through the c2p and the stage;
* the tuned mode's default drop-in ranges: every aux cell and every
  variable of the state written, as the reference's functions do.
"""
import functools

import numpy as np
import pytest
import torch

import _oracle
from grace_b200 import abi, params, workloads
from grace_b200.host import Blocks, Fields, GRMHDEquationsSystem
from parity import cons_rel_err, interior, prim_tol, state_residual, tuned_aux_mask

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10  # state-normalised relative error after one RK3 step
PIECES = (10.0, [1.8, 2.2, 2.0], [1e-5, 1e-4])  # kappa_0, gammas, piece densities


def _blast16(max_sigma=100.0):
    """The benchmark's blast wave at its cell geometry on a 3^3 brick of 16^3
    blocks around the overdense sphere (dx = 0.09375)."""
    P = params.blast()
    P.max_sigma = max_sigma  # the schema default: FOFC fires on the background
    su, f = workloads.blast(nb=(3, 3, 3), n=(16, 16, 16), lo=(-2.25,) * 3, hi=(2.25,) * 3)
    return P, su, f, 0.25 / su.idx()[0, 0]


def _gpu(P, su, f, dt, nsteps, mode, ranges=abi.RANGES_NEXT_STAGE, tuning=None, static_metric=False,
         fofc_cap=None):
    dev = torch.device("cuda:0")
    P = abi.Params.from_buffer_copy(P)
    P.ranges = ranges
    g = GRMHDEquationsSystem(P)
    g.reserve(Blocks(su.n[0], su.n[1], su.n[2], su.ngz, su.nq, su.idx(), device=dev))
    g.set_mode(mode)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    st, bx, by, bz, aux = f
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
    if fofc_cap is not None:
        g.set_fofc_list_capacity(fofc_cap)
    for _ in range(nsteps):
        g.rk3_step(dt, state, sp, spp, aux_d, bc)
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in (state.state, state.bx, state.by, state.bz)], aux_d.cpu().numpy(), g


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
    return state, aux, S.fofc_counts()


@functools.lru_cache(maxsize=None)
def _oracle_blast16():
    P, su, f, dt = _blast16()
    return _oracle_run(P, su, f, dt, 1)


def _check_state(gs, os_, ngz):
    e = cons_rel_err(interior(gs[0][:, :7], ngz), interior(os_[0][:, :7], ngz))
    assert e.max() < STEP_TOL, e
    for a, b in zip(gs[1:], os_[1:]):
        d = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert d < STEP_TOL


def _check_aux(ga, oa, sel):
    for v in (abi.RHO, abi.PRESS, abi.EPS, abi.TEMP):
        d = np.abs(ga[:, v][sel] - oa[:, v][sel])
        r = np.max(d / np.maximum(np.abs(oa[:, v][sel]), 1e-300))
        assert r < STEP_TOL, (v, r)
    np.testing.assert_array_equal(ga[:, abi.C2P_ERR][sel], oa[:, abi.C2P_ERR][sel])


# tuned candidates: the autotuner's pick; global-load flux at 4 CTAs/SM with
# the others at 4; 256-thread TMA flux tiles with the work-queue aux pass;
# the work-queue FOFC flag with the deferred-backup aux pass, and with the
# work-queue aux pass; the work-queue forms of the flux (TMA 128 and 256,
# global loads) and of the update
@pytest.mark.parametrize("tuning", [None, (0, 1, 1, 1), (2, 2, 2, 4), (1, 4, 1, 7), (1, 3, 1, 3), (4, 1, 4, 1),
                                    (5, 4, 3, 4), (3, 1, 5, 1)])
def test_benchmark_configuration_matches_oracle(tuning):
    """One SSP-RK3 step of the benchmark's exact code path (16^3 blocks,
    tuned, static-metric cache, next-stage ranges, FOFC list) against the
    oracle: state within the step tolerance, aux on the cells the tuned pass
    maintains with C2P_ERR bit for bit, and the same FOFC face and edge
    counts in the last substep."""
    P, su, f, dt = _blast16()
    gs, ga, g = _gpu(P, su, f, dt, 1, abi.MODE_TUNED, tuning=tuning, static_metric=True)
    os_, oa, counts = _oracle_blast16()
    _check_state(gs, os_, su.ngz)
    _check_aux(ga, oa, (slice(None), tuned_aux_mask(su)))
    st = g.status()
    assert st.fofc_faces > 1000
    assert (st.fofc_faces, st.fofc_edges) == counts
    assert st.device_flags == 0
    if tuning is None:
        # the autotuner picked one of the flux candidates
        assert g.tuning()["flux"]["min_ctas_per_sm"] in (4, 104, 102, 1004, 1104, 1102)
    else:
        t = g.tuning()
        assert t["flux"]["min_ctas_per_sm"] == [4, 104, 102, 1004, 1104, 1102][tuning[0]]
        assert t["update"]["min_ctas_per_sm"] == [1, 3, 4, 101, 103, 104][tuning[2]]
        assert t["fofc_flag"]["min_ctas_per_sm"] == [3, 4, 5, 103, 104, 105][tuning[1]]
        assert t["aux"]["min_ctas_per_sm"] == [3, 4, 5, 103, 104, 105, 203, 204, 205][tuning[3]]


@pytest.mark.parametrize("cap", [0, 7])
def test_fofc_list_overflow_matches_oracle(cap):
    """More tagged faces than the compacted list holds: the tuned stage
    recomputes them in its whole-box loop, with the oracle's results and
    counts."""
    P, su, f, dt = _blast16()
    gs, ga, g = _gpu(P, su, f, dt, 1, abi.MODE_TUNED, tuning=(1, 1, 1, 1), static_metric=True, fofc_cap=cap)
    os_, oa, counts = _oracle_blast16()
    _check_state(gs, os_, su.ngz)
    st = g.status()
    assert st.fofc_faces > cap
    assert (st.fofc_faces, st.fofc_edges) == counts


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
@pytest.mark.parametrize("c_limit", [0.0, 1e-3])
def test_llf_stage_matches_oracle(c_limit, mode):
    """The LLF solver (cmax = cmin = the largest |speed| of both sides) in
    every face of the stage, and with rusanov_use_c_limit = 1e-3 above the
    background density (1e-4) the light-cone floor alpha sqrt(g^dd) + |beta|
    on the background faces; blast wave on 8^3 blocks."""
    P = params.blast()
    P.riemann = abi.RIEMANN_LLF
    P.rusanov_use_c_limit = c_limit
    su, f = workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
    dt = 0.25 / su.idx()[0, 0]
    gs, ga, g = _gpu(P, su, f, dt, 1, mode, tuning=(1, 1, 1, 1))
    os_, oa, counts = _oracle_run(P, su, f, dt, 1)
    _check_state(gs, os_, su.ngz)
    sel = (slice(None), tuned_aux_mask(su)) if mode == abi.MODE_TUNED else (slice(None),)
    _check_aux(ga, oa, sel)
    assert (g.status().fofc_faces, g.status().fofc_edges) == counts
    assert g.status().device_flags == 0


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
@pytest.mark.parametrize("recon", [abi.RECON_WENOZ, abi.RECON_MC2])
def test_llf_with_uct_matches_oracle(recon, mode):
    """The LLF solver under the UCT EMF, whose edge EMFs take the Riemann
    speeds of the faces around each edge (evolve.cpp:1131-1340): Balsara-1
    on a 4x1x1 brick of 8^3 blocks, WENO-Z and MC2, one SSP-RK3 step
    against the oracle."""
    P = params.balsara1()
    P.riemann = abi.RIEMANN_LLF
    P.recon = recon
    su, f = workloads.balsara1(nb=(4, 1, 1), n=(8, 8, 8))
    dt = 0.4 / su.idx()[0, 0]
    gs, ga, g = _gpu(P, su, f, dt, 1, mode, tuning=(1, 1, 1, 1))
    os_, oa, counts = _oracle_run(P, su, f, dt, 1)
    _check_state(gs, os_, su.ngz)
    _check_aux(ga, oa, (slice(None),))
    assert g.status().device_flags == 0


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_pwpoly_three_pieces_c2p_matches_oracle(mode):
    """c2p with a three-piece cold polytrope (non-integer indices: pow) on
    states whose densities span all three pieces."""
    P = params.hybrid_pwpoly(PIECES[0], PIECES[1], PIECES[2], gamma_th=1.8, c2p_tol=1e-12, max_w=60.0,
                             max_sigma=2.0e3)
    rng = np.random.default_rng(21)
    n = 20000
    cons, prims = workloads.c2p_states(n, seed=21)
    # rescale the rest-mass densities into [1e-7, 1e-3] (log-uniform)
    # keeping each state's velocity, specific energy and magnetisation
    s = 10 ** rng.uniform(-7, -3, n) / prims[abi.P_RHO]
    cons[:7] *= s[None]
    cons[7:10] *= np.sqrt(s)[None]
    dev = torch.device("cuda:0")
    g = GRMHDEquationsSystem(P)
    g.set_mode(mode)
    c_d = torch.from_numpy(np.ascontiguousarray(cons)).to(dev)
    err_d = torch.zeros(n, dtype=torch.int32, device=dev)
    pr_g = g.conservs_to_prims(c_d, err=err_d).cpu().numpy()
    err_g = err_d.cpu().numpy().view(np.uint32)
    pr_o, _, err_o, _, _, _ = _oracle.c2p_batch(P, cons)
    rho = pr_o[abi.P_RHO]
    for lo, hi in ((0, 1e-5), (1e-5, 1e-4), (1e-4, 1)):
        assert np.sum((rho > lo) & (rho <= hi)) > 1000  # every piece is visited
    same = err_g == err_o
    assert same.mean() > 0.999
    res = state_residual(pr_g[:, same], pr_o[:, same])
    assert np.all(res < prim_tol(pr_o)[same]), res.max()


@pytest.mark.parametrize("mode", [abi.MODE_PLAIN, abi.MODE_TUNED])
def test_pwpoly_three_pieces_stage_matches_oracle(mode):
    """One RK3 step of the curved-metric blob (Kerr-Schild) with the
    three-piece cold EOS: the blob's densities (1e-7 to 1e-3) cross both
    piece boundaries."""
    from curved import curved_setup
    P, su, f = curved_setup(emf=abi.EMF_GS, fofc=1, pieces=PIECES)
    rho = f[4][:, abi.RHO]
    assert rho.min() < 1e-5 and rho.max() > 1e-4
    dt = 0.25 / su.idx()[0, 0]
    gs, ga, g = _gpu(P, su, f, dt, 1, mode, tuning=(1, 1, 1, 1))
    os_, oa, counts = _oracle_run(P, su, f, dt, 1)
    _check_state(gs, os_, su.ngz)
    sel = (slice(None), tuned_aux_mask(su)) if mode == abi.MODE_TUNED else (slice(None),)
    _check_aux(ga, oa, sel)
    assert g.status().device_flags == 0


@pytest.mark.parametrize("name", ["blast", "balsara"])
def test_tuned_default_ranges_fill_every_cell(name):
    """The drop-in contract in tuned mode: with the default GRB_RANGES_FULL
    the aux pass writes every cell of every block, ghosts included, and
    linop_apply combines all 23 variables, as compute_auxiliary_quantities
    and linop_apply do.  One RK3 step against the oracle on all 24^3 cells
    of aux (C2P_ERR bit for bit) and on every variable of every cell of the
    state."""
    if name == "blast":
        P = params.blast()
        su, f = workloads.blast(nb=(2, 2, 2), n=(8, 8, 8))
        dt = 0.25 / su.idx()[0, 0]
    else:
        P = params.balsara1()
        su, f = workloads.balsara1(nb=(4, 1, 1), n=(8, 8, 8))
        dt = 0.4 / su.idx()[0, 0]
    gs, ga, g = _gpu(P, su, f, dt, 1, abi.MODE_TUNED, ranges=abi.RANGES_FULL, tuning=(1, 1, 1, 1))
    os_, oa, _ = _oracle_run(P, su, f, dt, 1)
    _check_aux(ga, oa, (slice(None),))
    e = cons_rel_err(gs[0][:, :7], os_[0][:, :7])
    assert e.max() < STEP_TOL, e
    m, mo = gs[0][:, 7:], os_[0][:, 7:]
    assert np.max(np.abs(m - mo)) <= 1e-15 * np.max(np.abs(mo))


@pytest.mark.parametrize("aux", [6, 7, 8])
def test_deferred_backup_aux_pass_matches_oracle(aux):
    """The aux pass with the entropy backups deferred to a second kernel
    (tuned aux candidates 6..8) on the curved-metric blob with
    beta_fallback raised to 1e3, so that nearly every cell distrusts its
    Kastaun result and takes the backup: one RK3 step against the oracle,
    C2P_ERR bit for bit (ERR_ENT_BACKUP on most cells)."""
    from curved import curved_setup
    P, su, f = curved_setup(emf=abi.EMF_GS, fofc=1)
    P.beta_fallback = 1e3
    dt = 0.25 / su.idx()[0, 0]
    gs, ga, g = _gpu(P, su, f, dt, 1, abi.MODE_TUNED, tuning=(1, 1, 1, aux))
    assert g.tuning()["aux"]["min_ctas_per_sm"] == [203, 204, 205][aux - 6]
    os_, oa, counts = _oracle_run(P, su, f, dt, 1)
    _check_state(gs, os_, su.ngz)
    sel = (slice(None), tuned_aux_mask(su))
    _check_aux(ga, oa, sel)
    backup = (ga[:, abi.C2P_ERR][sel].astype(np.uint64) >> 19) & 1
    assert backup.mean() > 0.5
    assert g.status().device_flags == 0
