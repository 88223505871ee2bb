"""Initial data and hierarchies of the FMR configurations (CPU): the TOV
star model (K=100, Gamma=2, rho_c=1.28e-3: 1.40 solar masses, areal radius
9.59, the standard model of this polytrope) and the Fishbone-Moncrief torus
in Kerr-Schild (a=0.9375, r_in=6, r_pmax=12); their face fields discretely
divergence free in every block; the conserved variables they write invert,
through the oracle's c2p, to the primitives they write; the hierarchies
2:1 balanced with uneven per-level block counts."""
import numpy as np
import pytest

import _oracle
from grace_b200 import abi, params, workloads


def _div_b(H, bx, by, bz):
    g, n = H.ngz, H.n
    dx = H.spacings()
    d = ((bx[:, g:-g, g:-g, g + 1:g + n + 1] - bx[:, g:-g, g:-g, g:g + n]) / dx[:, 0, None, None, None] +
         (by[:, g:-g, g + 1:g + n + 1, g:-g] - by[:, g:-g, g:g + n, g:-g]) / dx[:, 1, None, None, None] +
         (bz[:, g + 1:g + n + 1, g:-g, g:-g] - bz[:, g:g + n, g:-g, g:-g]) / dx[:, 2, None, None, None])
    return float(np.max(np.abs(d * dx[:, 0, None, None, None])))


def _c2p_roundtrip(P, st, bx, by, bz, aux, H, sample=20000, seed=1):
    """c2p of the written conserved variables against the written prims on
    a sample of interior cells (flat or curved metric from the state)."""
    g, n = H.ngz, H.n
    rng = np.random.default_rng(seed)
    q = rng.integers(0, H.nq, sample)
    k, j, i = (rng.integers(g, g + n, sample) for _ in range(3))
    cons = np.zeros((10, sample))
    for v in range(7):
        cons[v] = st[q, v, k, j, i]
    cons[7] = 0.5 * (bx[q, k, j, i] + bx[q, k, j, i + 1])
    cons[8] = 0.5 * (by[q, k, j, i] + by[q, k, j + 1, i])
    cons[9] = 0.5 * (bz[q, k, j, i] + bz[q, k + 1, j, i])
    met = np.zeros((10, sample))
    for a in range(6):
        met[a] = st[q, abi.GXX + a, k, j, i]
    for a in range(3):
        met[6 + a] = st[q, abi.BETAX + a, k, j, i]
    met[9] = st[q, abi.ALP, k, j, i]
    pr, _, err, _, _, _ = _oracle.c2p_batch(P, cons, np.ascontiguousarray(met))
    rho = aux[q, abi.RHO, k, j, i]
    return np.abs(pr[abi.P_RHO] - rho) / rho, err


def test_tov_model_and_data():
    sol = workloads.tov_solution()
    assert abs(sol["M"] - 1.400) < 2e-3 and abs(sol["R"] - 9.586) < 5e-3
    H = workloads.tov_hierarchy(8)
    assert list(H.level_counts()) == [32, 224, 224, 224, 256]
    (st, bx, by, bz, aux), _ = workloads.magnetised_tov(H)
    assert np.all(np.isfinite(st)) and np.all(np.isfinite(aux))
    bmax = max(np.max(np.abs(x)) for x in (bx, by, bz))
    assert _div_b(H, bx, by, bz) < 1e-13 * bmax
    rel, err = _c2p_roundtrip(params.tov(), st, bx, by, bz, aux, H)
    inside = aux[:, abi.RHO].max() > 1e-4
    assert inside and np.median(rel) < 1e-12 and np.percentile(rel, 99) < 1e-8


def test_torus_model_and_data():
    H = workloads.torus_hierarchy(8)
    counts = list(H.level_counts())
    assert len(counts) == 4 and len(set(counts)) == 4  # uneven per-level counts
    st, bx, by, bz, aux = workloads.fm_torus(H)
    assert np.all(np.isfinite(st)) and np.all(np.isfinite(aux))
    assert 0.95 < aux[:, abi.RHO].max() <= 1.0 and aux[:, abi.RHO].min() >= 1e-8 * (1 - 1e-3)
    bmax = max(np.max(np.abs(x)) for x in (bx, by, bz))
    assert bmax > 0 and _div_b(H, bx, by, bz) < 1e-12 * bmax
    rel, err = _c2p_roundtrip(params.torus(), st, bx, by, bz, aux, H)
    assert np.median(rel) < 1e-12 and np.percentile(rel, 99) < 1e-8


@pytest.mark.parametrize("which", ["tov", "torus"])
def test_gather_maps_copy_same_level_ghosts_exactly(which):
    """The composite fill leaves every interior cell alone and fills each
    ghost cell whose place a same-level leaf covers with that leaf's value."""
    H = workloads.tov_hierarchy(8) if which == "tov" else workloads.torus_hierarchy(8)
    rng = np.random.default_rng(5)
    NN = H.n + 2 * H.ngz
    st = rng.standard_normal((H.nq, abi.N_EVOL_VARS, NN, NN, NN))
    z = np.zeros((H.nq, NN, NN, NN + 1)), np.zeros((H.nq, NN, NN + 1, NN)), np.zeros((H.nq, NN + 1, NN, NN))
    before = st.copy()
    H.fill_ghosts(st, *z)
    g, n = H.ngz, H.n
    assert np.array_equal(st[:, :, g:g + n, g:g + n, g:g + n], before[:, :, g:g + n, g:g + n, g:g + n])
    m = H.gather_maps()["cells"]
    same = (m["cnt"] == 1) & (m["w"][0] == 1.0)
    assert same.mean() > 0.5
    flat, ref = st.reshape(-1), before.reshape(-1)
    assert np.array_equal(flat[m["dst"][same]], ref[m["src"][0][same]])


@pytest.mark.parametrize("which", ["tov", "torus"])
def test_gather_sources_are_interior(which):
    """Every source of the ghost-fill maps is an interior cell or face (no
    source is written by the same fill), also beyond non-periodic
    boundaries, so the device fill can run every entry at once."""
    H = workloads.tov_hierarchy(8) if which == "tov" else workloads.torus_hierarchy(8)
    for key, m in H.gather_maps().items():
        used = np.arange(8)[:, None] < m["cnt"][None, :]
        assert not np.any(np.isin(m["src"][used], m["dst"])), key


def test_gather_runs_partition_the_maps_and_name_their_sources():
    """gather_runs: the runs' maps split every entry of the hierarchy's maps
    by the run of its destination, and deps[r] holds the run of every
    source block those entries read."""
    from grace_b200.host import Blocks, gather_runs
    H = workloads.tov_hierarchy(8)
    maps = H.gather_maps()
    blocks = Blocks(H.n, H.n, H.n, H.ngz, H.nq, H.idx(), device="cpu")
    runs, run_maps, deps = gather_runs(maps, blocks, 6)
    assert runs[0][0] == 0 and runs[-1][1] == H.nq and len(runs) == 6
    NN = H.n + 2 * H.ngz
    qs = {"cells": abi.N_EVOL_VARS * NN ** 3, 0: (NN + 1) * NN * NN, 1: (NN + 1) * NN * NN, 2: (NN + 1) * NN * NN}
    for key, m in maps.items():
        assert sum(rm[key]["dst"].size for rm in run_maps) == m["dst"].size
        got = np.sort(np.concatenate([rm[key]["dst"] for rm in run_maps]))
        np.testing.assert_array_equal(got, np.sort(m["dst"]))
        for r, ((q0, q1), rm) in enumerate(zip(runs, run_maps)):
            d = rm[key]["dst"] // qs[key]
            assert np.all((d >= q0) & (d < q1))
            used = np.arange(8)[:, None] < rm[key]["cnt"][None, :]
            src_q = rm[key]["src"][used] // qs[key]
            src_runs = {int(np.searchsorted([b for _, b in runs], q, side="right")) for q in np.unique(src_q)}
            assert src_runs <= deps[r], (key, r)
    assert any(len(d) > 1 for d in deps)
