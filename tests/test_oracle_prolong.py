"""FMR ghost-zone prolongation oracle (oracle/amr_oracle.hpp) pinned to the
reference's own prolongation functors (prolong_op and div_free_prolong_op of
include/grace/amr/ghostzone_kernels/prolongation_kernels.hh, with their index
maps and operators, compiled in place in oracle/_ref): bit for bit on random
data for every element of every kind, both variable lists, random
fine-neighbour flags; and the properties the operators are built for."""
import os

import numpy as np
import pytest

import _oracle

N, G = 16, 4
NN = N + 2 * G
NELEM = {0: 6, 1: 12, 2: 8}
FACE_SHAPES = [(NN, NN, NN + 1), (NN, NN + 1, NN), (NN + 1, NN, NN)]  # C order (z, y, x) of bx, by, bz


def _elements(kind, nq, rng):
    """Every element of the kind on each of nq fine quadrants, shuffled."""
    fq = np.repeat(np.arange(nq), NELEM[kind])
    el = np.tile(np.arange(NELEM[kind]), nq)
    order = rng.permutation(len(fq))
    return fq[order], el[order]


@pytest.mark.skipif(not os.path.exists(_oracle.REF), reason="pinning build absent")
@pytest.mark.parametrize("n", [16, 8, 4])
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_prolong_cells_matches_reference_functor(kind, n):
    rng = np.random.default_rng(40 + kind + n)
    nvars, nq = 5, 2
    NN = n + 2 * G
    N = n
    cbuf = rng.standard_normal((nq, nvars, NN, NN, NN))
    fq, el = _elements(kind, nq, rng)
    cmap = rng.permutation(nq)
    cq = cmap[fq]
    vlo, vhi = [0, 3], [1, 2, 4]
    out = {}
    for which in ("orc", "ref"):
        fine = np.zeros((nq, nvars, NN, NN, NN))
        _oracle.prolong_cells(which, kind, N, G, nvars, fine, cbuf, fq, cq, el, vlo, vhi)
        out[which] = fine
    np.testing.assert_array_equal(out["orc"], out["ref"])
    # every ghost cell of the kind's elements written, the interior untouched
    inner = (slice(None), slice(None)) + (slice(G, G + N),) * 3
    assert not out["orc"][inner].any()
    written = np.count_nonzero(out["orc"])
    per_q = {0: 6 * G * N * N, 1: 12 * G * G * N, 2: 8 * G ** 3}[kind]
    assert written == nq * nvars * per_q


@pytest.mark.skipif(not os.path.exists(_oracle.REF), reason="pinning build absent")
@pytest.mark.parametrize("n", [16, 8, 4])
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_prolong_faces_matches_reference_functor(kind, n):
    rng = np.random.default_rng(50 + kind + n)
    nq = 2
    M = n + 2 * G
    N = n
    shapes = [(M, M, M + 1), (M, M + 1, M), (M + 1, M, M)]
    cb = [rng.standard_normal((nq,) + s) for s in shapes]
    init = [rng.standard_normal((nq,) + s) for s in shapes]  # "fine data" where flags say so
    fq, el = _elements(kind, nq, rng)
    cq = rng.permutation(nq)[fq]
    hf = rng.integers(0, 2, size=(len(fq), 3, 2)).astype(np.int8)
    out = {}
    for which in ("orc", "ref"):
        fine = [a.copy() for a in init]
        _oracle.prolong_faces(which, kind, N, G, fine, cb, fq, cq, el, hf)
        out[which] = fine
    for a, b, i in zip(out["orc"], out["ref"], init):
        np.testing.assert_array_equal(a, b)
        assert np.count_nonzero(a != i) > 0


def _centres():
    x = np.arange(NN) - G + 0.5  # fine cell centres, interior origin, fine spacing 1
    xc = 2.0 * (np.arange(NN) - G) + 1.0  # coarse centres in fine units (coarse spacing 2)
    return x, xc


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_prolongation_reproduces_polynomials(kind):
    """The slope-limited operator is exact for monotone linear data (minmod
    returns the one slope) and the 5-point Lagrange operator for quartics."""
    x, xc = _centres()
    f_lin = lambda X, Y, Z: 1.5 + 0.25 * X - 0.5 * Y + 0.125 * Z
    f_q = lambda X, Y, Z: 0.01 * X ** 4 - 0.03 * X * Y ** 2 + 0.005 * Z ** 3 * Y + 2.0
    Xc, Yc, Zc = np.meshgrid(xc, xc, xc, indexing="ij")
    cbuf = np.stack([f_lin(Xc, Yc, Zc), f_q(Xc, Yc, Zc)]).transpose(0, 3, 2, 1)[None].copy()
    fine = np.zeros_like(cbuf)
    el = np.arange(NELEM[kind])
    _oracle.prolong_cells("orc", kind, N, G, 2, fine, cbuf, np.zeros_like(el), np.zeros_like(el), el, [0], [1])
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    want = np.stack([f_lin(X, Y, Z), f_q(X, Y, Z)]).transpose(0, 3, 2, 1)
    m = fine[0] != 0
    assert m[0].sum() == {0: 6 * G * N * N, 1: 12 * G * G * N, 2: 8 * G ** 3}[kind]
    np.testing.assert_allclose(fine[0, 0][m[0]], want[0][m[0]], rtol=0, atol=1e-13)
    np.testing.assert_allclose(fine[0, 1][m[1]], want[1][m[1]], rtol=0, atol=1e-10)


def _div_free_coarse(rng):
    """Coarse face B = discrete curl of a random edge vector potential on the
    coarse buffer's grid (coarse spacing 1): divergence zero to round-off in
    every coarse cell."""
    Ax = rng.standard_normal((NN + 1, NN + 1, NN))  # (z, y, x): edges along x
    Ay = rng.standard_normal((NN + 1, NN, NN + 1))
    Az = rng.standard_normal((NN, NN + 1, NN + 1))
    bx = (Az[:, 1:, :] - Az[:, :-1, :]) - (Ay[1:, :, :] - Ay[:-1, :, :])  # (NN, NN, NN+1)
    by = (Ax[1:, :, :] - Ax[:-1, :, :]) - (Az[:, :, 1:] - Az[:, :, :-1])  # (NN, NN+1, NN)
    bz = (Ay[:, :, 1:] - Ay[:, :, :-1]) - (Ax[:, 1:, :] - Ax[:, :-1, :])  # (NN+1, NN, NN)
    return [bx[None].copy(), by[None].copy(), bz[None].copy()]


def test_face_prolongation_preserves_divergence():
    """Prolonging divergence-free coarse faces into every face, edge and
    corner element leaves every fine ghost cell of those elements with
    divergence at round-off (Toth-Roe's construction), when no neighbour
    holds fine data."""
    rng = np.random.default_rng(7)
    cb = _div_free_coarse(rng)
    fine = [np.full((1,) + s, np.nan) for s in FACE_SHAPES]
    for kind in (0, 1, 2):
        el = np.arange(NELEM[kind])
        z = np.zeros_like(el)
        _oracle.prolong_faces("orc", kind, N, G, fine, cb, z, z, el, np.zeros((len(el), 3, 2), np.int8))
    bx, by, bz = fine[0][0], fine[1][0], fine[2][0]
    div = (bx[:, :, 1:] - bx[:, :, :-1]) + (by[:, 1:, :] - by[:, :-1, :]) + (bz[1:] - bz[:-1])
    ghost = np.ones((NN, NN, NN), bool)
    ghost[G:G + N, G:G + N, G:G + N] = False
    assert np.isfinite(div[ghost]).all()  # every face of every ghost cell written
    scale = max(np.abs(a).max() for a in cb)
    assert np.abs(div[ghost]).max() <= 1e-13 * scale
