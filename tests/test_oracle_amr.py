"""FMR restriction oracle (oracle/amr_oracle.hpp) pinned to the reference's
own restriction operators (include/grace/amr/ghostzone_kernels/pr_helpers.hh
compiled in place, oracle/_ref): bit for bit on random data, every child
position, both variable lists."""
import os

import numpy as np
import pytest

import _oracle

N, G = 16, 4
NN = N + 2 * G


@pytest.mark.skipif(not os.path.exists(_oracle.REF), reason="pinning build absent")
def test_restrict_cells_matches_reference_operators():
    rng = np.random.default_rng(21)
    nvars, nq, ncb = 5, 8, 8
    src = rng.standard_normal((nq, nvars, NN, NN, NN))
    src_q = np.arange(nq)
    dst_q = rng.permutation(ncb)[:nq]
    child = np.arange(8, dtype=np.uint8)  # every Morton child position
    vlo, vhi = [0, 3], [1, 2, 4]
    out = {}
    for which in ("orc", "ref"):
        dst = np.zeros((ncb, nvars, NN, NN, NN))
        _oracle.restrict_cells(which, N, G, nvars, src, dst, src_q, dst_q, child, vlo, vhi)
        out[which] = dst
    np.testing.assert_array_equal(out["orc"], out["ref"])
    # the coarse interior of every buffer was written, nothing else
    sl = (slice(None), slice(None), slice(G, G + N // 2), slice(G, G + N // 2), slice(G, G + N // 2))
    mask = np.zeros_like(out["orc"], dtype=bool)
    mask[sl] = True
    assert not out["orc"][~mask].any()
    assert np.all(out["orc"][sl] != 0.0)


def test_restriction_reproduces_polynomials():
    """Restriction is exact for the fields it should be: the 8-cell average
    for linear data (cell averages at the coarse centre) and the 5-point
    Lagrange stencils for quartics (point values at the coarse centre)."""
    x = np.arange(NN) - G + 0.5  # fine cell centres, fine spacing 1
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    lin = (1.5 + 0.25 * X - 0.5 * Y + 0.125 * Z).transpose(2, 1, 0)
    quart = (0.1 * X ** 4 - 0.3 * X * Y ** 2 + 0.05 * Z ** 3 * Y + 2.0).transpose(2, 1, 0)
    src = np.stack([lin, quart])[None]  # (1, 2, NN, NN, NN), C order = (z, y, x)
    dst = np.zeros_like(src)
    _oracle.restrict_cells("orc", N, G, 2, src, dst, [0], [0], [0], [0], [1])
    xc = 2 * np.arange(N // 2) + 1.0  # coarse centres in fine units (interior origin)
    XC, YC, ZC = np.meshgrid(xc, xc, xc, indexing="ij")
    sl = (slice(G, G + N // 2),) * 3
    np.testing.assert_allclose(dst[0, 0][sl], (1.5 + 0.25 * XC - 0.5 * YC + 0.125 * ZC).transpose(2, 1, 0),
                               rtol=0, atol=1e-13)
    np.testing.assert_allclose(dst[0, 1][sl], (0.1 * XC ** 4 - 0.3 * XC * YC ** 2 + 0.05 * ZC ** 3 * YC
                                               + 2.0).transpose(2, 1, 0), rtol=0, atol=1e-9)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_face_restriction_preserves_divergence(d):
    """The 4-face average of a divergence-free fine face field gives a
    divergence-free coarse face field (flux through each coarse face = sum
    of its 4 fine faces)."""
    rng = np.random.default_rng(5 + d)
    # fine face B from a vector potential: B = curl A on the fine grid
    A = [rng.standard_normal((NN + 1, NN + 1, NN + 1)) for _ in range(3)]  # edge-centred, (z, y, x)
    Ax, Ay, Az = A
    bx = (Az[:NN, 1:NN + 1, :NN + 1] - Az[:NN, :NN, :NN + 1]) - (Ay[1:NN + 1, :NN, :NN + 1] - Ay[:NN, :NN, :NN + 1])
    by = (Ax[1:NN + 1, :NN + 1, :NN] - Ax[:NN, :NN + 1, :NN]) - (Az[:NN, :NN + 1, 1:NN + 1] - Az[:NN, :NN + 1, :NN])
    bz = (Ay[:NN + 1, :NN, 1:NN + 1] - Ay[:NN + 1, :NN, :NN]) - (Ax[:NN + 1, 1:NN + 1, :NN] - Ax[:NN + 1, :NN, :NN])
    fine = [np.ascontiguousarray(b)[None] for b in (bx, by, bz)]
    coarse = [np.zeros_like(f) for f in fine]
    for k in range(3):
        _oracle.restrict_faces(k, N, G, fine[k], coarse[k], [0], [0])
    cx, cy, cz = (c[0] for c in coarse)
    h = N // 2
    s = slice(G, G + h)
    div = (cx[s, s, G + 1:G + h + 1] - cx[s, s, s]) + (cy[s, G + 1:G + h + 1, s] - cy[s, s, s]) + \
          (cz[G + 1:G + h + 1, s, s] - cz[s, s, s])
    assert np.max(np.abs(div)) < 1e-13
