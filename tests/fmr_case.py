"""Two-level FMR case for the reflux tests (test infrastructure): a 2x2x2
periodic brick of 8^3 blocks on [-3, 3]^3 whose block (0, 0, 0) is refined
into 8 children (15 leaves: 6 hanging faces, 24 hanging edges), the blast
wave's overdense sphere at the corner all levels share, uniform Bx, a
smooth shearing flow (nonzero EMFs from the first substep).  Ghosts
by the composite fill of grace_b200.fmr (same-level ghosts are exact
copies, so same-level faces see the same fluxes from both sides)."""
import numpy as np

from grace_b200 import abi, fmr, params, workloads


def two_level_case():
    H = fmr.Hierarchy((2, 2, 2), 8, (-3, -3, -3), (3, 3, 3), lambda l, b: l == 0 and b == (0, 0, 0), 1)
    st, bx, by, bz, aux = workloads.fmr_blast(H, flow=0.1)
    H.fill_ghosts(st, bx, by, bz)
    P = params.blast()
    return H, P, (st, bx, by, bz, aux)


def interior_mass(H, state):
    """Sum of D dV over the interiors of all leaves."""
    g, n = H.ngz, H.n
    m = 0.0
    for q, (l, _) in enumerate(H.leaves):
        m += float(np.sum(state[q, abi.DENS, g:g + n, g:g + n, g:g + n])) * float(np.prod(H.dx(l)))
    return m


def hanging_face_mismatch(H, R, fields):
    """Largest |coarse face B - mean of the 4 fine face B it covers| over all
    hanging faces, relative to the largest |B|: zero when the coarse and
    fine sides carry the same magnetic flux through the interface."""
    g, n, h = H.ngz, H.n, H.n // 2
    worst, scale = 0.0, max(float(np.max(np.abs(a))) for a in fields[1:])
    for i, (qc, face) in enumerate(zip(R["face_coarse_q"], R["face_coarse_id"])):
        d, side = face // 2, face & 1
        o1, o2 = fmr.ODIR[d]
        arr = fields[1 + d]
        # array index order (k, j, i): axis a sits at position 2 - a
        def plane(q, pos):
            sl = [slice(g, g + n)] * 3
            sl[2 - d] = pos
            return arr[q][tuple(sl)]  # 2-D, axes (o2, o1) in array order
        pc = plane(qc, g + n if side else g)
        for c in range(4):
            pf = plane(R["face_fine_q"][4 * i + c], g if side else g + n)
            a, b = c & 1, c >> 1
            fine = 0.25 * (pf[0::2, 0::2] + pf[1::2, 0::2] + pf[0::2, 1::2] + pf[1::2, 1::2])
            coarse = pc[b * h:(b + 1) * h, a * h:(a + 1) * h]
            worst = max(worst, float(np.max(np.abs(coarse - fine))))
    return worst / scale
