"""Parity metrics shared by the tests.

Conserved variables are compared cell by cell with a state-normalised
relative error: D, tau, Ye*D and s*D relative to their own magnitude,
the momenta S_i relative to max(|S|, tau + D) — the bound |S| <= tau + D
that the c2p's limit_conservatives enforces (c2p.cpp:138-150).  Plain
per-component relative errors are ill-posed for momenta that are zero up
to rounding (a resting background with 1e-3 pressure noise).  The entropy density
s* = D s is taken relative to D max(|s|, 1): s is a logarithm that may
cross zero."""
import numpy as np

from grace_b200 import abi


def cons_rel_err(a, b, floor=1e-300):
    """a, b: (nq, >=7, NZ, NY, NX) state arrays (interior slice); returns
    the max state-normalised relative error per HRSC variable."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    out = np.zeros(7)
    scale_S = np.maximum(np.max(np.abs(b[:, 1:4]), axis=1), np.abs(b[:, 4]) + np.abs(b[:, 0]))
    for v in range(7):
        d = np.abs(a[:, v] - b[:, v])
        if 1 <= v <= 3:
            s = scale_S
        elif v == 6:
            # s* = D s with the specific entropy s a logarithm: relative to
            # D max(|s|, 1), ill-posed where s crosses zero otherwise
            s = np.maximum(np.abs(b[:, v]), np.abs(b[:, 0]))
        else:
            s = np.abs(b[:, v])
        ok = (s > floor) | (d > 0)
        out[v] = np.max(np.where(ok, d / np.maximum(s, floor), 0.0))
    return out


def interior(x, g):
    return x[..., g:-g, g:-g, g:-g]


# ---- c2p primitives -------------------------------------------------------
PRIM_TOL = 1e-12  # relative, per primitive


def state_residual(a, b):
    """State-normalised infinity-norm residual of test/test_c2p.cpp:80-98:
    max |a-b| over (rho, eps, z^i) divided by max(|rho|, |eps|, |z|)."""
    zm = np.sqrt(np.sum(b[abi.P_ZX:abi.P_ZZ + 1] ** 2, axis=0))
    scale = np.maximum(np.maximum(np.abs(b[abi.P_RHO]), np.abs(b[abi.P_EPS])), np.maximum(zm, 1e-30))
    d = np.zeros(b.shape[1])
    for v in (abi.P_RHO, abi.P_EPS, abi.P_ZX, abi.P_ZY, abi.P_ZZ):
        d = np.maximum(d, np.abs(a[v] - b[v]))
    return d / scale


def prim_tol(prims):
    """Per-state tolerance: 1e-12, widened by W^2 for fast flows.  Brent stops
    within t = 1e-15 of the root in mu (kastaun_c2p.hh:372); through
    W = (1 - rbar^2 mu^2)^(-1/2) an abscissa shift dmu moves W (and
    rho = D/W) by ~W^2 dmu/mu, so two correct solvers that stop at different
    points of the tolerance window differ by up to ~1e-13 W^2."""
    W = np.sqrt(1.0 + np.sum(prims[abi.P_ZX:abi.P_ZZ + 1] ** 2, axis=0))
    return PRIM_TOL * np.maximum(1.0, W * W)


def tuned_aux_mask(su):
    """Cells that the tuned aux pass (GS EMF) maintains in every block: at
    least two indices in [g-1, n+g+1), or all three in [g-2, n+g+2).
    Boolean array (NZ, NY, NX)."""
    g = su.ngz
    axes = []
    for n in (su.n[2], su.n[1], su.n[0]):
        c = np.arange(n + 2 * g)
        axes.append(((c >= g - 1) & (c < n + g + 1), (c >= g - 2) & (c < n + g + 2)))
    tz, ty, tx = (a[0] for a in axes)
    dz, dy, dx = (a[1] for a in axes)
    T = (tz[:, None, None].astype(int) + ty[None, :, None].astype(int) + tx[None, None, :].astype(int))
    D = dz[:, None, None] & dy[None, :, None] & dx[None, None, :]
    return (T >= 2) | D
