"""Parity metrics shared by the tests.

Conserved variables are compared cell by cell with a state-normalised
relative error: D, tau, Ye*D and s*D relative to their own magnitude,
the momenta S_i relative to max(|S|, tau + D) — the bound |S| <= tau + D
that the c2p's limit_conservatives enforces (c2p.cpp:138-150).  Plain
per-component relative errors are ill-posed for momenta that are zero up
to rounding (a resting background with 1e-3 pressure noise)."""
import numpy as np


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
        else:
            s = np.abs(b[:, v])
        ok = (s > floor) | (d > 0)
        out[v] = np.max(np.where(ok, d / np.maximum(s, floor), 0.0))
    return out


def interior(x, g):
    return x[..., g:-g, g:-g, g:-g]
