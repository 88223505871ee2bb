"""Curved-metric Cowling setup for stage parity tests (test infrastructure).

Schwarzschild in Cartesian Kerr-Schild coordinates (M = 1), on a brick away
from the horizon: g_ij = delta_ij + 2H l_i l_j, beta^i = 2H l^i / (1 + 2H),
alpha = (1 + 2H)^(-1/2), H = M/r, l = x/r, set analytically in every cell
(ghosts included).  The extrinsic curvature only has to be smooth and the
same on both sides of a parity test: K_ij = (d_i beta_j + d_j beta_i) / (2
alpha) with beta_j = g_jk beta^k, by central differences of the analytic
fields.  Matter: a Gaussian polytropic blob (hybrid EOS, K = 100, Gamma = 2,
Gamma_th = 1.8) with a smooth rotating velocity and a field from a
vector potential A_z, so that the densitized face fields are discretely
divergence free.  Conserved variables come from the oracle's
prims_to_conservs on the curved metric."""
import ctypes as C

import numpy as np

import _oracle
from grace_b200 import abi, params
from grace_b200.workloads import BrickSetup


def ks_fields(x, y, z):
    r = np.sqrt(x * x + y * y + z * z)
    H = 1.0 / r
    l = np.stack([x, y, z]) / r
    g = np.empty((6,) + x.shape)
    for a, (i, j) in enumerate(((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))):
        g[a] = (1.0 if i == j else 0.0) + 2 * H * l[i] * l[j]
    beta = 2 * H * l / (1 + 2 * H)
    alp = 1.0 / np.sqrt(1 + 2 * H)
    return g, beta, alp


def _beta_low(x, y, z):
    g, b, _ = ks_fields(x, y, z)
    G = [[g[0], g[1], g[2]], [g[1], g[3], g[4]], [g[2], g[4], g[5]]]
    return np.stack([sum(G[j][k] * b[k] for k in range(3)) for j in range(3)])


def cold_pwpoly(e, rho):
    """Cold pressure and specific energy of the piecewise polytrope in the
    EOS parameters e (piece i for pw_rho[i] < rho <= pw_rho[i+1], the last
    piece above; piecewise_polytropic_eos.hh:51-190)."""
    n = e.n_pieces
    i = np.zeros(rho.shape, dtype=int)
    for k in range(1, n):
        i = np.where(rho > e.pw_rho[k], k, i)
    K = np.asarray(e.pw_kappa[:n])[i]
    G = np.asarray(e.pw_gamma[:n])[i]
    E = np.asarray(e.pw_eps[:n])[i]
    pc = K * rho ** G
    return pc, E + pc / (rho * (G - 1.0))


def curved_setup(nb=(2, 2, 2), n=(8, 8, 8), emf=abi.EMF_GS, fofc=1, pieces=None):
    """pieces: (kappa_0, gammas, rhos) of a piecewise-polytropic cold part
    (default: one piece, K = 100, Gamma = 2)."""
    kappa, gammas, rhos = pieces if pieces is not None else (100.0, [2.0], [])
    P = params.hybrid_pwpoly(kappa, gammas, rhos, gamma_th=1.8, emf=emf, fofc_enable=fofc,
                             max_sigma=1.0e4)
    su = BrickSetup(nb, n, (3.0, -1.0, -1.0), (5.0, 1.0, 1.0), 4, (False, False, False))
    state, bx, by, bz, aux = su.empty()
    X = su.cell_centres()
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    g, beta, alp = ks_fields(x, y, z)
    for a in range(6):
        state[:, abi.GXX + a] = g[a]
    state[:, abi.ALP] = alp
    for a in range(3):
        state[:, abi.BETAX + a] = beta[a]
    h = 1e-5
    dbl = []
    for d in range(3):
        e = [0.0, 0.0, 0.0]
        e[d] = h
        dbl.append((_beta_low(x + e[0], y + e[1], z + e[2]) - _beta_low(x - e[0], y - e[1], z - e[2])) / (2 * h))
    for a, (i, j) in enumerate(((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))):
        state[:, abi.KXX + a] = (dbl[i][j] + dbl[j][i]) / (2 * alp)
    # matter
    c, sig = np.array([4.0, 0.0, 0.0]), 0.5
    q2 = ((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / sig ** 2
    rho = 1e-3 * np.exp(-q2) + 1e-7
    eth = np.full_like(rho, 1e-4 / 0.8)
    pc, ec = cold_pwpoly(P.eos, rho)
    press = pc + 0.8 * rho * eth
    eps = ec + eth
    zv = 0.1 * np.exp(-0.5 * q2) * np.stack([-y, x - c[0], 0.3 * np.ones_like(x)])
    # densitized face fields from A_z on z-edges (cell corners in x-y)
    dx = su.dx
    for t, q in enumerate(su.blocks()):
        o = su.block_origin(q)
        NX, NY, NZ = su.N
        xe = o[0] + (np.arange(NX + 1) - 4) * dx[0]
        ye = o[1] + (np.arange(NY + 1) - 4) * dx[1]
        zc = o[2] + (np.arange(NZ) - 4 + 0.5) * dx[2]
        Z, Y, Xe = np.meshgrid(zc, ye, xe, indexing="ij")
        Az = 2e-4 * np.exp(-((Xe - c[0]) ** 2 + Y ** 2 + Z ** 2) / sig ** 2)
        bx[t] = (Az[:, 1:, :] - Az[:, :-1, :]) / dx[1]
        by[t] = -(Az[:, :, 1:] - Az[:, :, :-1]) / dx[0]
    bz[:] = 0.0
    Bt = np.stack([0.5 * (bx[..., :-1] + bx[..., 1:]), 0.5 * (by[:, :, :-1, :] + by[:, :, 1:, :]),
                   0.5 * (bz[:, :-1] + bz[:, 1:])])
    gdet = g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] * (g[1] * g[5] - g[2] * g[4]) + g[2] * (g[1] * g[4] - g[2] * g[3])
    sq = np.sqrt(gdet)
    # prims (13 per cell) -> densitized cons on the curved metric (oracle)
    npt = rho.size
    pr = np.zeros((13, npt))
    pr[abi.P_RHO], pr[abi.P_PRESS], pr[abi.P_EPS] = rho.ravel(), press.ravel(), eps.ravel()
    for a in range(3):
        pr[abi.P_ZX + a] = zv[a].ravel()
        pr[abi.P_BX + a] = (Bt[a] / sq).ravel()
    pr[abi.P_TEMP] = (eth * 0.8).ravel()
    pr[abi.P_ENT] = (np.log(eth * rho ** (-0.8)) / 0.8).ravel()
    met = np.zeros((10, npt))
    for a in range(6):
        met[a] = g[a].ravel()
    for a in range(3):
        met[6 + a] = beta[a].ravel()
    met[9] = alp.ravel()
    cons = np.zeros((10, npt))
    L = _oracle.lib("orc")
    L.orc_prims_to_conservs(C.byref(P), npt, _oracle.p(pr), _oracle.p(met), _oracle.p(cons))
    for v in range(7):
        state[:, v] = cons[v].reshape(rho.shape)
    aux[:, abi.RHO], aux[:, abi.PRESS], aux[:, abi.EPS] = rho, press, eps
    for a in range(3):
        aux[:, abi.ZVECX + a] = zv[a]
        aux[:, abi.BX + a] = Bt[a] / sq
    aux[:, abi.TEMP] = eth * 0.8
    aux[:, abi.ENTROPY] = np.log(eth * rho ** (-0.8)) / 0.8
    return P, su, (state, bx, by, bz, aux)
