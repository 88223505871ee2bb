"""Seeded synthetic inputs of the benchmark configurations (numpy, host).

None of these is a public benchmark suite; they are initial data written
directly from the configuration text (the reference's own initial-data
routines for these setups are absent or differ, see the design notes):
  * Balsara-1 shock tube (ideal gas Gamma=2), 1024x16x16 cells in 16^3 blocks
  * 3-D blast wave (ideal gas Gamma=4/3), 256^3 cells in 4096 blocks of 16^3
  * c2p micro-benchmark states (hybrid EOS K=100, Gamma=2, Gamma_th=1.8)
Initial data follow GRACE's convention (src/physics/grmhd.cpp:380-530):
primitives into aux, the metric into state, face B = B * sqrt(gamma), then
conserved variables from the primitives (set_conservs_from_prims,
src/physics/grmhd.cpp:676-759) — here on the flat metric.
"""
import numpy as np

from . import abi

SEED = 0x6A5CE


def flat_prims_to_cons(rho, press, eps, z, B, s, ye=None):
    """Conserved variables on the flat metric (sqrt(gamma)=1, alpha=1, beta=0).

    rho, press, eps, s: (...); z, B: (3, ...).  Returns (7, ...) in the order
    DENS, SX, SY, SZ, TAU, YESTAR, ENTROPYSTAR."""
    W = np.sqrt(1.0 + np.sum(z * z, axis=0))
    Bz = np.sum(B * z, axis=0)
    b = (B + Bz[None] * z) / W[None]
    b2 = (np.sum(B * B, axis=0) + Bz * Bz) / (W * W)
    rhoh = rho * (1.0 + eps) + press + b2
    D = rho * W
    tau = rhoh * W * W - press - 0.5 * b2 - Bz * Bz - D
    S = rhoh[None] * W[None] * z - Bz[None] * b
    out = np.zeros((7,) + rho.shape)
    out[0] = D
    out[1:4] = S
    out[4] = tau
    out[5] = D * (0.0 if ye is None else ye)
    out[6] = s * D
    return out


class BrickSetup:
    """A brick of nbx*nby*nbz blocks of n^3 cells on [lo, hi]^3 (flat metric)."""

    def __init__(self, nb, n, lo, hi, ngz=4, periodic=(False, False, False)):
        self.nb = tuple(nb)
        self.n = tuple(n)
        self.ngz = ngz
        self.lo = np.asarray(lo, float)
        self.hi = np.asarray(hi, float)
        self.periodic = tuple(periodic)
        self.nq = nb[0] * nb[1] * nb[2]
        self.dx = (self.hi - self.lo) / (np.asarray(nb) * np.asarray(n))
        self.N = tuple(ni + 2 * ngz for ni in n)

    def idx(self):
        return np.tile(1.0 / self.dx, (self.nq, 1))

    def block_origin(self, q):
        qc = (q % self.nb[0], (q // self.nb[0]) % self.nb[1], q // (self.nb[0] * self.nb[1]))
        return np.array([self.lo[a] + qc[a] * self.n[a] * self.dx[a] for a in range(3)])

    def coords(self):
        """Centre of cell (0,0,0) (a ghost cell) of each block."""
        return np.stack([self.block_origin(q) + (0.5 - self.ngz) * self.dx for q in range(self.nq)])

    def blocks(self, qr=None):
        return range(self.nq) if qr is None else range(*qr)

    def outer_faces(self):
        """(quad, face) of every block face on a non-periodic outer boundary
        of the brick, face = 2 axis + side (side 1 upper): the list GRACE's
        face iterator collects for the outflow diagnostic."""
        quad, face = [], []
        for q in range(self.nq):
            qc = (q % self.nb[0], (q // self.nb[0]) % self.nb[1], q // (self.nb[0] * self.nb[1]))
            for a in range(3):
                if self.periodic[a]:
                    continue
                if qc[a] == 0:
                    quad.append(q)
                    face.append(2 * a)
                if qc[a] == self.nb[a] - 1:
                    quad.append(q)
                    face.append(2 * a + 1)
        return np.array(quad, np.int64), np.array(face, np.uint8)

    def cell_centres(self, qr=None):
        """(nq, 3, NZ, NY, NX) physical cell centres, ghosts included."""
        NX, NY, NZ = self.N
        i = np.arange(NX)
        j = np.arange(NY)
        k = np.arange(NZ)
        qs = self.blocks(qr)
        out = np.empty((len(qs), 3, NZ, NY, NX))
        for t, q in enumerate(qs):
            o = self.block_origin(q)
            out[t, 0] = o[0] + (i[None, None, :] - self.ngz + 0.5) * self.dx[0]
            out[t, 1] = o[1] + (j[None, :, None] - self.ngz + 0.5) * self.dx[1]
            out[t, 2] = o[2] + (k[:, None, None] - self.ngz + 0.5) * self.dx[2]
        return out

    def global_cell_index(self, qr=None):
        """(nq, 3, NZ, NY, NX) global (unwrapped) integer cell coordinates."""
        NX, NY, NZ = self.N
        qs = self.blocks(qr)
        gi = np.empty((len(qs), 3, NZ, NY, NX), dtype=np.int64)
        for t, q in enumerate(qs):
            qc = (q % self.nb[0], (q // self.nb[0]) % self.nb[1], q // (self.nb[0] * self.nb[1]))
            gi[t, 0] = qc[0] * self.n[0] + np.arange(NX)[None, None, :] - self.ngz
            gi[t, 1] = qc[1] * self.n[1] + np.arange(NY)[None, :, None] - self.ngz
            gi[t, 2] = qc[2] * self.n[2] + np.arange(NZ)[:, None, None] - self.ngz
        return gi

    def empty(self, qr=None):
        NX, NY, NZ = self.N
        nq = len(self.blocks(qr))
        state = np.zeros((nq, abi.N_EVOL_VARS, NZ, NY, NX))
        bx = np.zeros((nq, NZ, NY, NX + 1))
        by = np.zeros((nq, NZ, NY + 1, NX))
        bz = np.zeros((nq, NZ + 1, NY, NX))
        aux = np.zeros((nq, abi.N_AUX_VARS, NZ, NY, NX))
        # flat Cowling metric: g = 1, alpha = 1, beta = K = 0
        state[:, abi.GXX] = state[:, abi.GYY] = state[:, abi.GZZ] = 1.0
        state[:, abi.ALP] = 1.0
        return state, bx, by, bz, aux


def _counter_uniform(gid, seed, nx_glob):
    """U(-1,1) from a counter hash of the global cell index (block-order free)."""
    key = (gid[:, 0].astype(np.uint64) + np.uint64(nx_glob[0]) *
           (gid[:, 1].astype(np.uint64) + np.uint64(nx_glob[1]) * gid[:, 2].astype(np.uint64)))
    x = key * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)
    x ^= x >> np.uint64(30)
    x *= np.uint64(0xBF58476D1CE4E5B9)
    x ^= x >> np.uint64(27)
    x *= np.uint64(0x94D049BB133111EB)
    x ^= x >> np.uint64(31)
    return (x >> np.uint64(11)).astype(np.float64) / float(1 << 53) * 2.0 - 1.0


def _fill(setup, gamma, rho, press, B_cell, Bface_fn, qr=None):
    """Write primitives / conserved / face B for an ideal gas on the flat metric."""
    state, bx, by, bz, aux = setup.empty(qr)
    eps = press / ((gamma - 1.0) * rho)
    T = eps * (gamma - 1.0)
    s = np.log(eps) / (gamma - 1.0) - np.log(rho)
    z = np.zeros((3,) + rho.shape)
    Bx, By, Bz = Bface_fn(bx.shape, by.shape, bz.shape)
    bx[:], by[:], bz[:] = Bx, By, Bz
    Bc = np.stack([0.5 * (bx[..., :-1] + bx[..., 1:]),
                   0.5 * (by[:, :, :-1, :] + by[:, :, 1:, :]),
                   0.5 * (bz[:, :-1] + bz[:, 1:])])
    cons = flat_prims_to_cons(rho, press, eps, z, Bc, s)
    state[:, 0:7] = np.moveaxis(cons, 0, 1)
    aux[:, abi.RHO] = rho
    aux[:, abi.PRESS] = press
    aux[:, abi.EPS] = eps
    aux[:, abi.TEMP] = T
    aux[:, abi.ENTROPY] = s
    aux[:, abi.BX:abi.BZ + 1] = np.moveaxis(Bc, 0, 1)
    return state, bx, by, bz, aux


def blast(nb=(16, 16, 16), n=(16, 16, 16), ngz=4, seed=SEED, qr=None, lo=(-6, -6, -6),
          hi=(6, 6, 6)):
    """3-D blast wave: Gamma=4/3, rho=1e-4 / p=5e-4 outside, rho=1e-2 / p=1
    inside r<0.8, Bx=0.1, domain [-6,6]^3, pressure x (1 + 1e-3 U(-1,1))
    seeded per global cell.  Outflow boundaries.  qr=(q0, q1) restricts the
    arrays to blocks q0..q1-1 (the values do not depend on the chunking);
    lo/hi select a sub-box of the domain (same cell size for a proportional
    block count)."""
    su = BrickSetup(nb, n, lo, hi, ngz, (False, False, False))
    X = su.cell_centres(qr)
    r = np.sqrt(np.sum(X * X, axis=1))
    inside = r < 0.8
    rho = np.where(inside, 1e-2, 1e-4)
    press = np.where(inside, 1.0, 5e-4)
    gid = su.global_cell_index(qr)
    ng = np.asarray(nb) * np.asarray(n) + 2 * ngz
    u = _counter_uniform(np.moveaxis(gid, 1, -1).reshape(-1, 3) + ngz, seed, ng).reshape(rho.shape)
    press = press * (1.0 + 1e-3 * u)

    def faces(sx, sy, sz):
        return np.full(sx, 0.1), np.zeros(sy), np.zeros(sz)

    return su, _fill(su, 4.0 / 3.0, rho, press, None, faces, qr)


def blast_drifting(nb=(2, 2, 2), n=(8, 8, 8), lo=(-0.5, -0.5, -0.5), hi=(2.5, 2.5, 2.5), z=(0.3, -0.2, 0.1)):
    """The blast wave moving with a uniform velocity (three-velocity times
    W, z) on a sub-box whose low faces cut through the overdense core: mass
    crosses every outer face, in through some and out through others, with
    a net flux of the core's density.  For the outflow diagnostic."""
    su, (st, bx, by, bz, aux) = blast(nb=nb, n=n, lo=lo, hi=hi)
    rho, press, eps, s = aux[:, abi.RHO], aux[:, abi.PRESS], aux[:, abi.EPS], aux[:, abi.ENTROPY]
    Bc = np.moveaxis(aux[:, abi.BX:abi.BZ + 1], 1, 0)
    zz = np.empty((3,) + rho.shape)
    for a in range(3):
        zz[a] = z[a]
    st[:, 0:7] = np.moveaxis(flat_prims_to_cons(rho, press, eps, zz, Bc, s), 0, 1)
    aux[:, abi.ZVECX:abi.ZVECZ + 1] = np.moveaxis(zz, 0, 1)
    return su, (st, bx, by, bz, aux)


def balsara1(nb=(64, 1, 1), n=(16, 16, 16), ngz=4):
    """Balsara-1 shock tube: Gamma=2; left rho=1,p=1,B=(0.5,1,0); right
    rho=0.125,p=0.1,B=(0.5,-1,0); x in [-0.5,0.5], y,z in [-1/128,1/128]
    (1024x16x16 cells at the default size); periodic y,z, outflow x."""
    su = BrickSetup(nb, n, (-0.5, -1 / 128, -1 / 128), (0.5, 1 / 128, 1 / 128), ngz,
                    (False, True, True))
    X = su.cell_centres()
    left = X[:, 0] < 0.0
    rho = np.where(left, 1.0, 0.125)
    press = np.where(left, 1.0, 0.1)
    NX, NY, NZ = su.N

    def faces(sx, sy, sz):
        Bx = np.full(sx, 0.5)
        # By lives on y-faces at cell-centred x
        xl = X[:, 0][:, :, :1, :]  # (nq, NZ, 1, NX)
        By = np.broadcast_to(np.where(xl < 0.0, 1.0, -1.0), sy).copy()
        return Bx, By, np.zeros(sz)

    return su, _fill(su, 2.0, rho, press, None, faces)


def c2p_states(n, seed=SEED, kappa=100.0, gamma=2.0, gamma_th=1.8):
    """c2p micro-benchmark states on the flat metric with the hybrid EOS:
    rho log-U[1e-12,1e-3], eps_th log-U[1e-6,10] above the cold curve,
    W U[1,50), sigma=b^2/rho log-U[1e-4,1e3], isotropic directions for the
    velocity and the field.  Returns (cons (10,n), prims (13,n))."""
    rng = np.random.default_rng(seed)
    rho = 10 ** rng.uniform(-12, -3, n)
    eth = 10 ** rng.uniform(-6, 1, n)
    W = rng.uniform(1.0, 50.0, n)
    sig = 10 ** rng.uniform(-4, 3, n)

    def unit():
        v = rng.standard_normal((3, n))
        return v / np.linalg.norm(v, axis=0)[None]

    z = np.sqrt(W * W - 1.0)[None] * unit()
    ec = kappa * rho ** (gamma - 1.0) / (gamma - 1.0)
    eps = ec + eth
    gm = gamma_th - 1.0
    press = kappa * rho ** gamma + gm * rho * eth
    T = eth * gm
    s = np.log(np.maximum(eth, 1e-13) * rho ** (-gm)) / gm
    Bd = unit()
    Bzd = np.sum(Bd * z, axis=0)
    b2_unit = (1.0 + Bzd * Bzd) / (W * W)
    B = np.sqrt(sig * rho / b2_unit)[None] * Bd
    cons7 = flat_prims_to_cons(rho, press, eps, z, B, s)
    cons = np.zeros((10, n))
    cons[0:7] = cons7
    cons[7:10] = B
    prims = np.zeros((13, n))
    prims[abi.P_RHO], prims[abi.P_PRESS], prims[abi.P_EPS] = rho, press, eps
    prims[abi.P_ZX:abi.P_ZZ + 1] = z
    prims[abi.P_TEMP], prims[abi.P_ENT] = T, s
    prims[abi.P_BX:abi.P_BZ + 1] = B
    return cons, prims


def fmr_blast(hier, bx0=0.1, r0=0.8, gamma=4.0 / 3.0, flow=0.0):
    """The blast wave (Gamma=4/3, rho=1e-4 / p=5e-4 outside, rho=1e-2 / p=1
    inside r<r0, uniform Bx) on the leaves of a static FMR hierarchy
    (grace_b200.fmr.Hierarchy), with a smooth 1e-3 relative pressure ripple
    instead of cell noise so that every level samples the same field; flow:
    amplitude of a smooth shearing velocity (W v = flow x (sin 0.7y,
    sin 0.9z, sin 1.1x)) that makes the EMFs nonzero from the first
    substep.  Returns (state, bx, by, bz, aux) in the library layout."""
    NN = hier.n + 2 * hier.ngz
    nq = hier.nq
    state = np.zeros((nq, abi.N_EVOL_VARS, NN, NN, NN))
    bx = np.full((nq, NN, NN, NN + 1), bx0)
    by = np.zeros((nq, NN, NN + 1, NN))
    bz = np.zeros((nq, NN + 1, NN, NN))
    aux = np.zeros((nq, abi.N_AUX_VARS, NN, NN, NN))
    state[:, abi.GXX] = state[:, abi.GYY] = state[:, abi.GZZ] = 1.0
    state[:, abi.ALP] = 1.0
    X = hier.cell_centres()
    r = np.sqrt(np.sum(X * X, axis=1))
    inside = r < r0
    rho = np.where(inside, 1e-2, 1e-4)
    press = np.where(inside, 1.0, 5e-4) * (1.0 + 1e-3 * np.sin(1.3 * X[:, 0]) * np.cos(0.7 * X[:, 1] + 0.4 * X[:, 2]))
    eps = press / ((gamma - 1.0) * rho)
    s = np.log(eps) / (gamma - 1.0) - np.log(rho)
    z = np.zeros((3,) + rho.shape)
    if flow:
        z[0] = flow * np.sin(0.7 * X[:, 1])
        z[1] = flow * np.sin(0.9 * X[:, 2])
        z[2] = flow * np.sin(1.1 * X[:, 0])
    Bc = np.zeros((3,) + rho.shape)
    Bc[0] = bx0
    cons = flat_prims_to_cons(rho, press, eps, z, Bc, s)
    aux[:, abi.ZVECX:abi.ZVECZ + 1] = np.moveaxis(z, 0, 1)
    state[:, 0:7] = np.moveaxis(cons, 0, 1)
    aux[:, abi.RHO], aux[:, abi.PRESS], aux[:, abi.EPS] = rho, press, eps
    aux[:, abi.TEMP] = eps * (gamma - 1.0)
    aux[:, abi.ENTROPY] = s
    aux[:, abi.BX] = bx0
    return state, bx, by, bz, aux


# ---------------------------------------------------------------------------
# Magnetised TOV star in the Cowling approximation
def tov_solution(kappa=100.0, gamma=2.0, rho_c=1.28e-3, dr=2e-3, p_floor_rel=1e-12):
    """Static spherical star of the polytrope P = kappa rho^gamma (TOV
    equations in the areal radius r, fourth-order Runge-Kutta, mass m,
    pressure P, log lapse nu, isotropic radius), matched at the surface to
    Schwarzschild's exterior in isotropic coordinates.  Returns a dict of
    the tables (areal r, isotropic radius riso, m, P, nu) and the star's
    mass M, areal radius R and isotropic radius Riso."""
    gm1 = gamma - 1.0

    def energy(P):
        P = max(P, 0.0)
        rho = (P / kappa) ** (1.0 / gamma)
        return rho + P / gm1

    def rhs(r, y):
        m, P, nu, lri = y
        e = energy(P)
        den = r * (r - 2.0 * m)
        dnu = (m + 4.0 * np.pi * r ** 3 * P) / den
        return np.array([4.0 * np.pi * r * r * e, -(e + P) * dnu, dnu, 1.0 / (r * np.sqrt(1.0 - 2.0 * m / r))])

    Pc = kappa * rho_c ** gamma
    ec = energy(Pc)
    r = dr
    # series start: m = 4/3 pi e_c r^3, P ~ P_c, nu ~ 0, riso ~ r
    y = np.array([4.0 / 3.0 * np.pi * ec * r ** 3, Pc, 0.0, np.log(r)])
    rs, ys = [0.0, r], [np.array([0.0, Pc, 0.0, -np.inf]), y.copy()]
    pf = p_floor_rel * Pc
    while True:
        k1 = rhs(r, y)
        k2 = rhs(r + 0.5 * dr, y + 0.5 * dr * k1)
        k3 = rhs(r + 0.5 * dr, y + 0.5 * dr * k2)
        k4 = rhs(r + dr, y + dr * k3)
        yn = y + dr / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
        if yn[1] <= pf:
            lam = (pf - y[1]) / (yn[1] - y[1])
            R = r + lam * dr
            ysurf = y + lam * (yn - y)
            rs.append(R)
            ysurf[1] = 0.0
            ys.append(ysurf)
            break
        r += dr
        y = yn
        rs.append(r)
        ys.append(y.copy())
    rs = np.asarray(rs)
    Y = np.stack(ys)
    M = Y[-1, 0]
    # exterior matching: nu(R) = 1/2 ln(1 - 2M/R), riso(R) from Schwarzschild
    nu = Y[:, 2] + (0.5 * np.log(1.0 - 2.0 * M / R) - Y[-1, 2])
    Riso = 0.5 * (R - M + np.sqrt(R * (R - 2.0 * M)))
    riso = np.exp(Y[:, 3] - Y[-1, 3]) * Riso
    riso[0] = 0.0
    return {"r": rs, "riso": riso, "m": Y[:, 0], "P": np.maximum(Y[:, 1], 0.0), "nu": nu, "M": M, "R": R,
            "Riso": Riso, "kappa": kappa, "gamma": gamma}


def tov_metric(sol, ri):
    """Conformal factor psi^4 and lapse at isotropic radii ri (arrays)."""
    M, Riso = sol["M"], sol["Riso"]
    inside = ri < Riso
    rr = np.interp(ri, sol["riso"], sol["r"])
    # r / riso -> its central limit at the centre
    c0 = sol["r"][1] / sol["riso"][1]
    ratio = np.where(ri > 0, rr / np.maximum(ri, 1e-300), c0)
    psi4_in = ratio ** 2
    alp_in = np.exp(np.interp(ri, sol["riso"], sol["nu"]))
    h = M / (2.0 * np.maximum(ri, 1e-300))
    psi4_out = (1.0 + h) ** 4
    alp_out = (1.0 - h) / (1.0 + h)
    return np.where(inside, psi4_in, psi4_out), np.where(inside, alp_in, alp_out)


def tov_pressure(sol, ri):
    return np.where(ri < sol["Riso"], np.interp(ri, sol["riso"], sol["P"]), 0.0)


def magnetised_tov(hier, kappa=100.0, gamma=2.0, rho_c=1.28e-3, gamma_th=1.8, rho_atm=1e-10,
                   eps_th=1e-4, bmax=1e-4, p_cut=0.04, a_n=2.0, noise=1e-3, seed=SEED):
    """The magnetised polytropic neutron star in Cowling (the TOV solution
    above: K=100, Gamma=2, rho_c=1.28e-3, ~1.4 solar masses) on the leaves
    of a static FMR hierarchy: conformally flat metric psi^4 delta_ij, the
    lapse, zero shift and extrinsic curvature (static); rest-mass density
    with seeded relative noise (counter hash of each cell's level and
    integer position), cold pressure and energy of the polytrope plus a
    small uniform specific thermal energy eps_th (hybrid EOS with Gamma_th;
    1e-4 keeps the entropy, a logarithm of eps - eps_cold, well conditioned
    next to eps_cold ~ 0.1 at the centre); atmosphere rho_atm outside; an
    interior poloidal field from A = A_b max(P - p_cut P_c, 0)^a_n (-y, x, 0)
    (the form of GRACE's Avec_poloidal_id_t), taken as the discrete curl on
    each block's edges (div B = 0 to round-off) and scaled so that
    max |B| = bmax.  Returns ((state, bx, by, bz, aux), tov solution)."""
    sol = tov_solution(kappa, gamma, rho_c)
    NN = hier.n + 2 * hier.ngz
    nq = hier.nq
    g = hier.ngz
    state = np.zeros((nq, abi.N_EVOL_VARS, NN, NN, NN))
    aux = np.zeros((nq, abi.N_AUX_VARS, NN, NN, NN))
    X = hier.cell_centres()
    ri = np.sqrt(np.sum(X * X, axis=1))
    psi4, alp = tov_metric(sol, ri)
    state[:, abi.GXX] = state[:, abi.GYY] = state[:, abi.GZZ] = psi4
    state[:, abi.ALP] = alp
    Pc = kappa * rho_c ** gamma
    P = tov_pressure(sol, ri)
    rho = np.maximum((P / kappa) ** (1.0 / gamma), rho_atm)
    # seeded noise per cell, independent of the block order
    key = np.zeros((nq, 3, NN, NN, NN), dtype=np.int64)
    r = np.arange(NN)
    for q, (l, b) in enumerate(hier.leaves):
        key[q, 0] = b[0] * hier.n + r[None, None, :] + (l << 20)
        key[q, 1] = b[1] * hier.n + r[None, :, None]
        key[q, 2] = b[2] * hier.n + r[:, None, None]
    u = _counter_uniform(np.moveaxis(key, 1, -1).reshape(-1, 3) + 64, seed, np.array([1 << 22, 1 << 22])).reshape(rho.shape)
    rho = np.where(P > 0, rho * (1.0 + noise * u), rho)
    Pcold = kappa * rho ** gamma
    ecold = kappa * rho ** (gamma - 1.0) / (gamma - 1.0)
    press = Pcold + (gamma_th - 1.0) * rho * eps_th
    eps = ecold + eps_th
    # face B (densitized: sqrt(gamma) B^i) as the discrete curl of the edge
    # potential, block by block
    bx = np.zeros((nq, NN, NN, NN + 1))
    by = np.zeros((nq, NN, NN + 1, NN))
    bz = np.zeros((nq, NN + 1, NN, NN))
    Afun = lambda Pv: np.maximum(Pv - p_cut * Pc, 0.0) ** a_n
    f = np.arange(NN + 1)
    c = np.arange(NN)
    for q, (l, b) in enumerate(hier.leaves):
        d = hier.dx(l)
        o = hier.lo + np.asarray(b) * hier.n * d
        xf, yf, zf = o[0] + (f - g) * d[0], o[1] + (f - g) * d[1], o[2] + (f - g) * d[2]
        xc, yc, zc = o[0] + (c - g + 0.5) * d[0], o[1] + (c - g + 0.5) * d[1], o[2] + (c - g + 0.5) * d[2]
        # A_x on x-edges (xc, yf, zf), A_y on y-edges (xf, yc, zf); array order (z, y, x)
        Zx, Yx, Xx = np.meshgrid(zf, yf, xc, indexing="ij")
        Ax = -Yx * Afun(tov_pressure(sol, np.sqrt(Xx ** 2 + Yx ** 2 + Zx ** 2)))
        Zy, Yy, Xy = np.meshgrid(zf, yc, xf, indexing="ij")
        Ay = Xy * Afun(tov_pressure(sol, np.sqrt(Xy ** 2 + Yy ** 2 + Zy ** 2)))
        # Bx(x face, yc, zc) = -dAy/dz ; By(xc, y face, zc) = dAx/dz ;
        # Bz(xc, yc, z face) = dAy/dx - dAx/dy
        bx[q] = -(Ay[1:, :, :] - Ay[:-1, :, :]) / d[2]
        by[q] = (Ax[1:, :, :] - Ax[:-1, :, :]) / d[2]
        bz[q] = (Ay[:, :, 1:] - Ay[:, :, :-1]) / d[0] - (Ax[:, 1:, :] - Ax[:, :-1, :]) / d[1]
    sq = psi4 ** 1.5  # sqrt(gamma) = psi^6
    Bc = np.stack([0.5 * (bx[..., :-1] + bx[..., 1:]), 0.5 * (by[:, :, :-1, :] + by[:, :, 1:, :]),
                   0.5 * (bz[:, :-1] + bz[:, 1:])]) / sq[None]
    bmag = np.sqrt(psi4 * np.sum(Bc * Bc, axis=0))
    scale = bmax / max(float(np.max(bmag)), 1e-300)
    bx *= scale
    by *= scale
    bz *= scale
    Bc *= scale
    # conserved variables of a static fluid (v = 0, W = 1)
    b2 = psi4 * np.sum(Bc * Bc, axis=0)
    gmth = gamma_th - 1.0
    s = np.log(eps_th * rho ** (-gmth)) / gmth
    D = sq * rho
    state[:, abi.DENS] = D
    state[:, abi.TAU] = sq * (rho * eps + 0.5 * b2)
    state[:, abi.ENTROPYSTAR] = D * s
    aux[:, abi.RHO], aux[:, abi.PRESS], aux[:, abi.EPS] = rho, press, eps
    aux[:, abi.TEMP] = eps_th * gmth
    aux[:, abi.ENTROPY] = s
    aux[:, abi.BX:abi.BZ + 1] = np.moveaxis(Bc, 0, 1)
    return (state, bx, by, bz, aux), sol


def tov_hierarchy(n=16):
    """The FMR hierarchy of the magnetised TOV star: the cube +-48 (M_sun
    units) in 4^3 base blocks of n^3 cells, refined where a block comes
    within 26, 14, 8, 3.5 of the centre (levels 0..3), five levels, outflow
    boundaries: 32 / 224 / 224 / 224 / 256 blocks on levels 0..4 (uneven
    per-level counts), finest spacing 0.09375 at n = 16."""
    from . import fmr
    radii = (26.0, 14.0, 8.0, 3.5)
    half, nb0 = 48.0, 4

    def refine(l, b):
        if l >= len(radii):
            return False
        size = 2 * half / nb0 / 2 ** l
        lo = -half + np.asarray(b) * size
        hi = lo + size
        d = np.sqrt(np.sum(np.maximum(0.0, np.maximum(lo, -hi)) ** 2))
        return d < radii[l]

    return fmr.Hierarchy((nb0,) * 3, n, (-half,) * 3, (half,) * 3, refine, len(radii), periodic=(False,) * 3)


# ---------------------------------------------------------------------------
# General 3+1 metric helpers and the Fishbone-Moncrief torus in Kerr-Schild
def sym3(g6):
    """(6, ...) symmetric components xx, xy, xz, yy, yz, zz -> (3, 3, ...)."""
    xx, xy, xz, yy, yz, zz = g6
    return np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])


def curved_prims_to_cons(g6, beta, alp, rho, press, eps, z, B, s):
    """Densitized conserved variables (7, ...) DENS, S_i, TAU, YESTAR (0),
    ENTROPYSTAR from primitives on a 3+1 metric (g6 the spatial metric's 6
    components, beta^i, alpha): z^i = W v^i, B^i (not densitized).  The
    usual ideal-MHD expressions: b^0 = W B.v / alpha, b^2 = (B^2 +
    alpha^2 (b^0)^2) / W^2, D = rho W, S_i = (rho h + b^2) W^2 v_i -
    alpha b^0 b_i, tau = (rho h + b^2) W^2 - (P + b^2/2) - alpha^2 (b^0)^2 - D,
    all times sqrt(gamma)."""
    G = sym3(g6)
    det = (G[0, 0] * (G[1, 1] * G[2, 2] - G[1, 2] ** 2) - G[0, 1] * (G[0, 1] * G[2, 2] - G[0, 2] * G[1, 2]) +
           G[0, 2] * (G[0, 1] * G[1, 2] - G[0, 2] * G[1, 1]))
    sq = np.sqrt(det)
    zl = np.einsum("ij...,j...->i...", G, z)
    W = np.sqrt(1.0 + np.sum(z * zl, axis=0))
    v = z / W
    vl = zl / W
    Bl = np.einsum("ij...,j...->i...", G, B)
    Bv = np.sum(B * vl, axis=0)
    B2 = np.sum(B * Bl, axis=0)
    b0 = W * Bv / alp
    b2 = (B2 + alp * alp * b0 * b0) / (W * W)
    # b_i = gamma_ij b^j + beta_i b^0 with b^j = (B^j + alpha b^0 W (v^j - beta^j/alpha)) / W
    bu = (B + alp * b0 * W * (v - beta / alp)) / W
    betal = np.einsum("ij...,j...->i...", G, beta)
    bl = np.einsum("ij...,j...->i...", G, bu) + betal * b0
    rhoh = rho * (1.0 + eps) + press
    D = rho * W
    out = np.zeros((7,) + rho.shape)
    out[0] = sq * D
    out[1:4] = sq * ((rhoh + b2) * W * W * vl - alp * b0 * bl)
    out[4] = sq * ((rhoh + b2) * W * W - (press + 0.5 * b2) - alp * alp * b0 * b0 - D)
    out[6] = sq * D * s
    return out, sq, b2


def kerr_schild(x, y, z, a, r_reg=0.5):
    """Cartesian Kerr-Schild (M = 1): spatial metric g6, shift beta^i, lapse,
    and the Boyer-Lindquist radius r (at least r_reg)."""
    R2 = x * x + y * y + z * z
    r2 = 0.5 * (R2 - a * a + np.sqrt((R2 - a * a) ** 2 + 4.0 * a * a * z * z))
    # regularised well inside the horizon (r_+ = 1 + sqrt(1 - a^2)): the
    # excised region needs finite values, not the ring singularity
    r2 = np.maximum(r2, r_reg * r_reg)
    r = np.sqrt(r2)
    H = r2 * r / (r2 * r2 + a * a * z * z)
    l = np.stack([(r * x + a * y) / (r2 + a * a), (r * y - a * x) / (r2 + a * a), z / r])
    g6 = np.stack([1.0 + 2 * H * l[0] * l[0], 2 * H * l[0] * l[1], 2 * H * l[0] * l[2],
                   1.0 + 2 * H * l[1] * l[1], 2 * H * l[1] * l[2], 1.0 + 2 * H * l[2] * l[2]])
    beta = 2 * H * l / (1.0 + 2 * H)
    alp = 1.0 / np.sqrt(1.0 + 2 * H)
    return g6, beta, alp, r


def kerr_schild_curvature(x, y, z, a, h=1e-5):
    """Extrinsic curvature K_ij of the stationary Kerr-Schild slice,
    K_ij = (D_i beta_j + D_j beta_i) / (2 alpha), with the derivatives of
    the metric and of beta_j = gamma_jk beta^k by central differences of the
    analytic fields (step h).  Returns the 6 components (xx, xy, xz, yy,
    yz, zz)."""
    P = (x, y, z)

    def at(d, sgn):
        q = [x, y, z]
        q = [q[k] + (sgn * h if k == d else 0.0) for k in range(3)]
        g6, beta, alp, _ = kerr_schild(q[0], q[1], q[2], a)
        G = sym3(g6)
        return G, np.einsum("ij...,j...->i...", G, beta)

    g6, beta, alp, _ = kerr_schild(*P, a)
    G = sym3(g6)
    Gi = np.linalg.inv(np.moveaxis(G, (0, 1), (-2, -1)))
    Gi = np.moveaxis(Gi, (-2, -1), (0, 1))
    dG, dbl = [], []
    for d in range(3):
        Gp, blp = at(d, +1)
        Gm, blm = at(d, -1)
        dG.append((Gp - Gm) / (2 * h))
        dbl.append((blp - blm) / (2 * h))
    dG = np.stack(dG)      # [d][i][j]: d_d g_ij
    dbl = np.stack(dbl)    # [d][j]: d_d beta_j
    betal = np.einsum("ij...,j...->i...", G, beta)
    # Gamma_kij (lowered first index) = (d_i g_kj + d_j g_ki - d_k g_ij) / 2
    Gam_l = 0.5 * (np.einsum("ikj...->kij...", dG) + np.einsum("jki...->kij...", dG) - dG)
    Gam = np.einsum("lk...,kij...->lij...", Gi, Gam_l)
    Dbl = dbl - np.einsum("kij...,k...->ij...", Gam, betal)  # D_i beta_j
    K = (Dbl + np.einsum("ij...->ji...", Dbl)) / (2.0 * alp)
    return np.stack([K[0, 0], K[0, 1], K[0, 2], K[1, 1], K[1, 2], K[2, 2]])


def fm_torus(hier, a=0.9375, r_in=6.0, r_pmax=12.0, gamma=4.0 / 3.0, kappa=1e-3, rho_atm=1e-8,
             beta_p=100.0, a_cut=0.2, noise=2e-2, rho_noise=1e-3, seed=SEED):
    """Fishbone-Moncrief torus in the fixed Kerr-Schild metric on the leaves
    of a static FMR hierarchy, written from the configuration text (the
    reference's own torus initial data is not part of its sources): the
    torus of constant specific angular momentum set by r_pmax, inner edge
    r_in, polytrope P = kappa rho^gamma with rho normalised to 1 at its
    maximum, the orbital velocity transformed from Boyer-Lindquist to
    Cartesian Kerr-Schild; atmosphere rho_atm (at rest in the Kerr-Schild
    frame, pressure of the same polytrope); a poloidal field from
    A = A_b max(rho/rho_max - a_cut, 0) (-y, x, 0) as the discrete curl on
    each block's edges, scaled so that max P / max(b^2/2) = beta_p; seeded
    relative pressure noise, and seeded relative density noise in
    (-rho_noise, 0] everywhere (atmosphere included: without it the data are
    mirror symmetric about z = 0, the mass flux through the equatorial faces
    is a rounding residue and the sign that upwinds the Gardiner-Stone EMF
    there is arbitrary).  Returns (state, bx, by, bz, aux)."""
    def lnh_bl(r, th, l):
        sth, cth = np.sin(th), np.cos(th)
        DD = r * r - 2 * r + a * a
        AA = (r * r + a * a) ** 2 - DD * a * a * sth * sth
        SS = r * r + a * a * cth * cth
        t = np.sqrt(1.0 + 4.0 * l * l * SS * SS * DD / (AA * AA * sth * sth))
        return 0.5 * np.log((1.0 + t) / (SS * DD / AA)) - 0.5 * t - 2.0 * a * r * l / AA

    # Fishbone-Moncrief angular momentum of the pressure maximum
    rp = r_pmax
    sr = np.sqrt(rp)
    l = (((a * a - 2 * a * sr + rp * rp) * ((-2 * a * rp * (a * a - 2 * a * sr + rp * rp)) /
         np.sqrt(2 * a * sr + (rp - 3) * rp) + ((a + (rp - 2) * sr) * (rp ** 3 + a * a * (2 + rp))) /
         np.sqrt(1 + 2 * a / rp ** 1.5 - 3 / rp))) / (rp ** 3 * np.sqrt(2 * a * sr + (rp - 3) * rp) *
                                                      (a * a + (rp - 2) * rp)))
    lnh_in = lnh_bl(r_in, 0.5 * np.pi, l)
    # rho_max at the pressure maximum (equator, r_pmax)
    hmax = np.exp(lnh_bl(r_pmax, 0.5 * np.pi, l) - lnh_in)
    rho_max = ((hmax - 1) * (gamma - 1) / (kappa * gamma)) ** (1 / (gamma - 1))

    def fluid(x, y, z):
        g6, beta, alp, r = kerr_schild(x, y, z, a)
        th = np.arccos(np.clip(z / np.maximum(r, 1e-300), -1, 1))
        sth = np.maximum(np.sin(th), 1e-12)
        with np.errstate(invalid="ignore", divide="ignore"):
            lnh = np.where(r >= r_in, lnh_bl(np.maximum(r, r_in), th, l) - lnh_in, -1.0)
        inside = (r >= r_in) & (lnh > 0)
        h = np.exp(np.where(inside, lnh, 0.0))
        rho = np.where(inside, ((h - 1) * (gamma - 1) / (kappa * gamma)) ** (1 / (gamma - 1)) / rho_max, rho_atm)
        # u^phi in Boyer-Lindquist (= Kerr-Schild's when u^r = 0)
        rr = np.maximum(r, r_in)
        DD = rr * rr - 2 * rr + a * a
        AA = (rr * rr + a * a) ** 2 - DD * a * a * sth * sth
        SS = rr * rr + a * a * np.cos(th) ** 2
        em2chi = SS * SS * DD / (AA * AA * sth * sth)
        up1 = np.sqrt((-1 + np.sqrt(1 + 4 * l * l * em2chi)) / 2)
        uphi = 2 * a * rr * np.sqrt(1 + up1 * up1) / np.sqrt(AA * SS * DD) + np.sqrt(SS / AA) * up1 / sth
        uphi = np.where(inside, uphi, 0.0)
        # Cartesian KS: u^x = -y u^phi, u^y = x u^phi; u^t from u.u = -1
        ui = np.stack([-y * uphi, x * uphi, np.zeros_like(x)])
        G = sym3(g6)
        uil = np.einsum("ij...,j...->i...", G, ui)
        # g_tt = -alp^2 + beta.beta, g_ti = beta_i: solve for u^t > 0
        betal = np.einsum("ij...,j...->i...", G, beta)
        gtt = -alp * alp + np.sum(beta * betal, axis=0)
        A_ = gtt
        B_ = 2 * np.sum(betal * ui, axis=0)
        C_ = np.sum(ui * uil, axis=0) + 1.0
        with np.errstate(invalid="ignore"):
            ut = (-B_ - np.sqrt(B_ * B_ - 4 * A_ * C_)) / (2 * A_)
        # z^i = u^i + u^t beta^i in the torus; the atmosphere at rest for the
        # normal observers (z = 0, regular in the ergoregion too)
        zv = np.where(inside[None], ui + ut * beta, 0.0)
        rho = np.maximum(rho, rho_atm)
        return g6, beta, alp, r, rho, zv

    NN = hier.n + 2 * hier.ngz
    nq = hier.nq
    g = hier.ngz
    X = hier.cell_centres()
    x, y, zc = X[:, 0], X[:, 1], X[:, 2]
    g6, beta, alp, r, rho, zv = fluid(x, y, zc)
    Kc = kerr_schild_curvature(x, y, zc, a)
    key = np.zeros((nq, 3, NN, NN, NN), dtype=np.int64)
    rr_ = np.arange(NN)
    for q, (lv, b) in enumerate(hier.leaves):
        key[q, 0] = b[0] * hier.n + rr_[None, None, :] + (lv << 20)
        key[q, 1] = b[1] * hier.n + rr_[:, None] * 0 + rr_[None, :, None]
        key[q, 2] = b[2] * hier.n + rr_[:, None, None]
    gid = np.moveaxis(key, 1, -1).reshape(-1, 3) + 64
    u = _counter_uniform(gid, seed, np.array([1 << 22, 1 << 22])).reshape(rho.shape)
    u_rho = _counter_uniform(gid, seed + 1, np.array([1 << 22, 1 << 22])).reshape(rho.shape)
    rho = rho * (1.0 + 0.5 * rho_noise * (u_rho - 1.0))
    press = kappa * (rho * rho_max) ** gamma / rho_max  # normalised units: P / rho_max
    press = press * (1.0 + noise * u)
    eps = press / ((gamma - 1.0) * rho)
    s = np.log(eps) / (gamma - 1.0) - np.log(rho)
    # field: discrete curl of A = f(rho(x)) (-y, x, 0) on each block's edges
    bx = np.zeros((nq, NN, NN, NN + 1))
    by = np.zeros((nq, NN, NN + 1, NN))
    bz = np.zeros((nq, NN + 1, NN, NN))
    def rho_only(xx, yy, zz):
        # the torus density alone (the vector potential's profile)
        R2 = xx * xx + yy * yy + zz * zz
        r = np.sqrt(0.5 * (R2 - a * a + np.sqrt((R2 - a * a) ** 2 + 4.0 * a * a * zz * zz)))
        th = np.arccos(np.clip(zz / np.maximum(r, 1e-300), -1, 1))
        with np.errstate(invalid="ignore", divide="ignore"):
            lnh = np.where(r >= r_in, lnh_bl(np.maximum(r, r_in), th, l) - lnh_in, -1.0)
        h = np.exp(np.where((r >= r_in) & (lnh > 0), lnh, 0.0))
        return ((h - 1) * (gamma - 1) / (kappa * gamma)) ** (1 / (gamma - 1)) / rho_max

    fA = lambda xx, yy, zz: np.maximum(rho_only(xx, yy, zz) - a_cut, 0.0)
    f_ = np.arange(NN + 1)
    c_ = np.arange(NN)
    for q, (lv, b) in enumerate(hier.leaves):
        d = hier.dx(lv)
        o = hier.lo + np.asarray(b) * hier.n * d
        xf, yf, zf = o[0] + (f_ - g) * d[0], o[1] + (f_ - g) * d[1], o[2] + (f_ - g) * d[2]
        xc, yc, zcc = o[0] + (c_ - g + 0.5) * d[0], o[1] + (c_ - g + 0.5) * d[1], o[2] + (c_ - g + 0.5) * d[2]
        Zx, Yx, Xx = np.meshgrid(zf, yf, xc, indexing="ij")
        Ax = -Yx * fA(Xx, Yx, Zx)
        Zy, Yy, Xy = np.meshgrid(zf, yc, xf, indexing="ij")
        Ay = Xy * fA(Xy, Yy, Zy)
        bx[q] = -(Ay[1:, :, :] - Ay[:-1, :, :]) / d[2]
        by[q] = (Ax[1:, :, :] - Ax[:-1, :, :]) / d[2]
        bz[q] = (Ay[:, :, 1:] - Ay[:, :, :-1]) / d[0] - (Ax[:, 1:, :] - Ax[:, :-1, :]) / d[1]
    G = sym3(g6)
    det = (G[0, 0] * (G[1, 1] * G[2, 2] - G[1, 2] ** 2) - G[0, 1] * (G[0, 1] * G[2, 2] - G[0, 2] * G[1, 2]) +
           G[0, 2] * (G[0, 1] * G[1, 2] - G[0, 2] * G[1, 1]))
    sq = np.sqrt(det)
    Bc = np.stack([0.5 * (bx[..., :-1] + bx[..., 1:]), 0.5 * (by[:, :, :-1, :] + by[:, :, 1:, :]),
                   0.5 * (bz[:, :-1] + bz[:, 1:])]) / sq[None]
    _, _, b2 = curved_prims_to_cons(g6, beta, alp, rho, press, eps, zv, Bc, s)
    scale = np.sqrt(float(np.max(press)) / (beta_p * 0.5 * max(float(np.max(b2)), 1e-300)))
    for arr in (bx, by, bz, Bc):
        arr *= scale
    cons, sq, b2 = curved_prims_to_cons(g6, beta, alp, rho, press, eps, zv, Bc, s)
    state = np.zeros((nq, abi.N_EVOL_VARS, NN, NN, NN))
    aux = np.zeros((nq, abi.N_AUX_VARS, NN, NN, NN))
    state[:, 0:7] = np.moveaxis(cons, 0, 1)
    for k in range(6):
        state[:, abi.GXX + k] = g6[k]
        state[:, abi.KXX + k] = Kc[k]
    state[:, abi.ALP] = alp
    for k in range(3):
        state[:, abi.BETAX + k] = beta[k]
    aux[:, abi.RHO], aux[:, abi.PRESS], aux[:, abi.EPS] = rho, press, eps
    aux[:, abi.TEMP] = eps * (gamma - 1.0)
    aux[:, abi.ENTROPY] = s
    aux[:, abi.ZVECX:abi.ZVECZ + 1] = np.moveaxis(zv, 0, 1)
    aux[:, abi.BX:abi.BZ + 1] = np.moveaxis(Bc, 0, 1)
    return state, bx, by, bz, aux


def torus_hierarchy(n=16):
    """The FMR hierarchy of the torus: the cube +-40 (units of M) in 4^3
    base blocks of n^3 cells, four levels, refined where a block comes
    within 10, 5, 2.5 of the torus' pressure-maximum ring (cylindrical radius
    12 in the equatorial plane) or within 3, 2, 1.5 of the black hole
    (levels 0..2), then 2:1 balanced; outflow boundaries; uneven per-level
    counts."""
    from . import fmr
    half, nb0 = 40.0, 4
    ring, hole = (10.0, 5.0, 2.5), (3.0, 2.0, 1.5)

    def refine(l, b):
        if l >= len(ring):
            return False
        size = 2 * half / nb0 / 2 ** l
        lo = -half + np.asarray(b) * size
        hi = lo + size
        # distance from the box to the origin and to the ring R = 12, z = 0
        d0 = np.sqrt(np.sum(np.maximum(0.0, np.maximum(lo, -hi)) ** 2))
        # sample the box for the ring distance (boxes are few)
        t = np.linspace(0, 1, 9)
        X, Y, Z = np.meshgrid(lo[0] + t * size, lo[1] + t * size, lo[2] + t * size, indexing="ij")
        dr = np.sqrt((np.sqrt(X ** 2 + Y ** 2) - 12.0) ** 2 + Z ** 2).min()
        return dr < ring[l] or d0 < hole[l]

    return fmr.Hierarchy((nb0,) * 3, n, (-half,) * 3, (half,) * 3, refine, len(ring), periodic=(False,) * 3)
