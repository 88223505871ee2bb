"""Parameter construction mirroring GRACE's YAML schema defaults.

Defaults come from parameters/grmhd.yaml and parameters/eos.yaml of the
reference; the piecewise-polytrope tables are derived as in
src/physics/eos/eos_storage.cpp:53-100 (setup_cold_polytrope).  The C
library exports the same helpers (grb_params_defaults,
grb_eos_setup_pwpoly); tests check that both produce identical bytes.
"""
import math

from . import abi


def defaults(eos_kind=abi.EOS_IDEAL_GAS):
    p = abi.Params()
    e = p.eos
    e.kind = eos_kind
    e.n_pieces = 1
    e.gamma = 5.0 / 3.0
    e.gamma_th = 1.8
    e.eps_max = 1.0e5          # eos.eps_maximum
    e.entropy_min = 1.0e-13    # eos.entropy_minimum
    e.temp_atm = 0.0           # grmhd.atmosphere.temp_fl
    p.rho_fl = 1.0e-14
    p.ye_fl = 0.0              # eos ye_atmosphere() of the ideal / hybrid EOS
    p.temp_fl = 0.0
    p.atmo_tol = 1.0e-3
    p.excise_by_radius = 0     # excision_criterion: lapse
    p.r_ex = 1.0
    p.alp_ex = 0.05
    p.rho_ex = p.rho_fl
    p.temp_ex = 0.0
    p.ye_ex = 0.0
    p.c2p_tol = 1.0e-10
    p.max_w = 50.0
    p.max_sigma = 100.0
    p.beta_fallback = 1.0e-2
    p.alp_bh_thresh = 0.2
    p.use_ent_backup = 1
    p.rusanov_use_c_limit = 0.0
    p.fofc_enable = 1
    p.dmp_enable = 1
    p.dmp_M = 1.2
    p.recon = abi.RECON_WENOZ
    p.riemann = abi.RIEMANN_HLL
    p.emf = abi.EMF_GS
    p.ranges = abi.RANGES_FULL  # aux / linop write every cell (the drop-in contract)
    return p


def setup_pwpoly(e, kappa_0, gammas, rhos):
    """Fill e.pw_* from kappa_0, gammas[n], rhos[n-1] (eos_storage.cpp:53-100)."""
    n = len(gammas)
    if n < 1 or n > abi.MAX_PIECES or len(rhos) != n - 1:
        raise ValueError("piecewise polytrope: need n gammas and n-1 densities, n <= 8")
    r = [0.0] + list(rhos)
    for i in range(n - 1):
        if not r[i + 1] > r[i]:
            raise ValueError("piecewise polytrope densities must ascend")
    k = [0.0] * n
    eps = [0.0] * n
    prs = [0.0] * n
    k[0] = kappa_0
    for i in range(1, n):
        k[i] = k[i - 1] * math.pow(r[i], gammas[i - 1] - gammas[i])
        eps[i] = (eps[i - 1]
                  + k[i - 1] * math.pow(r[i], gammas[i - 1] - 1.0) / (gammas[i - 1] - 1.0)
                  - k[i] * math.pow(r[i], gammas[i] - 1.0) / (gammas[i] - 1.0))
        prs[i] = k[i] * math.pow(r[i], gammas[i])
    e.n_pieces = n
    for i in range(abi.MAX_PIECES):
        e.pw_kappa[i] = k[i] if i < n else 0.0
        e.pw_gamma[i] = gammas[i] if i < n else 0.0
        e.pw_rho[i] = r[i] if i < n else 0.0
        e.pw_eps[i] = eps[i] if i < n else 0.0
        e.pw_press[i] = prs[i] if i < n else 0.0
    return e


def ideal_gas(gamma, **kw):
    p = defaults(abi.EOS_IDEAL_GAS)
    p.eos.gamma = gamma
    return _apply(p, kw)


def hybrid_pwpoly(kappa_0, gammas, rhos=(), gamma_th=1.8, **kw):
    p = defaults(abi.EOS_HYBRID_PWPOLY)
    setup_pwpoly(p.eos, kappa_0, list(gammas), list(rhos))
    p.eos.gamma_th = gamma_th
    return _apply(p, kw)


def _apply(p, kw):
    for key, val in kw.items():
        if key in ("temp_fl",):
            p.temp_fl = val
            p.eos.temp_atm = val       # the EOS atmosphere temperature is temp_fl
            p.temp_ex = val
        elif key in ("rho_fl",):
            p.rho_fl = val
            p.rho_ex = val
        elif hasattr(p.eos, key) and key not in ("kind",):
            setattr(p.eos, key, val)
        elif hasattr(p, key):
            setattr(p, key, val)
        else:
            raise KeyError(key)
    return p


# --- presets: the physics of the benchmark configurations ------------------
def balsara1():
    """Balsara-1 shock tube: ideal gas Gamma=2, WENO-Z + HLLE + UCT, no FOFC."""
    return ideal_gas(2.0, emf=abi.EMF_UCT, fofc_enable=0)


def blast():
    """3-D blast wave: ideal gas Gamma=4/3, WENO-Z + HLLE + Gardiner-Stone + FOFC.

    The unperturbed background has b^2/rho = 0.1^2 / 1e-4 = 100, exactly the
    schema default max_sigma, so the magnetisation clamp of limit_primitives
    (c2p.cpp:101-114) would fire on every background cell; the ceiling is
    raised to 1e3 so that it acts only on states the blast itself creates."""
    return ideal_gas(4.0 / 3.0, emf=abi.EMF_GS, fofc_enable=1, max_sigma=1.0e3)


def c2p_bench():
    """c2p micro-benchmark: hybrid EOS (K=100, Gamma=2, Gamma_th=1.8), 1e-12 acceptance,
    W and sigma ceilings above the sampled ranges."""
    return hybrid_pwpoly(100.0, [2.0], [], gamma_th=1.8, c2p_tol=1e-12, max_w=60.0,
                         max_sigma=2.0e3)


def tov():
    """Magnetised TOV star: hybrid EOS (cold polytrope K=100, Gamma=2;
    thermal Gamma_th=1.8), WENO-Z + HLLE + Gardiner-Stone + FOFC; atmosphere
    floor 1e-12 below the 1e-10 atmosphere of the initial data."""
    return hybrid_pwpoly(100.0, [2.0], [], gamma_th=1.8, emf=abi.EMF_GS, fofc_enable=1, rho_fl=1e-12)


def torus():
    """Fishbone-Moncrief torus: ideal gas Gamma=4/3, WENO-Z + HLLE +
    Gardiner-Stone + FOFC; atmosphere floor 1e-9 below the 1e-8 atmosphere
    of the initial data."""
    return ideal_gas(4.0 / 3.0, emf=abi.EMF_GS, fofc_enable=1, rho_fl=1e-9)
