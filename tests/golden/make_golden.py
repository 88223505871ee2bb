"""Generate the golden fixtures of tests/golden/ from the reference.

Run in a checkout where the GRACE sources are present (the pinning build
oracle/_ref/libgrace_ref.so is built from them by `make -C oracle ref`):

    python tests/golden/make_golden.py /path/to/grace

Fixtures written (small, committed):
  geom_sources.json   the two input -> output golden vectors of the
                      reference's test/test_grmhd_kernels.cpp:375-470,
                      parsed from that file
  c2p_ref.npz         conservs_to_prims of the reference's own code on
                      seeded states (hybrid and ideal-gas EOS, flat and
                      Schwarzschild-CKS metrics) and on the structured
                      sweep of test/test_c2p.cpp:130-218
  kernels_ref.npz     W, b^mu, vtilde, characteristic speeds, conserved
                      and fluxes of the reference's SymPy kernels, WENO-Z /
                      MC2 / minmod / donor reconstruction, on seeded inputs
  stage_ref.npz       one SSP-RK3 step of the small blast-wave (GS + FOFC)
                      and Balsara-1 (UCT) setups with the reference's
                      per-cell numerics driven by the restated loops
"""
import ctypes as C
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from grace_b200 import abi, params, workloads  # noqa: E402
import _oracle  # noqa: E402


def parse_geom_sources(src):
    txt = open(src).read()
    start = txt.index('TEST_CASE("GRMHD kernels / Geom source vs Python reference"')
    body = txt[start:]
    out = []
    for sec in re.split(r'SECTION\(', body)[1:3]:
        def arr(name):
            m = re.search(r"std::array<double,\s*\d+>\s+" + name + r"\s*=\s*\{([^}]*)\}", sec)
            return [float(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()]

        def scal(name):
            m = re.search(r"double const " + name + r"\s*=\s*([-+0-9.eE]+)", sec)
            return float(m.group(1))
        ds = re.search(r"double const ds_ref\[3\]\s*=\s*\{([^}]*)\}", sec).group(1)
        out.append({
            "gdd": arr("gdd"), "guu": arr("guu"), "Kdd": arr("Kdd"), "betau": arr("betau"),
            "dgdd_dx": arr("dgdd_dx"), "dbetau_dx": arr("dbetau_dx"), "dalp_dx": arr("dalp_dx"),
            "B": arr("B"), "z": arr("z"), "alp": scal("alp"), "rho": scal("rho"),
            "press": scal("press"), "eps": scal("eps"), "W": scal("W"),
            "dtau_ref": scal("dtau_ref"),
            "ds_ref": [float(x) for x in ds.replace("\n", " ").split(",") if x.strip()],
        })
    return out


def c2p_structured_states():
    """The structured sweep of test/test_c2p.cpp:40-76 and 130-185: rho in
    10^{-12,-8,-5,-3,-1.5,-0.5}, T in {1e-3,0.1,1,10}, W in {1.05,1.5,2,3},
    six axis directions; primitives on the flat metric."""
    dirs = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    out = []
    for d in dirs:
        for W in (1.05, 1.5, 2.0, 3.0):
            for T in (1e-3, 1e-1, 1.0, 10.0):
                for lr in (-12.0, -8.0, -5.0, -3.0, -1.5, -0.5):
                    out.append((10 ** lr, T, W, d))
    return out


def main(ref_root):
    L = _oracle.lib("ref")
    assert L is not None, "build oracle/_ref first: make -C oracle ref"
    gs = parse_geom_sources(os.path.join(ref_root, "test", "test_grmhd_kernels.cpp"))
    json.dump(gs, open(os.path.join(HERE, "geom_sources.json"), "w"), indent=1)

    # ---- c2p on seeded states
    res = {}
    for tag, P in (("hybrid", params.c2p_bench()),
                   ("ideal", params.ideal_gas(4.0 / 3.0, c2p_tol=1e-12, max_w=60.0, max_sigma=2e3))):
        cons, prims = workloads.c2p_states(3000, seed=21)
        if tag == "ideal":
            # ideal gas: same kinematics, eps from T with Gamma=4/3
            pass
        pr, co, err, fl, it, rc = _oracle.c2p_batch(P, cons, None, "ref")
        res[f"{tag}_cons"] = cons
        res[f"{tag}_prims"] = pr
        res[f"{tag}_cons_out"] = co
        res[f"{tag}_err"] = err
        res[f"{tag}_floored"] = fl
    # Schwarzschild-CKS at R=4 (test_c2p.cpp:249-274), hybrid EOS
    P = params.c2p_bench()
    _, prims = workloads.c2p_states(1000, seed=22)
    n = prims.shape[1]
    H, fac = 0.25, 1.5
    metric = np.zeros((10, n))
    metric[0], metric[3], metric[5] = fac, 1.0, 1.0
    metric[6] = 2 * H / fac
    metric[9] = 1 / np.sqrt(fac)
    cons = np.zeros((10, n))
    L.ref_prims_to_conservs(C.byref(P), n, _oracle.p(np.ascontiguousarray(prims)), _oracle.p(metric),
                            _oracle.p(cons))
    cons[7:10] = prims[abi.P_BX:abi.P_BZ + 1] * np.sqrt(fac)
    pr, co, err, fl, it, rc = _oracle.c2p_batch(P, cons, metric, "ref")
    res.update(curved_cons=cons, curved_metric=metric, curved_prims=pr, curved_err=err)
    # structured sweep, hybrid Gamma=2 K=168.5819 Gamma_th=1.8 (test/configs/c2p_test_gamma2.yaml)
    Ps = params.hybrid_pwpoly(1.685819e+02, [2.0], [], gamma_th=1.8)
    st = c2p_structured_states()
    n = len(st)
    pr0 = np.zeros((13, n))
    T = np.array([s[1] for s in st])
    rho = np.array([s[0] for s in st])
    press = np.zeros(n)
    eps = np.zeros(n)
    cs2 = np.zeros(n)
    t2, r2 = T.copy(), rho.copy()
    L.ref_eos_press_eps_csnd2_temp_rho(C.byref(Ps), n, _oracle.p(t2), _oracle.p(r2), _oracle.p(press),
                                       _oracle.p(eps), _oracle.p(cs2))
    eth = T / 0.8
    pr0[abi.P_RHO], pr0[abi.P_TEMP], pr0[abi.P_PRESS], pr0[abi.P_EPS] = rho, T, press, eps
    pr0[abi.P_ENT] = np.log(np.maximum(eth, 1e-13) * rho ** (-0.8)) / 0.8
    for t, s in enumerate(st):
        zm = np.sqrt(s[2] ** 2 - 1)
        pr0[abi.P_ZX:abi.P_ZZ + 1, t] = [zm * c for c in s[3]]
    cons = np.zeros((10, n))
    L.ref_prims_to_conservs(C.byref(Ps), n, _oracle.p(pr0), None, _oracle.p(cons))
    pr, co, err, fl, it, rc = _oracle.c2p_batch(Ps, cons, None, "ref")
    res.update(sweep_prims0=pr0, sweep_cons=cons, sweep_prims=pr, sweep_err=err, sweep_floored=fl)
    np.savez_compressed(os.path.join(HERE, "c2p_ref.npz"), **res)

    # ---- per-state kernels and reconstruction
    rng = np.random.default_rng(23)
    n = 1500
    inp = np.zeros((n, 24))
    inp[:, 0] = 0.3 + 0.7 * rng.random(n)
    inp[:, 1:4] = 0.2 * rng.standard_normal((n, 3))
    inp[:, 4] = 1 + 0.3 * rng.random(n)
    inp[:, 7] = 1 + 0.3 * rng.random(n)
    inp[:, 9] = 1 + 0.3 * rng.random(n)
    inp[:, [5, 6, 8]] = 0.1 * rng.standard_normal((n, 3))
    inp[:, 10] = 10 ** rng.uniform(-8, 0, n)
    inp[:, 11] = inp[:, 10] * 10 ** rng.uniform(-3, 1, n)
    inp[:, 12] = rng.uniform(0.01, 2, n)
    inp[:, 13] = rng.uniform(0.01, 0.5, n)
    inp[:, 14:17] = 2 * rng.standard_normal((n, 3))
    inp[:, 17:20] = 0.1 * rng.standard_normal((n, 3))
    inp[:, 20] = rng.standard_normal(n)
    kern = {"kernel_in": inp}
    for d in range(3):
        out = np.zeros((n, 32))
        L.ref_kernels(n, _oracle.p(inp), d, _oracle.p(out))
        kern[f"kernel_out_{d}"] = out
    u = rng.standard_normal((n, 6)).cumsum(axis=1)
    kern["recon_in"] = u
    for k in range(4):
        uL, uR = np.zeros(n), np.zeros(n)
        L.ref_recon(k, n, _oracle.p(u), _oracle.p(uL), _oracle.p(uR))
        kern[f"recon_{k}"] = np.stack([uL, uR])
    np.savez_compressed(os.path.join(HERE, "kernels_ref.npz"), **kern)

    # ---- one RK3 step of the small setups with the reference numerics
    stage = {}
    for name, P, (su, f), cfl in (
            ("blast", params.blast(), workloads.blast(nb=(2, 2, 2), n=(8, 8, 8)), 0.25),
            ("balsara", params.balsara1(), workloads.balsara1(nb=(4, 1, 1), n=(8, 8, 8)), 0.4)):
        st_, bx, by, bz, aux = [x.copy() for x in f]
        S = _oracle.Stage(P, su.n[0], su.n[1], su.n[2], su.ngz, su.nq, "ref")
        state = [st_, bx, by, bz]
        _oracle.fill_ghosts("ref", su, state)
        S.compute_aux(su.idx().copy(), state, aux)
        sp = [x.copy() for x in state]
        spp = [x.copy() for x in state]
        _oracle.rk3_step(S, su, cfl / su.idx()[0, 0], state, sp, spp, aux, "ref")
        g = su.ngz
        stage[f"{name}_cons"] = state[0][:, :7, g:-g, g:-g, g:-g]
        stage[f"{name}_bx"], stage[f"{name}_by"], stage[f"{name}_bz"] = state[1], state[2], state[3]
        stage[f"{name}_rho"] = aux[:, abi.RHO, g:-g, g:-g, g:-g]
    np.savez_compressed(os.path.join(HERE, "stage_ref.npz"), **stage)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else _oracle.ref_dir())
