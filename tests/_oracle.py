"""ctypes access to the CPU oracle (oracle/liboracle.so) and, when it was
built in this checkout, the reference-numerics pinning build
(oracle/_ref/libgrace_ref.so).  Test infrastructure only."""
import ctypes as C
import os
import subprocess

import numpy as np

from grace_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "liboracle.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libgrace_ref.so")

VP = C.c_void_p


def _bind(lib, pre):
    P = C.POINTER
    sig = {
        "create": (VP, [P(abi.Params), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64]),
        "destroy": (None, [VP]),
        "advance_substep": (C.c_int, [VP, VP, VP, C.c_double, C.c_double] + [VP] * 9),
        "compute_aux": (C.c_int, [VP, VP, VP] + [VP] * 5),
        "reset_diag": (None, [VP, VP]),
        "find_stable_timestep": (C.c_double, [VP, VP, VP, VP, C.c_double]),
        "linop": (None, [VP] + [VP] * 12 + [C.c_double, C.c_double]),
        "scratch": (C.c_int64, [VP, C.c_int, VP]),
        "boundary_outflow": (C.c_double, [VP, C.c_int64, VP, VP, VP, C.c_double, C.c_double]),
        "fofc_counts": (None, [VP, P(C.c_int64), P(C.c_int64)]),
        "set_reflux": (None, [VP, C.c_int64, VP, VP, VP, C.c_int64, VP, VP, C.c_int32, C.c_int64, VP, VP, VP, VP, VP,
                              C.c_int64, VP, VP, VP]),
        "c2p_batch": (C.c_int, [P(abi.Params), C.c_int64, VP, VP, VP, VP, VP, VP, C.c_int32, VP]),
        "prims_to_conservs": (C.c_int, [P(abi.Params), C.c_int64, VP, VP, VP]),
        "eos_press_eps_csnd2_temp_rho": (C.c_int, [P(abi.Params), C.c_int64, VP, VP, VP, VP, VP]),
        "recon": (None, [C.c_int, C.c_int64, VP, VP, VP]),
        "kernels": (None, [C.c_int64, VP, C.c_int, VP]),
        "geom_sources": (None, [C.c_int64, VP, VP]),
        "fill_ghosts_brick": (None, [C.c_int] * 7 + [VP, VP, VP, VP, VP]),
        "restrict_cells": (None, [C.c_int, C.c_int, C.c_int, VP, VP, C.c_int64, VP, VP, VP, VP, C.c_int, VP,
                                  C.c_int]),
        "restrict_faces": (None, [C.c_int, C.c_int, C.c_int, VP, VP, C.c_int64, VP, VP]),
        "prolong_cells": (None, [C.c_int] * 4 + [VP, VP, C.c_int64, VP, VP, VP, VP, C.c_int, VP, C.c_int]),
        "prolong_faces": (None, [C.c_int] * 3 + [VP] * 6 + [C.c_int64, VP, VP, VP, VP]),
    }
    for name, (res, args) in sig.items():
        if not hasattr(lib, pre + name):  # the pinning build exports a subset
            continue
        fn = getattr(lib, pre + name)
        fn.restype = res
        fn.argtypes = args
    return lib


def restrict_cells(which, n, ngz, nvars, src, dst, src_q, dst_q, child, vlo, vhi):
    """FMR restriction of cell variables into coarse buffers (amr_oracle.hpp)."""
    L = lib(which)
    q = lambda a, t: np.ascontiguousarray(a, dtype=t)
    sq, dq, ch = q(src_q, np.int64), q(dst_q, np.int64), q(child, np.uint8)
    vl, vh = q(vlo, np.int32), q(vhi, np.int32)
    getattr(L, which + "_restrict_cells")(n, ngz, nvars, p(src), p(dst), len(sq), p(sq), p(dq), p(ch),
                                          p(vl), len(vl), p(vh), len(vh))


def restrict_faces(dir, n, ngz, src, dst, src_q, dst_q):
    L = lib("orc")
    q = lambda a: np.ascontiguousarray(a, dtype=np.int64)
    sq, dq = q(src_q), q(dst_q)
    L.orc_restrict_faces(dir, n, ngz, p(src), p(dst), len(sq), p(sq), p(dq))


def prolong_cells(which, kind, n, ngz, nvars, fine, cbuf, fine_q, cbuf_q, elem, vlo, vhi):
    """FMR prolongation of cell variables into the ghost elements of one kind
    (0 faces, 1 edges, 2 corners) from coarse buffers (amr_oracle.hpp)."""
    L = lib(which)
    q = lambda a, t: np.ascontiguousarray(a, dtype=t)
    fq, cq, el = q(fine_q, np.int64), q(cbuf_q, np.int64), q(elem, np.uint8)
    vl, vh = q(vlo, np.int32), q(vhi, np.int32)
    getattr(L, which + "_prolong_cells")(kind, n, ngz, nvars, p(fine), p(cbuf), len(fq), p(fq), p(cq), p(el),
                                         p(vl), len(vl), p(vh), len(vh))


def prolong_faces(which, kind, n, ngz, fine, cbuf, fine_q, cbuf_q, elem, have_fine):
    """Divergence-preserving prolongation of face B into the ghost elements of
    one kind; fine, cbuf: (bx, by, bz) arrays; have_fine (nelems, 3, 2)."""
    L = lib(which)
    q = lambda a, t: np.ascontiguousarray(a, dtype=t)
    fq, cq, el, hf = q(fine_q, np.int64), q(cbuf_q, np.int64), q(elem, np.uint8), q(have_fine, np.int8)
    getattr(L, which + "_prolong_faces")(kind, n, ngz, p(fine[0]), p(fine[1]), p(fine[2]), p(cbuf[0]), p(cbuf[1]),
                                         p(cbuf[2]), len(fq), p(fq), p(cq), p(el), p(hf))


def build_oracle():
    """Build liboracle.so (and the pinning build when the GRACE sources are
    present; oracle/Makefile knows where) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", "ref-if-present"], check=True)


def ref_dir():
    """The GRACE source tree the pinning build compiles (oracle/Makefile's
    REF: GRACE_REF_DIR or its default)."""
    return subprocess.run(["make", "-s", "--no-print-directory", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                          check=True, capture_output=True, text=True).stdout.strip()


_cache = {}


def lib(which="orc"):
    if which in _cache:
        return _cache[which]
    path = ORACLE if which == "orc" else REF
    if not os.path.exists(path):
        if which == "orc":
            build_oracle()
        if not os.path.exists(path):
            return None
    L = _bind(C.CDLL(path), which + "_")
    _cache[which] = L
    return L


def p(a):
    return a.ctypes.data_as(VP) if a is not None else None


def mlp_lib():
    """liboracle.so with the bracket-network oracle bound (orc_ only)."""
    L = lib("orc")
    P = C.POINTER
    for name, res, args in (
            ("orc_mlp_num_params", C.c_int, []),
            ("orc_mlp_features", None, [P(abi.Params), C.c_int64, VP, VP, VP]),
            ("orc_mlp_forward", None, [VP, C.c_int64, VP, C.c_int32, VP]),
            ("orc_mlp_loss_grad", C.c_double, [VP, C.c_int64, VP, VP, C.c_int32, VP]),
            ("orc_c2p_batch_guess", C.c_int, [P(abi.Params), C.c_int64, VP, VP, VP, VP, VP, VP, VP, VP,
                                              VP, VP])):
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def mlp_features(params, cons, metric=None):
    n = cons.shape[1]
    f = np.zeros((abi.MLP_IN, n), np.float32)
    mlp_lib().orc_mlp_features(C.byref(params), n, p(np.ascontiguousarray(cons)),
                               p(np.ascontiguousarray(metric) if metric is not None else None), p(f))
    return f


def mlp_forward(P, feat, emulate=True):
    n = feat.shape[1]
    out = np.zeros(n)
    mlp_lib().orc_mlp_forward(p(np.ascontiguousarray(P, np.float32)), n,
                              p(np.ascontiguousarray(feat, np.float32)), 1 if emulate else 0, p(out))
    return out


def mlp_loss_grad(P, feat, tgt, emulate=True):
    n = feat.shape[1]
    g = np.zeros(abi.MLP_NUM_WEIGHTS)
    loss = mlp_lib().orc_mlp_loss_grad(p(np.ascontiguousarray(P, np.float32)), n,
                                       p(np.ascontiguousarray(feat, np.float32)),
                                       p(np.ascontiguousarray(tgt, np.float32)), 1 if emulate else 0, p(g))
    return loss, g


def c2p_batch_guess(params, cons, lo, hi, metric=None):
    n = cons.shape[1]
    pr = np.zeros((13, n))
    co = np.zeros((10, n))
    err = np.zeros(n, np.uint32)
    it = np.zeros(n, np.int32)
    gu = np.zeros(n, np.int8)
    mu = np.zeros(n)
    rc = mlp_lib().orc_c2p_batch_guess(C.byref(params), n, p(np.ascontiguousarray(cons)), p(metric),
                                       p(np.ascontiguousarray(lo)), p(np.ascontiguousarray(hi)), p(pr), p(co),
                                       p(err), p(it), p(gu), p(mu))
    return pr, co, err, it, gu, mu, rc


class Stage:
    """Oracle stage driver on host numpy arrays (GRACE LayoutLeft shapes)."""

    def __init__(self, params, nx, ny, nz, g, nq, which="orc"):
        self.L = lib(which)
        self.pre = which + "_"
        self.params = params
        self.h = getattr(self.L, self.pre + "create")(C.byref(params), nx, ny, nz, g, nq)

    def __del__(self):
        try:
            getattr(self.L, self.pre + "destroy")(self.h)
        except Exception:
            pass

    def advance_substep(self, idx, dt, dtfact, new, old, aux, coords=None):
        return getattr(self.L, self.pre + "advance_substep")(
            self.h, p(idx), p(coords), dt, dtfact, p(new[0]), p(new[1]), p(new[2]), p(new[3]),
            p(old[0]), p(old[1]), p(old[2]), p(old[3]), p(aux))

    def compute_aux(self, idx, st, aux, coords=None):
        return getattr(self.L, self.pre + "compute_aux")(self.h, p(idx), p(coords), p(st[0]), p(st[1]),
                                                         p(st[2]), p(st[3]), p(aux))

    def reset_diag(self, aux):
        getattr(self.L, self.pre + "reset_diag")(self.h, p(aux))

    def find_stable_timestep(self, st, aux, dx, cfl):
        """find_stable_timestep_impl: min over interior cells of
        cfl / cmax * dx(0, q)."""
        return getattr(self.L, self.pre + "find_stable_timestep")(self.h, p(st[0]), p(aux), p(dx), cfl)

    def linop(self, A, B, Cf, b, c):
        Cp = [p(x) for x in Cf] if Cf is not None else [None] * 4
        getattr(self.L, self.pre + "linop")(self.h, *[p(x) for x in A], *[p(x) for x in B], *Cp, b, c)

    def set_reflux(self, r, flux_same=False):
        """Reflux descriptor lists (the dict of grace_b200.fmr.Hierarchy.reflux_lists)."""
        self._rf = {k: np.ascontiguousarray(v) for k, v in r.items()}  # kept alive
        x = self._rf
        getattr(self.L, self.pre + "set_reflux")(
            self.h, len(x["face_coarse_q"]), p(x["face_coarse_q"]), p(x["face_coarse_id"]), p(x["face_fine_q"]),
            len(x["same_face_q"]) // 2, p(x["same_face_q"]), p(x["same_face_id"]), 1 if flux_same else 0,
            len(x["edge_nsides"]), p(x["edge_nsides"]), p(x["edge_id"]), p(x["edge_is_fine"]), p(x["edge_q"]),
            p(x["edge_off"]), len(x["same_edge_nsides"]), p(x["same_edge_nsides"]), p(x["same_edge_id"]),
            p(x["same_edge_q"]))

    def fofc_counts(self):
        f, e = C.c_int64(), C.c_int64()
        getattr(self.L, self.pre + "fofc_counts")(self.h, C.byref(f), C.byref(e))
        return f.value, e.value

    def boundary_outflow(self, quad, face, dx, dt, dtfact):
        """Mass outflux of the last substep through the listed faces."""
        q = np.ascontiguousarray(quad, dtype=np.int64)
        f = np.ascontiguousarray(face, dtype=np.uint8)
        d = np.ascontiguousarray(dx, dtype=np.float64)
        return getattr(self.L, self.pre + "boundary_outflow")(self.h, len(q), p(q), p(f), p(d), dt, dtfact)

    def scratch(self, which):
        n = getattr(self.L, self.pre + "scratch")(self.h, which, None)
        out = np.empty(n)
        getattr(self.L, self.pre + "scratch")(self.h, which, p(out))
        return out


def fill_ghosts(which, setup, fields):
    L = lib(which)
    per = np.asarray([int(x) for x in setup.periodic], dtype=np.int32)
    getattr(L, which + "_fill_ghosts_brick")(setup.n[0], setup.n[1], setup.n[2], setup.ngz,
                                             setup.nb[0], setup.nb[1], setup.nb[2], p(per),
                                             p(fields[0]), p(fields[1]), p(fields[2]), p(fields[3]))


def rk3_step(st, setup, dt, state, state_p, state_pp, aux, which="orc"):
    """One SSP-RK3 step of evolve_impl (evolve.cpp:147-225) on host arrays."""
    idx = setup.idx().copy()
    bc = lambda f: fill_ghosts(which, setup, f)
    st.reset_diag(aux)
    st.advance_substep(idx, dt, 1.0, state_p, state, aux)
    bc(state_p)
    st.compute_aux(idx, state_p, aux)
    st.linop(state_pp, state, state_p, 0.75, 0.25)
    st.advance_substep(idx, dt, 0.25, state_pp, state_p, aux)
    bc(state_pp)
    st.compute_aux(idx, state_pp, aux)
    st.linop(state, state, state_pp, 1.0 / 3, 2.0 / 3.0)
    st.advance_substep(idx, dt, 2.0 / 3.0, state, state_pp, aux)
    bc(state)
    st.compute_aux(idx, state, aux)
    st.linop(state_p, state, None, 1.0, 0.0)


def c2p_batch(params, cons, metric=None, which="orc", dry_run=False):
    L = lib(which)
    n = cons.shape[1]
    cons = np.ascontiguousarray(cons)
    pr = np.zeros((13, n))
    co = np.zeros((10, n))
    err = np.zeros(n, np.uint32)
    fl = np.zeros(n, np.int32)
    it = np.zeros(n, np.int32)
    rc = getattr(L, which + "_c2p_batch")(C.byref(params), n, p(cons), p(metric), p(pr), p(co), p(err),
                                          p(fl), 1 if dry_run else 0, p(it))
    return pr, co, err, fl, it, rc
