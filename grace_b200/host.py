"""Host-side mirror of GRACE's Cowling GRMHD evolution interface.

The names and argument meanings follow the reference's free functions:
  advance_substep(t, dt, dtfact, new_state, old_state, new_stag, old_stag)
      src/evolution/evolve.cpp:1671-1717
  compute_auxiliary_quantities(state, sstate, aux)
      src/evolution/auxiliaries.cpp:81-180
  linop_apply(A, B, C, AS, BS, CS, b, c)
      include/grace/utils/tstep_utils.hh:54-229
  evolve_impl<eos_t>() RK3 branch
      src/evolution/evolve.cpp:190-225
Every call goes through the C ABI of libgrace_b200.so on torch CUDA tensors
(device memory and streams only; all arithmetic is in the CUDA library).
Errors surface as RuntimeError with the library's status code, as GRACE's
ERROR() macro would abort the run.
"""
import contextlib
import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, abi


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream_ptr(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


@dataclass
class Fields:
    """One evolved state: GRACE's var_array_t + staggered_variable_arrays_t.

    state: (nq, 23, NZ, NY, NX) float64, bx: (nq, NZ, NY, NX+1),
    by: (nq, NZ, NY+1, NX), bz: (nq, NZ+1, NY, NX) — C order, which is
    GRACE's LayoutLeft (i fastest, block index slowest).
    """
    state: torch.Tensor
    bx: torch.Tensor
    by: torch.Tensor
    bz: torch.Tensor

    def c(self):
        return abi.Fields(self.state.data_ptr(), self.bx.data_ptr(), self.by.data_ptr(),
                          self.bz.data_ptr())

    def copy_(self, other):
        self.state.copy_(other.state)
        self.bx.copy_(other.bx)
        self.by.copy_(other.by)
        self.bz.copy_(other.bz)
        return self

    def clone(self):
        return Fields(self.state.clone(), self.bx.clone(), self.by.clone(), self.bz.clone())

    def to(self, device):
        return Fields(self.state.to(device), self.bx.to(device), self.by.to(device),
                      self.bz.to(device))

    def view(self, q0, q1):
        """Blocks [q0, q1) of the four arrays (views, no copy)."""
        return Fields(self.state[q0:q1], self.bx[q0:q1], self.by[q0:q1], self.bz[q0:q1])


class Blocks:
    """Block geometry: nq blocks of nx*ny*nz interior cells with ngz ghosts."""

    def __init__(self, nx, ny, nz, ngz, nq, idx, coords=None, device="cuda"):
        self.nx, self.ny, self.nz, self.ngz, self.nq = nx, ny, nz, ngz, nq
        self.NX, self.NY, self.NZ = nx + 2 * ngz, ny + 2 * ngz, nz + 2 * ngz
        self.idx = torch.as_tensor(idx, dtype=torch.float64, device=device).reshape(nq, 3).contiguous()
        self.coords = (None if coords is None else
                       torch.as_tensor(coords, dtype=torch.float64, device=device).reshape(nq, 3).contiguous())
        self.device = device

    def c(self):
        return abi.Grid(self.nx, self.ny, self.nz, self.ngz, self.nq, self.idx.data_ptr(),
                        self.coords.data_ptr() if self.coords is not None else None)

    def view(self, q0, q1):
        """The run of blocks [q0, q1): the same geometry, nq = q1 - q0, the
        spacings and coordinates as views of this object's (no copy)."""
        if not 0 <= q0 < q1 <= self.nq:
            raise ValueError(f"block run [{q0}, {q1}) outside [0, {self.nq})")
        v = object.__new__(Blocks)
        v.__dict__.update(self.__dict__)
        v.nq = q1 - q0
        v.idx = self.idx[q0:q1]
        v.coords = None if self.coords is None else self.coords[q0:q1]
        v.q0 = q0
        return v

    def new_fields(self):
        z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=self.device)
        return Fields(z(self.nq, abi.N_EVOL_VARS, self.NZ, self.NY, self.NX),
                      z(self.nq, self.NZ, self.NY, self.NX + 1),
                      z(self.nq, self.NZ, self.NY + 1, self.NX),
                      z(self.nq, self.NZ + 1, self.NY, self.NX))

    def new_aux(self):
        return torch.zeros(self.nq, abi.N_AUX_VARS, self.NZ, self.NY, self.NX,
                           dtype=torch.float64, device=self.device)


def brick_runs(nb, periodic, nruns):
    """Runs of blocks for rk3_step_host on a brick of nb = (nbx, nby, nbz)
    blocks (block q = bx + nbx (by + nby bz)): nruns consecutive runs of
    whole z-slabs, as even as the slabs allow, and for each run the set of
    runs whose blocks its ghost fill reads (the face, edge and corner
    neighbours, wrapping along periodic axes; a non-periodic outer face
    copies from the block itself)."""
    nbx, nby, nbz = nb
    nruns = max(1, min(int(nruns), nbz))
    cuts = [round(r * nbz / nruns) for r in range(nruns + 1)]
    slab = nbx * nby
    runs = [(cuts[r] * slab, cuts[r + 1] * slab) for r in range(nruns)]
    run_of_z = np.zeros(nbz, dtype=np.int64)
    for r in range(nruns):
        run_of_z[cuts[r]:cuts[r + 1]] = r
    deps = []
    for r in range(nruns):
        d = set()
        for z in range(cuts[r], cuts[r + 1]):
            for o in (-1, 0, 1):
                zz = z + o
                if periodic[2]:
                    zz %= nbz
                elif not 0 <= zz < nbz:
                    continue
                d.add(int(run_of_z[zz]))
        deps.append(d)
    return runs, deps


def gather_runs(maps, blocks, nruns):
    """Runs of blocks for rk3_step_host on a hierarchy filled by gather maps
    (grace_b200.fmr.Hierarchy.gather_maps): nruns consecutive runs of about
    nq / nruns blocks; for each run the part of the maps whose destinations
    lie in its blocks, and the runs whose blocks those entries read (the
    run itself included).  Returns (runs, run_maps, deps)."""
    nq = blocks.nq
    nruns = max(1, min(int(nruns), nq))
    cuts = [round(r * nq / nruns) for r in range(nruns + 1)]
    runs = [(cuts[r], cuts[r + 1]) for r in range(nruns)]
    run_of = np.zeros(nq, dtype=np.int64)
    for r, (q0, q1) in enumerate(runs):
        run_of[q0:q1] = r
    NX, NY, NZ = blocks.NX, blocks.NY, blocks.NZ
    qstride = {"cells": abi.N_EVOL_VARS * NX * NY * NZ, 0: (NX + 1) * NY * NZ, 1: NX * (NY + 1) * NZ,
               2: NX * NY * (NZ + 1)}
    run_maps = [dict() for _ in runs]
    deps = [{r} for r in range(nruns)]
    for key, m in maps.items():
        dst_run = run_of[m["dst"] // qstride[key]]
        used = np.arange(m["src"].shape[0])[:, None] < m["cnt"][None, :]
        src_run = run_of[np.where(used, m["src"], 0) // qstride[key]]
        for r in range(nruns):
            sel = dst_run == r
            run_maps[r][key] = {"cnt": np.ascontiguousarray(m["cnt"][sel]), "dst": np.ascontiguousarray(m["dst"][sel]),
                                "src": np.ascontiguousarray(m["src"][:, sel]), "w": np.ascontiguousarray(m["w"][:, sel])}
            deps[r] |= {int(x) for x in np.unique(src_run[:, sel][used[:, sel]])}
    return runs, run_maps, deps


class GRMHDEquationsSystem:
    """grmhd_equations_system_t<eos_t> + the evolve.cpp drivers, on the GPU."""

    def __init__(self, params, variant="default"):
        """variant "exact": the -fmad=false build of the library (parity
        tests); the default build otherwise."""
        self.lib = _lib.load(variant)
        self.params = params
        h = ctypes.c_void_p()
        _lib.check(self.lib.grb_create(ctypes.byref(h), ctypes.byref(params)), "grb_create")
        self.h = h
        self._grid = None

    def close(self):
        if self.h:
            self.lib.grb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, blocks):
        self._grid = blocks.c()
        _lib.check(self.lib.grb_reserve(self.h, ctypes.byref(self._grid)), "grb_reserve")
        self.blocks = blocks

    def advance_substep(self, t, dt, dtfact, new_state, old_state, aux, stream=None):
        g = self.blocks.c()
        nf, of = new_state.c(), old_state.c()
        _lib.check(self.lib.grb_advance_substep(self.h, ctypes.byref(g), t, dt, dtfact,
                                                ctypes.byref(nf), ctypes.byref(of), _ptr(aux),
                                                _stream_ptr(stream)), "grb_advance_substep")

    def compute_auxiliary_quantities(self, state, aux, stream=None):
        g = self.blocks.c()
        f = state.c()
        _lib.check(self.lib.grb_compute_auxiliary_quantities(self.h, ctypes.byref(g), ctypes.byref(f),
                                                             _ptr(aux), _stream_ptr(stream)),
                   "grb_compute_auxiliary_quantities")

    def compute_auxiliary_quantities_dt(self, state, aux, dx, cfl, dt_out, stream=None):
        """compute_auxiliary_quantities fused with find_stable_timestep_impl:
        dt_out (float64 device tensor, one element) receives the minimum of
        cfl / cmax * dx(0, q) over the interior cells."""
        g = self.blocks.c()
        f = state.c()
        _lib.check(self.lib.grb_compute_auxiliary_quantities_dt(self.h, ctypes.byref(g), ctypes.byref(f), _ptr(aux),
                                                                _ptr(dx), cfl, _ptr(dt_out), _stream_ptr(stream)),
                   "grb_compute_auxiliary_quantities_dt")

    def find_stable_timestep(self, state, aux, dx, cfl, dt_out, stream=None):
        """find_stable_timestep_impl on this rank's blocks (separate pass)."""
        g = self.blocks.c()
        f = state.c()
        _lib.check(self.lib.grb_find_stable_timestep(self.h, ctypes.byref(g), ctypes.byref(f), _ptr(aux), _ptr(dx),
                                                     cfl, _ptr(dt_out), _stream_ptr(stream)),
                   "grb_find_stable_timestep")

    def reset_c2p_diagnostics(self, aux, stream=None):
        g = self.blocks.c()
        _lib.check(self.lib.grb_reset_c2p_diagnostics(self.h, ctypes.byref(g), _ptr(aux),
                                                      _stream_ptr(stream)), "grb_reset_c2p_diagnostics")

    def linop_apply(self, A, B, C, b, c=0.0, stream=None):
        g = self.blocks.c()
        fa, fb = A.c(), B.c()
        fc = C.c() if C is not None else None
        _lib.check(self.lib.grb_linop_apply(self.h, ctypes.byref(g), ctypes.byref(fa), ctypes.byref(fb),
                                            ctypes.byref(fc) if fc is not None else None, b, c,
                                            _stream_ptr(stream)), "grb_linop_apply")

    def linop_apply3(self, A, B, C, D, b, c, d, stream=None):
        """The three-term linop_apply (tstep_utils.hh:231-311): A = b B + c C +
        d D on every cell and face (grb_linop_apply3)."""
        g = self.blocks.c()
        f = [x.c() for x in (A, B, C, D)]
        _lib.check(self.lib.grb_linop_apply3(self.h, ctypes.byref(g), *[ctypes.byref(x) for x in f], b, c, d,
                                             _stream_ptr(stream)), "grb_linop_apply3")

    def fill_ghosts_brick(self, fields, nb, periodic, stream=None, blocks=None):
        """Ghost fill of a brick of same-level blocks (grb_fill_ghosts_brick);
        blocks = (q0, q1): only the ghost zones of those blocks
        (grb_fill_ghosts_brick_range)."""
        g = self.blocks.c()
        f = fields.c()
        per = (ctypes.c_int32 * 3)(*[int(bool(x)) for x in periodic])
        if blocks is None:
            _lib.check(self.lib.grb_fill_ghosts_brick(self.h, ctypes.byref(g), ctypes.byref(f), nb[0], nb[1],
                                                      nb[2], per, _stream_ptr(stream)), "grb_fill_ghosts_brick")
        else:
            _lib.check(self.lib.grb_fill_ghosts_brick_range(self.h, ctypes.byref(g), ctypes.byref(f), nb[0],
                                                            nb[1], nb[2], per, int(blocks[0]), int(blocks[1]),
                                                            _stream_ptr(stream)), "grb_fill_ghosts_brick_range")

    @contextlib.contextmanager
    def block_range(self, q0, q1):
        """Within the context every call of this object runs on the blocks
        [q0, q1) of the reserved grid only (pass Fields.view(q0, q1) and
        aux[q0:q1] as its arrays).  Stages are block-local once the ghost
        zones are filled, so a run of blocks gives the same bits as the
        whole grid there; the static-metric cache is found at block q0."""
        full = self.blocks
        self.blocks = full.view(q0, q1)
        try:
            yield self
        finally:
            self.blocks = full

    def restrict_to_coarse(self, fine, cbuf, src_q, dst_q, child_id=None, vars_lo=(), vars_ho=(),
                           faces=True, stream=None):
        """FMR restriction into coarse buffers (grb_restrict_to_coarse).
        fine, cbuf: Fields on the device (same block geometry); src_q,
        dst_q: int64 device tensors; child_id: uint8 device tensor (needed
        with vars_ho); faces: also restrict face B."""
        g = self.blocks.c()
        ff = abi.Fields(fine.state.data_ptr(), *(x.data_ptr() if faces else None for x in (fine.bx, fine.by, fine.bz)))
        fc = abi.Fields(cbuf.state.data_ptr(), *(x.data_ptr() if faces else None for x in (cbuf.bx, cbuf.by, cbuf.bz)))
        for t, dt in ((src_q, torch.int64), (dst_q, torch.int64)):
            if t.dtype != dt or not t.is_cuda or not t.is_contiguous():
                raise ValueError("src_q / dst_q must be contiguous int64 device tensors")
        if child_id is not None and (child_id.dtype != torch.uint8 or not child_id.is_cuda):
            raise ValueError("child_id must be a uint8 device tensor")
        lo = (ctypes.c_int32 * max(1, len(vars_lo)))(*vars_lo)
        hi = (ctypes.c_int32 * max(1, len(vars_ho)))(*vars_ho)
        _lib.check(self.lib.grb_restrict_to_coarse(
            self.h, ctypes.byref(g), ctypes.byref(ff), ctypes.byref(fc), src_q.numel(), src_q.data_ptr(),
            dst_q.data_ptr(), child_id.data_ptr() if child_id is not None else None, lo, len(vars_lo), hi,
            len(vars_ho), _stream_ptr(stream)), "grb_restrict_to_coarse")

    def accumulate_boundary_outflow(self, quad, face, dx, dt, dtfact, outflow, stream=None):
        """Add the substep's mass outflux through the listed outer-boundary
        faces to the device scalar `outflow` (grb_accumulate_boundary_outflow).
        quad: int64, face: uint8 device tensors; dx: float64 device tensor
        (nq, 3) of cell spacings; outflow: float64 device tensor of one
        element."""
        for t, dt_ in ((quad, torch.int64), (face, torch.uint8), (dx, torch.float64), (outflow, torch.float64)):
            if t.dtype != dt_ or not t.is_cuda or not t.is_contiguous():
                raise ValueError("quad, face, dx and outflow must be contiguous device tensors of the documented types")
        g = self.blocks.c()
        _lib.check(self.lib.grb_accumulate_boundary_outflow(
            self.h, ctypes.byref(g), quad.numel(), quad.data_ptr(), face.data_ptr(), dx.data_ptr(), float(dt),
            float(dtfact), outflow.data_ptr(), _stream_ptr(stream)), "grb_accumulate_boundary_outflow")

    def prolong_to_ghosts(self, fine, cbuf, elem_kind, fine_q, cbuf_q, elem_id, have_fine=None, vars_lo=(),
                          vars_ho=(), faces=True, stream=None):
        """FMR prolongation into the ghost elements of one kind
        (grb_prolong_to_ghosts; elem_kind 0 faces, 1 edges, 2 corners).
        fine, cbuf: Fields on the device (same block geometry); fine_q,
        cbuf_q: int64 device tensors; elem_id: uint8 device tensor;
        have_fine: int8 device tensor (nelems, 3, 2), needed with faces."""
        g = self.blocks.c()
        ff = abi.Fields(fine.state.data_ptr(), *(x.data_ptr() if faces else None for x in (fine.bx, fine.by, fine.bz)))
        fc = abi.Fields(cbuf.state.data_ptr(), *(x.data_ptr() if faces else None for x in (cbuf.bx, cbuf.by, cbuf.bz)))
        for t, dt in ((fine_q, torch.int64), (cbuf_q, torch.int64), (elem_id, torch.uint8)):
            if t.dtype != dt or not t.is_cuda or not t.is_contiguous():
                raise ValueError("fine_q / cbuf_q must be int64 and elem_id uint8 contiguous device tensors")
        if faces and (have_fine is None or have_fine.dtype != torch.int8 or not have_fine.is_cuda
                      or not have_fine.is_contiguous() or have_fine.numel() != 6 * fine_q.numel()):
            raise ValueError("have_fine must be a contiguous int8 device tensor of shape (nelems, 3, 2)")
        lo = (ctypes.c_int32 * max(1, len(vars_lo)))(*vars_lo)
        hi = (ctypes.c_int32 * max(1, len(vars_ho)))(*vars_ho)
        _lib.check(self.lib.grb_prolong_to_ghosts(
            self.h, ctypes.byref(g), ctypes.byref(ff), ctypes.byref(fc), elem_kind, fine_q.numel(),
            fine_q.data_ptr(), cbuf_q.data_ptr(), elem_id.data_ptr(),
            have_fine.data_ptr() if (faces and have_fine is not None) else None, lo, len(vars_lo), hi,
            len(vars_ho), _stream_ptr(stream)), "grb_prolong_to_ghosts")

    def set_static_metric(self, fields=None, stream=None):
        """Cowling: cache the metric derivatives of `fields` for the tuned
        update (grb_set_static_metric); None frees the cache."""
        g = self.blocks.c()
        f = fields.c() if fields is not None else None
        _lib.check(self.lib.grb_set_static_metric(self.h, ctypes.byref(g), ctypes.byref(f) if f is not None else None,
                                                  _stream_ptr(stream)), "grb_set_static_metric")

    def packed_host_fields(self, pin=True):
        """Host Fields in the packed interior layout of grb_copy_evolved_packed."""
        b = self.blocks
        e = lambda *s: torch.empty(*s, dtype=torch.float64, pin_memory=pin)
        return Fields(e(b.nq, abi.N_HRSC, b.nz, b.ny, b.nx), e(b.nq, b.nz, b.ny, b.nx + 1),
                      e(b.nq, b.nz, b.ny + 1, b.nx), e(b.nq, b.nz + 1, b.ny, b.nx))

    def copy_evolved_packed(self, host, dev, to_device, stream=None, arrays=(True, True, True, True)):
        """Interior of the evolved variables between packed host tensors
        (packed_host_fields) and the device Fields (grb_copy_evolved_packed);
        `arrays` selects state, bx, by, bz."""
        b = self.blocks
        shapes = [(b.nq, abi.N_HRSC, b.nz, b.ny, b.nx), (b.nq, b.nz, b.ny, b.nx + 1),
                  (b.nq, b.nz, b.ny + 1, b.nx), (b.nq, b.nz + 1, b.ny, b.nx)]
        for h, shp in zip((host.state, host.bx, host.by, host.bz), shapes):
            if h.device.type != "cpu" or not h.is_contiguous() or h.dtype != torch.float64 or \
                    tuple(h.shape) != shp:
                raise ValueError(f"packed host array must be a contiguous float64 CPU tensor of shape {shp}")
        g = b.c()
        ph = [x.data_ptr() if on else None for x, on in zip((host.state, host.bx, host.by, host.bz), arrays)]
        pd = [x.data_ptr() if on else None for x, on in zip((dev.state, dev.bx, dev.by, dev.bz), arrays)]
        fh, fd = abi.Fields(*ph), abi.Fields(*pd)
        _lib.check(self.lib.grb_copy_evolved_packed(self.h, ctypes.byref(g), ctypes.byref(fh), ctypes.byref(fd),
                                                    1 if to_device else 0, _stream_ptr(stream)),
                   "grb_copy_evolved_packed")

    def copy_evolved_interior(self, host, dev, to_device, stream=None):
        """Interior of the evolved variables between pinned host tensors and
        the device Fields `dev` (grb_copy_evolved_interior).  host: Fields of
        pinned CPU tensors shaped like dev's, except that host.state may hold
        only the 7 HRSC variables, (nq, 7, NZ, NY, NX)."""
        for h, d in zip((host.state, host.bx, host.by, host.bz), (dev.state, dev.bx, dev.by, dev.bz)):
            if h.device.type != "cpu" or not h.is_pinned() or not h.is_contiguous() or h.dtype != torch.float64:
                raise ValueError("host arrays must be contiguous pinned float64 CPU tensors")
            if h is not host.state and tuple(h.shape) != tuple(d.shape):
                raise ValueError("host face array shape differs from the device one")
        nv = host.state.shape[1]
        if tuple(host.state.shape) != (dev.state.shape[0], nv) + tuple(dev.state.shape[2:]) or \
                nv not in (abi.N_HRSC, dev.state.shape[1]):
            raise ValueError("host state must be (nq, 7 or 23, NZ, NY, NX) like the device state")
        g = self.blocks.c()
        fh, fd = host.c(), dev.c()
        _lib.check(self.lib.grb_copy_evolved_interior(self.h, ctypes.byref(g), ctypes.byref(fh), int(nv),
                                                      ctypes.byref(fd), 1 if to_device else 0,
                                                      _stream_ptr(stream)), "grb_copy_evolved_interior")

    def conservs_to_prims(self, cons, metric=None, cons_out=None, err=None, use_learned=False,
                          stream=None, diag=None):
        """Batched c2p: cons (10, n) float64 -> prims (13, n).  diag: dict
        with optional device tensors "iters" (int32 [n]), "guess_used"
        (int8 [n]), "mu" (float64 [n]), "bracket" (float64 [2, n])."""
        n = cons.shape[1]
        prims = torch.empty(abi.P_CS2 + 1, n, dtype=torch.float64, device=cons.device)
        if diag is None:
            _lib.check(self.lib.grb_c2p_batch(self.h, n, _ptr(cons), _ptr(metric), _ptr(prims), _ptr(cons_out),
                                              _ptr(err), 1 if use_learned else 0, _stream_ptr(stream)),
                       "grb_c2p_batch")
        else:
            d = abi.C2PDiag(*[_ptr(diag.get(k)) for k in ("iters", "guess_used", "mu", "bracket")])
            _lib.check(self.lib.grb_c2p_batch_diag(self.h, n, _ptr(cons), _ptr(metric), _ptr(prims),
                                                   _ptr(cons_out), _ptr(err), 1 if use_learned else 0,
                                                   ctypes.byref(d), _stream_ptr(stream)), "grb_c2p_batch_diag")
        return prims

    # ---- learned c2p bracket -------------------------------------------
    def train_c2p_model(self, cons, metric=None, stream=None, **cfg):
        """Train the bracket network on the GPU from the states cons (10, n);
        cfg: steps, batch, lr, lr_min, seed, calib_states.  Returns the
        training report as a dict."""
        c = abi.TrainConfig()
        self.lib.grb_train_config_defaults(ctypes.byref(c))
        for k, v in cfg.items():
            setattr(c, k, v)
        r = abi.TrainReport()
        _lib.check(self.lib.grb_c2p_train(self.h, cons.shape[1], _ptr(cons), _ptr(metric), ctypes.byref(c),
                                          ctypes.byref(r), _stream_ptr(stream)), "grb_c2p_train")
        out = {k: getattr(r, k) for k, _ in abi.TrainReport._fields_}
        out["delta_cand"] = list(r.delta_cand)
        out["calib_ms"] = list(r.calib_ms)
        out["calib_cost"] = list(r.calib_cost)
        return out

    def c2p_model(self):
        """The model's parameter block (numpy float32 [MLP_NUM_PARAMS])."""
        import numpy as np
        P = np.zeros(abi.MLP_NUM_PARAMS, np.float32)
        _lib.check(self.lib.grb_c2p_model_get(self.h, P.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), P.size),
                   "grb_c2p_model_get")
        return P

    def set_c2p_model(self, P):
        import numpy as np
        P = np.ascontiguousarray(P, dtype=np.float32)
        _lib.check(self.lib.grb_c2p_model_set(self.h, P.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), P.size),
                   "grb_c2p_model_set")

    def c2p_features(self, cons, metric=None, mu=None, stream=None):
        n = cons.shape[1]
        feat = torch.empty(abi.MLP_IN, n, dtype=torch.float32, device=cons.device)
        tgt = torch.empty(n, dtype=torch.float32, device=cons.device)
        _lib.check(self.lib.grb_c2p_features(self.h, n, _ptr(cons), _ptr(metric), _ptr(mu), _ptr(feat), _ptr(tgt),
                                             _stream_ptr(stream)), "grb_c2p_features")
        return feat, tgt

    def mlp_eval(self, feat, params=None, stream=None):
        n = feat.shape[1]
        out = torch.empty(n, dtype=torch.float32, device=feat.device)
        _lib.check(self.lib.grb_mlp_eval(self.h, n, _ptr(params), _ptr(feat), _ptr(out), _stream_ptr(stream)),
                   "grb_mlp_eval")
        return out

    def mlp_grad(self, params, feat, tgt, stream=None):
        """(gradient [MLP_NUM_WEIGHTS], loss) of the batch MSE."""
        g = torch.empty(abi.MLP_NUM_WEIGHTS + 1, dtype=torch.float32, device=feat.device)
        _lib.check(self.lib.grb_mlp_grad(self.h, feat.shape[1], _ptr(params), _ptr(feat), _ptr(tgt), _ptr(g),
                                         _stream_ptr(stream)), "grb_mlp_grad")
        return g[:-1], float(g[-1])

    def set_mode(self, mode):
        """abi.MODE_PLAIN (reference launch ranges, one thread per item) or
        abi.MODE_TUNED (needed faces only, faster math, tuned variants)."""
        _lib.check(self.lib.grb_set_mode(self.h, mode), "grb_set_mode")

    def autotune(self, new_state, old_state, aux, stream=None):
        g = self.blocks.c()
        nf, of = new_state.c(), old_state.c()
        _lib.check(self.lib.grb_autotune(self.h, ctypes.byref(g), ctypes.byref(nf), ctypes.byref(of),
                                         _ptr(aux), _stream_ptr(stream)), "grb_autotune")
        return self.tuning()

    def tuning(self):
        v = (ctypes.c_int32 * 4)()
        ms = (ctypes.c_float * 12)()
        _lib.check(self.lib.grb_get_tuning(self.h, v, ms), "grb_get_tuning")
        fam = ["flux", "fofc_flag", "update", "aux"]
        out = {f: {"min_ctas_per_sm": v[i], "ms": [round(ms[3 * i + k], 4) for k in range(3)]}
               for i, f in enumerate(fam)}
        forms = (ctypes.c_float * 5)()
        _lib.check(self.lib.grb_get_tuning_forms(self.h, forms, 5), "grb_get_tuning_forms")
        r = lambda x: round(x, 4) if x < 1e29 else None
        out["fofc_flag"]["queue_ms"] = r(forms[0])
        out["aux"]["queue_ms"] = r(forms[1])
        out["aux"]["deferred_ms"] = r(forms[2])
        out["flux"]["queue_ms"] = r(forms[3])
        out["update"]["queue_ms"] = r(forms[4])
        return out

    def set_tuning(self, flux=0, flag=0, update=0, aux=0):
        """Pick tuned-mode candidates without timing (grb_set_tuning: indices
        0..2 grid launches, 3..5 their work-queue forms; aux 6..8 the
        deferred-backup form)."""
        v = (ctypes.c_int32 * 4)(flux, flag, update, aux)
        _lib.check(self.lib.grb_set_tuning(self.h, v), "grb_set_tuning")

    def fill_ghosts_gather(self, fields, maps, nvars=abi.N_HRSC, stream=None):
        """Ghost fill by gather maps (grb_fill_ghosts_gather).  maps: the dict
        of grace_b200.fmr.Hierarchy.gather_maps (numpy), or one run's part of
        it (gather_runs), uploaded on first use and kept by this object."""
        cache = self.__dict__.setdefault("_gmaps", {})
        key = id(maps)
        if key not in cache:
            dev = self.blocks.device
            up = lambda m: {k: torch.from_numpy(np.ascontiguousarray(m[k])).to(dev) for k in ("cnt", "dst", "src", "w")}
            # the maps object is kept with its upload, so its id stays its own
            cache[key] = (maps, {k: up(v) for k, v in maps.items()})
        G = cache[key][1]
        mk = lambda t: abi.Gather(t["dst"].numel(), t["cnt"].data_ptr(), t["dst"].data_ptr(), t["src"].data_ptr(),
                                  t["w"].data_ptr())
        cells = mk(G["cells"])
        faces = (abi.Gather * 3)(mk(G[0]), mk(G[1]), mk(G[2]))
        g = self.blocks.c()
        f = fields.c()
        _lib.check(self.lib.grb_fill_ghosts_gather(self.h, ctypes.byref(g), ctypes.byref(f), ctypes.byref(cells),
                                                   nvars, faces, _stream_ptr(stream)), "grb_fill_ghosts_gather")

    def set_reflux(self, lists=None, same_level_flux_average=False):
        """Reflux descriptor lists (grb_set_reflux): a dict of numpy arrays in
        the grb_reflux layout (grace_b200.fmr.Hierarchy.reflux_lists), copied
        to the device and kept by this object; None turns refluxing off."""
        if lists is None:
            _lib.check(self.lib.grb_set_reflux(self.h, None), "grb_set_reflux")
            self._reflux = None
            return
        dev = self.blocks.device
        d = {k: torch.from_numpy(v.copy()).to(dev) for k, v in lists.items()}
        self._reflux = d  # the library reads these arrays on every substep
        P = lambda k: d[k].data_ptr() if d[k].numel() else None
        r = abi.Reflux(len(d["face_coarse_q"]), P("face_coarse_q"), P("face_coarse_id"), P("face_fine_q"),
                       len(d["same_face_q"]) // 2, P("same_face_q"), P("same_face_id"),
                       1 if same_level_flux_average else 0,
                       len(d["edge_nsides"]), P("edge_nsides"), P("edge_id"), P("edge_is_fine"), P("edge_q"),
                       P("edge_off"),
                       len(d["same_edge_nsides"]), P("same_edge_nsides"), P("same_edge_id"), P("same_edge_q"))
        _lib.check(self.lib.grb_set_reflux(self.h, ctypes.byref(r)), "grb_set_reflux")

    def set_fofc_list_capacity(self, faces):
        """Capacity of the compacted FOFC face list of the tuned stage
        (grb_set_fofc_list_capacity); 0 forces the whole-box recompute."""
        _lib.check(self.lib.grb_set_fofc_list_capacity(self.h, int(faces)), "grb_set_fofc_list_capacity")

    def set_kernel_timing(self, on):
        _lib.check(self.lib.grb_set_kernel_timing(self.h, 1 if on else 0), "grb_set_kernel_timing")

    def kernel_times(self):
        """{kind: (ms, launch groups)} accumulated since the last call."""
        n = len(abi.KIND_NAMES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int64 * n)()
        _lib.check(self.lib.grb_kernel_times(self.h, ms, cnt, n), "grb_kernel_times")
        return {abi.KIND_NAMES[k]: (ms[k], cnt[k]) for k in range(n)}

    def status(self):
        st = abi.Status()
        _lib.check(self.lib.grb_get_status(self.h, ctypes.byref(st)), "grb_get_status")
        return st

    # --- evolve_impl<eos_t>() RK3 branch (evolve.cpp:147-225, 427-428) -----
    def rk3_step(self, dt, state, state_p, state_pp, aux, bc, t=0.0, stream=None, next_dt=None,
                 fused_dt=False, after_update=None):
        """One SSP-RK3 step.  `bc(fields)` applies the boundary conditions
        (GRACE's amr::apply_boundary_conditions); on entry aux holds the
        primitives of `state` and state_p equals state.  next_dt = (dx, cfl,
        dt_out): the step ends with find_stable_timestep into dt_out, as a
        separate pass after the last aux pass or, with fused_dt, inside it.
        after_update(): called (host side, stream order) right after the last
        substep, when the interior face B of `state` is final (the boundary
        fill and the aux pass that follow change only ghosts and cell
        variables)."""
        self.reset_c2p_diagnostics(aux, stream)
        self.advance_substep(t, dt, 1.0, state_p, state, aux, stream)
        bc(state_p)
        self.compute_auxiliary_quantities(state_p, aux, stream)
        self.linop_apply(state_pp, state, state_p, 0.75, 0.25, stream)
        self.advance_substep(t, dt, 0.25, state_pp, state_p, aux, stream)
        bc(state_pp)
        self.compute_auxiliary_quantities(state_pp, aux, stream)
        self.linop_apply(state, state, state_pp, 1.0 / 3, 2.0 / 3.0, stream)
        self.advance_substep(t, dt, 2.0 / 3.0, state, state_pp, aux, stream)
        if after_update is not None:
            after_update()
        bc(state)
        if next_dt is not None and fused_dt:
            self.compute_auxiliary_quantities_dt(state, aux, *next_dt, stream=stream)
        else:
            self.compute_auxiliary_quantities(state, aux, stream)
            if next_dt is not None:
                self.find_stable_timestep(state, aux, *next_dt, stream=stream)
        self.linop_apply(state_p, state, None, 1.0, 0.0, stream)

    # --- the other explicit branches of evolve_impl (evolve.cpp:173-332) ---
    # Same entry condition as rk3_step (aux holds the primitives of state,
    # state_p equals state: GRACE copies it at the start of every step,
    # evolve.cpp:147) and the same exit (state_p set to the new state).

    def euler_step(self, dt, state, state_p, aux, bc, t=0.0, stream=None):
        """Forward Euler (evolve.cpp:173-178): state += dt L(state_p)."""
        self.reset_c2p_diagnostics(aux, stream)
        self.advance_substep(t, dt, 1.0, state, state_p, aux, stream)
        bc(state)
        self.compute_auxiliary_quantities(state, aux, stream)
        self.linop_apply(state_p, state, None, 1.0, 0.0, stream)

    def rk2_step(self, dt, state, state_p, aux, bc, t=0.0, stream=None):
        """Midpoint RK2 (evolve.cpp:179-189): state_p += dt/2 L(state), then
        state += dt L(state_p)."""
        self.reset_c2p_diagnostics(aux, stream)
        self.advance_substep(t, dt, 0.5, state_p, state, aux, stream)
        bc(state_p)
        self.compute_auxiliary_quantities(state_p, aux, stream)
        self.advance_substep(t, dt, 1.0, state, state_p, aux, stream)
        bc(state)
        self.compute_auxiliary_quantities(state, aux, stream)
        self.linop_apply(state_p, state, None, 1.0, 0.0, stream)

    # four-stage low-storage coefficients (delta, gamma1, gamma2, beta) of the
    # reference's rk4 branch, stage by stage (evolve.cpp:226-332)
    RK4_COEFFS = ((1.0, 0.0, 1.0, 1.193743905974738),
                  (0.217683334308543, 0.121098479554482, 0.721781678111411, 0.099279895495783),
                  (1.065841341361089, -3.843833699660025, 2.121209265338722, 1.131678018054042),
                  (0.0, 0.546370891121863, 0.198653035682705, 0.310665766509336))

    def rk4_step(self, dt, state, state_p, stage, aux, bc, t=0.0, stream=None):
        """The rk4 branch of evolve_impl (evolve.cpp:226-332): four stages of
        a low-storage scheme over state (s1), state_p (s2) and a staging
        buffer `stage` (s3, any Fields of the same shape holding the static
        metric), each a two-term linop_apply or two, advance_substep with
        dtfact = beta, the boundary fill and the primitives pass."""
        s1, s2, s3 = state, state_p, stage
        (d1, g11, g21, b1), (d2, g12, g22, b2), (d3, g13, g23, b3), (d4, g14, g24, b4) = self.RK4_COEFFS
        self.reset_c2p_diagnostics(aux, stream)
        # stage 1: s3 = gamma1 s1 + gamma2 s2; s3 += beta dt F(s1)
        self.linop_apply(s3, s1, s2, g11, g21, stream)
        self.advance_substep(t, dt, b1, s3, s1, aux, stream)
        bc(s3)
        self.compute_auxiliary_quantities(s3, aux, stream)
        # stage 2: s2 += delta s3; s1 = gamma1 s3 + gamma2 s2; s1 += beta dt F(s3)
        self.linop_apply(s2, s2, s3, 1.0, d2, stream)
        self.linop_apply(s1, s3, s2, g12, g22, stream)
        self.advance_substep(t, dt, b2, s1, s3, aux, stream)
        bc(s1)
        self.compute_auxiliary_quantities(s1, aux, stream)
        # stage 3: s2 += delta s1; s3 = gamma1 s1 + gamma2 s2; s3 += beta dt F(s1)
        self.linop_apply(s2, s2, s1, 1.0, d3, stream)
        self.linop_apply(s3, s1, s2, g13, g23, stream)
        self.advance_substep(t, dt, b3, s3, s1, aux, stream)
        bc(s3)
        self.compute_auxiliary_quantities(s3, aux, stream)
        # stage 4 (delta = 0: no s2 update): s1 = gamma1 s3 + gamma2 s2; s1 += beta dt F(s3)
        self.linop_apply(s1, s3, s2, g14, g24, stream)
        self.advance_substep(t, dt, b4, s1, s3, aux, stream)
        bc(s1)
        self.compute_auxiliary_quantities(s1, aux, stream)
        self.linop_apply(state_p, state, None, 1.0, 0.0, stream)

    def rk3_step_host(self, dt, host, state, state_p, state_pp, aux, bc, runs, fill_run, deps, t=0.0,
                      streams=None, after=None, wait=True, whole_grid_substeps=False):
        """One SSP-RK3 step of a state held in packed pinned host arrays
        (packed_host_fields): upload, boundary fill and primitives of the
        uploaded state, the step, download — the same kernels in the same
        per-block order as

            copy_evolved_packed(host, state, True); bc(state);
            compute_auxiliary_quantities(state, aux);
            linop_apply(state_p, state, None, 1.0); rk3_step(...);
            copy_evolved_packed(host, state, False)

        (state_p is set to the state whose primitives were just computed:
        rk3_step's entry condition), so the same bits, but pipelined
        over runs of blocks on three streams: the upload of each run overlaps
        the first substep of the runs before it, the download of each run
        the last substep of the runs after it.

        runs: [(q0, q1)] consecutive runs covering [0, nq).
        fill_run(fields, s, stream): the boundary fill of the ghost zones of
        run s alone; deps[s]: the runs whose interiors it reads (brick_runs
        gives both for a brick).
        bc(fields): the fill of every block (the middle substep).
        streams: (upload, download) CUDA streams, new ones by default; the
        caller's current stream runs the kernels.  On return (stream order)
        host holds the new interior and state, state_p, aux on the device
        are as after rk3_step.

        Consecutive steps: wait=False leaves the downloads pending (the
        caller's stream does not wait for them) and returns one event per
        run, recorded when its download is done; passed as `after` to the
        next call (same arrays and streams, nothing else touching them in
        between), each run's upload waits for that run's download only, so
        the uploads of a step overlap the last substep of the step before.
        The caller's stream waits for the download stream before it reads
        host.

        whole_grid_substeps=True (refluxing: its corrections couple blocks of
        different runs): the first and last substeps run on the whole grid
        too; the uploads then overlap the fills and primitives passes of the
        runs before them, the downloads the primitives passes of the runs
        after them (gather_runs gives runs, fill maps and deps for an FMR
        hierarchy)."""
        main = torch.cuda.current_stream()
        up, down = streams if streams is not None else (torch.cuda.Stream(), torch.cuda.Stream())
        S = len(runs)
        if after is not None and len(after) != S:
            raise ValueError("after: one event per run of the previous step")
        deps = [set(d) | {s} for s, d in enumerate(deps)]
        # readers[r]: the runs whose ghost fill reads run r's interior.  A
        # run's primitives pass may write corrected conserved variables
        # back into its interior, so it waits until those fills are done
        # (as the whole-grid order fills every block before any primitives).
        readers = [{t for t in range(S) if r in deps[t]} for r in range(S)]
        # the uploads read host arrays the previous step's downloads wrote,
        # into device blocks the previous step has finished with
        if after is None:
            up.wait_stream(main)
            up.wait_stream(down)
        ev_up = []
        for r, (q0, q1) in enumerate(runs):
            if after is not None:
                up.wait_event(after[r])
            with self.block_range(q0, q1):
                self.copy_evolved_packed(host.view(q0, q1), state.view(q0, q1), True, stream=up)
            e = torch.cuda.Event()
            e.record(up)
            ev_up.append(e)
        # first substep, run by run as the runs they read arrive
        filled, ready = set(), set()
        for s in range(S):
            for d in sorted(deps[s]):
                main.wait_event(ev_up[d])
            fill_run(state, s, main)
            filled.add(s)
            for r, (q0, q1) in enumerate(runs):
                if r in ready or not readers[r] <= filled:
                    continue
                with self.block_range(q0, q1):
                    sv, pv, a = state.view(q0, q1), state_p.view(q0, q1), aux[q0:q1]
                    self.compute_auxiliary_quantities(sv, a, main)
                    self.reset_c2p_diagnostics(a, main)
                    self.linop_apply(pv, sv, None, 1.0, 0.0, main)
                    if not whole_grid_substeps:
                        self.advance_substep(t, dt, 1.0, pv, sv, a, main)
                ready.add(r)
        if whole_grid_substeps:
            self.advance_substep(t, dt, 1.0, state_p, state, aux, main)
        # middle substep on the whole grid
        bc(state_p)
        self.compute_auxiliary_quantities(state_p, aux, main)
        self.linop_apply(state_pp, state, state_p, 0.75, 0.25, main)
        self.advance_substep(t, dt, 0.25, state_pp, state_p, aux, main)
        bc(state_pp)
        self.compute_auxiliary_quantities(state_pp, aux, main)
        self.linop_apply(state, state, state_pp, 1.0 / 3, 2.0 / 3.0, main)
        # last substep run by run; a run is filled once the runs it reads
        # are updated, and finished (primitives, state_p) and downloaded
        # once the runs reading it are filled
        updated, filled, finished = set(), set(), set()
        ev_down = [None] * S
        if whole_grid_substeps:
            self.advance_substep(t, dt, 2.0 / 3.0, state, state_pp, aux, main)
            updated = set(range(S))
        for s, (q0, q1) in enumerate(runs):
            if not whole_grid_substeps:
                with self.block_range(q0, q1):
                    self.advance_substep(t, dt, 2.0 / 3.0, state.view(q0, q1), state_pp.view(q0, q1), aux[q0:q1],
                                         main)
            updated.add(s)
            for r in range(S):
                if r not in filled and deps[r] <= updated:
                    fill_run(state, r, main)
                    filled.add(r)
            for r, (r0, r1) in enumerate(runs):
                if r in finished or r not in filled or not readers[r] <= filled:
                    continue
                with self.block_range(r0, r1):
                    sv = state.view(r0, r1)
                    self.compute_auxiliary_quantities(sv, aux[r0:r1], main)
                    self.linop_apply(state_p.view(r0, r1), sv, None, 1.0, 0.0, main)
                e = torch.cuda.Event()
                e.record(main)
                down.wait_event(e)
                with self.block_range(r0, r1):
                    self.copy_evolved_packed(host.view(r0, r1), state.view(r0, r1), False, stream=down)
                ev_down[r] = torch.cuda.Event()
                ev_down[r].record(down)
                finished.add(r)
        if len(ready) != S or len(finished) != S:
            raise ValueError("runs / deps do not cover every run")
        main.wait_stream(up)
        if wait:
            main.wait_stream(down)
        return ev_down

    def capture_rk3_step(self, dt, state, state_p, state_pp, aux, bc, t=0.0, next_dt=None, fused_dt=False):
        """Capture one rk3_step (same arguments) into a CUDA graph.  The
        arrays and dt are baked into the graph: each graph.replay() advances
        the same arrays by one step with no host work per kernel.  Call after
        at least one eager step (first-call set-up such as shared-memory
        attributes and autotuning happens outside the capture).  Returns
        (graph, kernels launched per replay)."""
        n0 = self.status().launches
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.rk3_step(dt, state, state_p, state_pp, aux, bc, t, next_dt=next_dt, fused_dt=fused_dt)
        return graph, self.status().launches - n0
