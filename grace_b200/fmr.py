"""Static FMR hierarchies of cubic blocks on the host (numpy): the leaf
blocks of nested refinement, their spacings and coordinates, and the reflux
descriptor lists the library's grb_set_reflux takes.

This stands in, on one rank, for what GRACE's host side derives from its
p4est forest: the leaves (quadrants) of every level, and the reflux face and
edge descriptors its face and edge iterators collect
(src/amr/ghost_helpers/iterate_faces.cpp:150-280, iterate_edges.cpp:330-407,
include/grace/amr/amr_ghosts.hh:190-330), found here by geometry on the
integer lattice of the finest level.  It also carries a composite ghost fill
for tests and benchmarks of multi-level block lists: every ghost cell takes
the value of the leaf data at its place (a copy from a same-level leaf, the
containing coarser cell, or the 8-cell average of the finer cells; face B
likewise with faces), which keeps same-level ghosts bitwise consistent.  The
fill is a host harness, not GRACE's prolongation.

Conventions: face id = 2 axis + side (side 1 the upper face); edge id =
4 axis + s_a + 2 s_b (p4est's), s_a, s_b the sides along the edge's other
two axes in x, y, z order.  Block q's arrays follow the library's layout.
"""
import itertools

import numpy as np

from . import abi

ODIR = ((1, 2), (0, 2), (0, 1))  # the two axes orthogonal to an axis
# coarse face -> the coarse edge ids of its two middle lines
# (iterate_faces.cpp:205-212) and p4est's face -> edge table (index_helpers.hh:587-595)
FACE_COARSE_EDGES = ((4, 8), (5, 9), (0, 8), (1, 10), (0, 4), (2, 6))
F2E = ((8, 10, 4, 6), (9, 11, 5, 7), (8, 9, 0, 2), (10, 11, 1, 3), (4, 5, 0, 1), (6, 7, 2, 3))


class Hierarchy:
    """Leaves of a nested refinement of a brick of cubic blocks.

    nb0: base-level blocks per axis; n: cells per block side; lo, hi: domain
    corners; refine(level, b): True to split base-or-finer block b (integer
    block coordinates at its level) into 8 children, up to max_level;
    periodic: per axis.  Leaves are ordered by level, then z, y, x."""

    def __init__(self, nb0, n, lo, hi, refine, max_level, periodic=(True, True, True), ngz=4):
        self.nb0 = tuple(int(x) for x in nb0)
        self.n, self.ngz, self.L = int(n), int(ngz), int(max_level)
        self.lo, self.hi = np.asarray(lo, float), np.asarray(hi, float)
        self.periodic = tuple(bool(p) for p in periodic)
        leaves = []

        def walk(l, b):
            if l < self.L and refine(l, b):
                for c in itertools.product((0, 1), repeat=3):
                    walk(l + 1, (2 * b[0] + c[2], 2 * b[1] + c[1], 2 * b[2] + c[0]))
            else:
                leaves.append((l, b))

        for bz in range(self.nb0[2]):
            for by in range(self.nb0[1]):
                for bx in range(self.nb0[0]):
                    walk(0, (bx, by, bz))
        # finest-cell lattice: a level-l block spans E(l) finest cells
        self.N = tuple(self.nb0[a] * self.n * 2 ** self.L for a in range(3))
        self._set_leaves(leaves)
        self._balance()
        self._check_balance()

    def _set_leaves(self, leaves):
        leaves = sorted(leaves, key=lambda t: (t[0], t[1][2], t[1][1], t[1][0]))
        self.leaves = leaves
        self.index = {t: q for q, t in enumerate(leaves)}
        self.nq = len(leaves)

    def _balance(self):
        """Refine leaves until every face, edge and corner neighbour is at
        most one level finer (p4est's 2:1 balance)."""
        while True:
            split = set()
            for l, b in self.leaves:
                E = self.E(l)
                for d in itertools.product((-1, 0, 1), repeat=3):
                    if d == (0, 0, 0):
                        continue
                    # probe the neighbour region at the finest spacing along its boundary
                    for u in range(0, E, max(1, E // 4)):
                        p = [b[a] * E + (E if d[a] > 0 else (-1 if d[a] < 0 else u)) for a in range(3)]
                        t = self.leaf_at(p)
                        if t is not None and t[0] - l > 1:
                            split.add((l, b))
                            break
                    if (l, b) in split:
                        break
            if not split:
                return
            leaves = [t for t in self.leaves if t not in split]
            for l, b in split:
                for c in itertools.product((0, 1), repeat=3):
                    leaves.append((l + 1, (2 * b[0] + c[2], 2 * b[1] + c[1], 2 * b[2] + c[0])))
            self._set_leaves(leaves)

    # ---- geometry ---------------------------------------------------------
    def E(self, l):
        return self.n * 2 ** (self.L - l)

    def dx(self, l):
        return (self.hi - self.lo) / (np.asarray(self.nb0) * self.n * 2 ** l)

    def idx(self):
        return np.stack([1.0 / self.dx(l) for l, _ in self.leaves])

    def spacings(self):
        return np.stack([self.dx(l) for l, _ in self.leaves])

    def level_counts(self):
        return np.bincount([l for l, _ in self.leaves], minlength=self.L + 1)

    def coords(self):
        """Centre of cell (0,0,0) (a ghost cell) of every block."""
        out = []
        for l, b in self.leaves:
            d = self.dx(l)
            out.append(self.lo + (np.asarray(b) * self.n + 0.5 - self.ngz) * d)
        return np.stack(out)

    def cell_centres(self):
        """(nq, 3, NZ, NY, NX) physical cell centres, ghosts included."""
        NN = self.n + 2 * self.ngz
        r = np.arange(NN)
        out = np.empty((self.nq, 3, NN, NN, NN))
        for q, (l, b) in enumerate(self.leaves):
            d = self.dx(l)
            o = self.lo + np.asarray(b) * self.n * d
            out[q, 0] = o[0] + (r[None, None, :] - self.ngz + 0.5) * d[0]
            out[q, 1] = o[1] + (r[None, :, None] - self.ngz + 0.5) * d[1]
            out[q, 2] = o[2] + (r[:, None, None] - self.ngz + 0.5) * d[2]
        return out

    def wrap(self, p):
        """Finest-lattice point p wrapped on periodic axes; None outside."""
        out = []
        for a in range(3):
            x = p[a]
            if self.periodic[a]:
                x %= self.N[a]
            elif x < 0 or x >= self.N[a]:
                return None
            out.append(x)
        return tuple(out)

    def leaf_at(self, p):
        """(level, block) of the leaf containing finest-lattice point p."""
        w = self.wrap(p)
        if w is None:
            return None
        for l in range(self.L, -1, -1):
            E = self.E(l)
            t = (l, (w[0] // E, w[1] // E, w[2] // E))
            if t in self.index:
                return t
        raise AssertionError("lattice point not covered by a leaf")

    def _check_balance(self):
        """2:1 balance across faces, edges and corners (as p4est keeps it)."""
        for l, b in self.leaves:
            E = self.E(l)
            for d in itertools.product((-1, 0, 1), repeat=3):
                if d == (0, 0, 0):
                    continue
                for u in range(0, E, max(1, E // 4)):
                    p = [b[a] * E + (E if d[a] > 0 else (-1 if d[a] < 0 else u)) for a in range(3)]
                    t = self.leaf_at(p)
                    if t is not None:
                        assert abs(t[0] - l) <= 1, f"hierarchy not 2:1 balanced at level {l} block {b}"

    # ---- reflux descriptors -------------------------------------------------
    def reflux_lists(self):
        """The grb_reflux lists as numpy arrays (dict of the struct's fields)."""
        hf_cq, hf_cid, hf_fq = [], [], []
        sf_q, sf_id, seen_faces = [], [], set()
        for q, (l, b) in enumerate(self.leaves):
            E = self.E(l)
            for face in range(6):
                a, side = face // 2, face & 1
                # a point just across the face, at the face's lowest corner
                p = [b[k] * E for k in range(3)]
                p[a] = (b[a] + 1) * E if side else b[a] * E - 1
                t = self.leaf_at(p)
                if t is None:
                    continue
                if t[0] == l:
                    key = (a, self.wrap([b[k] * E + (E if (k == a and side) else 0) for k in range(3)]))
                    if key in seen_faces:
                        continue
                    seen_faces.add(key)
                    sf_q += [q, self.index[t]]
                    sf_id += [face, face ^ 1]
                elif t[0] == l + 1:
                    # hanging face: the 4 finer blocks across it, c = a' + 2 b'
                    h = E // 2
                    fq = []
                    for c in range(4):
                        pp = list(p)
                        pp[ODIR[a][0]] += (c & 1) * h
                        pp[ODIR[a][1]] += (c >> 1) * h
                        fq.append(self.index[self.leaf_at(pp)])
                    hf_cq.append(q)
                    hf_cid.append(face)
                    hf_fq += fq
        e_ns, e_id, e_fine, e_q, e_off = [], [], [], [], []
        se_ns, se_id, se_q = [], [], []
        seen_edges = set()
        for q, (l, b) in enumerate(self.leaves):
            E = self.E(l)
            for eid in range(12):
                a = eid // 4
                o1, o2 = ODIR[a]
                x1 = (b[o1] + (eid & 1)) * E
                x2 = (b[o2] + ((eid >> 1) & 1)) * E
                start = b[a] * E
                sides = []
                ok, coarser = True, False
                for pj in (0, 1):
                    for pi in (0, 1):
                        p = [0, 0, 0]
                        p[a] = start
                        p[o1] = x1 if pi else x1 - 1
                        p[o2] = x2 if pj else x2 - 1
                        t = self.leaf_at(p)
                        if t is None:
                            continue
                        Et = self.E(t[0])
                        wp = self.wrap(p)
                        # the line must lie on that leaf's edge
                        if Et > E:
                            coarser = True
                            on1 = (wp[o1] + (0 if pi else 1)) % Et == 0
                            on2 = (wp[o2] + (0 if pj else 1)) % Et == 0
                            if not (on1 and on2):
                                ok = False
                        sides.append((pi, pj, t, p))
                if not ok or coarser:
                    continue
                key = (a, self.wrap([x1 if k == o1 else x2 if k == o2 else start for k in range(3)]))
                if key in seen_edges:
                    continue
                seen_edges.add(key)
                fine_sides = [s for s in sides if s[2][0] == l + 1]
                rec_id, rec_fine, rec_q, rec_off = [], [], [], []
                for pi, pj, t, p in sides:
                    sid = 4 * a + (1 - pi) + 2 * (1 - pj)
                    rec_id.append(sid)
                    if t[0] == l + 1:
                        pp = list(p)
                        pp[a] += E // 2
                        rec_fine.append(1)
                        rec_q += [self.index[t], self.index[self.leaf_at(pp)]]
                    else:
                        rec_fine.append(0)
                        rec_q += [self.index[t], self.index[t]]
                    rec_off += [0, 0]
                pad = 4 - len(sides)
                if fine_sides:
                    e_ns.append(len(sides))
                    e_id += rec_id + [0] * pad
                    e_fine += rec_fine + [0] * pad
                    e_q += rec_q + [0] * (2 * pad)
                    e_off += rec_off + [0] * (2 * pad)
                else:
                    se_ns.append(len(sides))
                    se_id += rec_id + [0] * pad
                    se_q += rec_q[0::2] + [0] * pad
        # the middle lines of every hanging face (iterate_faces.cpp:197-280)
        for i, (qc, face) in enumerate(zip(hf_cq, hf_cid)):
            fdir = face // 2
            fq = hf_fq[4 * i:4 * i + 4]
            for idir in (0, 1):
                edir = ODIR[fdir][idir]
                rec_id = [FACE_COARSE_EDGES[face][idir]]
                rec_fine = [0]
                rec_q = [qc, qc]
                rec_off = [int(fdir == ODIR[edir][1]), int(fdir == ODIR[edir][0])]
                for iside in (0, 1):
                    rec_id.append(F2E[face ^ 1][2 * (1 - idir) + (1 - iside)])
                    rec_fine.append(1)
                    for ich2 in (0, 1):
                        ich = ich2 + 2 * iside if idir == 0 else iside + 2 * ich2
                        rec_q.append(fq[ich])
                    rec_off += [0, 0]
                e_ns.append(3)
                e_id += rec_id + [0]
                e_fine += rec_fine + [0]
                e_q += rec_q + [0, 0]
                e_off += rec_off + [0, 0]
        a64 = lambda x: np.asarray(x, dtype=np.int64)
        u8 = lambda x: np.asarray(x, dtype=np.uint8)
        return {"face_coarse_q": a64(hf_cq), "face_coarse_id": u8(hf_cid), "face_fine_q": a64(hf_fq),
                "same_face_q": a64(sf_q), "same_face_id": u8(sf_id),
                "edge_nsides": u8(e_ns), "edge_id": u8(e_id), "edge_is_fine": u8(e_fine), "edge_q": a64(e_q),
                "edge_off": u8(e_off),
                "same_edge_nsides": u8(se_ns), "same_edge_id": u8(se_id), "same_edge_q": a64(se_q)}

    # ---- composite ghost fill ------------------------------------------------
    def _lookup(self, P):
        """Vectorised leaf_at over finest-lattice points P (m, 3) already
        inside the domain: (level, qindex) arrays."""
        lev = np.full(len(P), -1, dtype=np.int64)
        qi = np.full(len(P), -1, dtype=np.int64)
        if not hasattr(self, "_level_keys"):
            self._level_keys = {}
            for l in range(self.L + 1):
                nbl = [self.nb0[a] * 2 ** l for a in range(3)]
                mine = [(b, q) for q, (ll, b) in enumerate(self.leaves) if ll == l]
                keys = np.array([(b[2] * nbl[1] + b[1]) * nbl[0] + b[0] for b, _ in mine], dtype=np.int64)
                qs = np.array([q for _, q in mine], dtype=np.int64)
                order = np.argsort(keys)
                self._level_keys[l] = (keys[order], qs[order], nbl)
        for l in range(self.L, -1, -1):
            keys, qs, nbl = self._level_keys[l]
            if len(keys) == 0:
                continue
            E = self.E(l)
            todo = lev < 0
            B = P[todo] // E
            k = (B[:, 2] * nbl[1] + B[:, 1]) * nbl[0] + B[:, 0]
            pos = np.clip(np.searchsorted(keys, k), 0, len(keys) - 1)
            hit = keys[pos] == k
            idx = np.flatnonzero(todo)[hit]
            lev[idx] = l
            qi[idx] = qs[pos[hit]]
        assert np.all(lev >= 0)
        return lev, qi

    def _domain(self, P, s):
        """Wrap periodic axes; on the others move a point outside the domain
        to the nearest cell centre of its own spacing s inside it (a ghost
        cell beyond a non-periodic boundary takes the data of the nearest
        leaf region of its size: zero-gradient), so that the region of size
        s around it stays inside the domain."""
        P = P.copy()
        for a in range(3):
            if self.periodic[a]:
                P[:, a] %= self.N[a]
            else:
                P[:, a] = np.clip(P[:, a], s // 2, self.N[a] - s // 2)
        return P

    def gather_maps(self):
        """Ghost-fill gather maps for the cells (key "cells") and the face
        arrays staggered along x, y, z (keys 0, 1, 2), each a dict in the
        format of grb_gather: cnt (m,) used slots, dst (m,) element offsets of
        variable 0, src (8, m) and w (8, m) slot-major, vstride the offset
        between variables.  A ghost cell takes the
        leaf data at its place: a copy from a same-level cell, the containing
        coarser cell, or the mean of the 8 finer cells; a ghost face a copy,
        the coarser face it lies on (or the linear interpolation between the
        two coarser faces around it), or the mean of the 4 finer faces."""
        if hasattr(self, "_gmaps"):
            return self._gmaps
        n, g = self.n, self.ngz
        NN = n + 2 * g
        lv = np.array([l for l, _ in self.leaves], dtype=np.int64)
        bb = np.array([b for _, b in self.leaves], dtype=np.int64)
        out = {}
        for arr in ("cells", 0, 1, 2):
            shp = [NN, NN, NN]
            if arr != "cells":
                shp[arr] += 1  # extent along the staggered axis (x, y, z order)
            per = shp[0] * shp[1] * shp[2]
            K, J, I = np.meshgrid(np.arange(shp[2]), np.arange(shp[1]), np.arange(shp[0]), indexing="ij")
            c = [I.ravel(), J.ravel(), K.ravel()]
            gh = np.zeros(per, bool)
            for a in range(3):
                hi = n + g + (1 if arr == a else 0)
                gh |= (c[a] < g) | (c[a] >= hi)
            loc = np.flatnonzero(gh)
            cl = [x[loc] for x in c]
            Q = np.repeat(np.arange(self.nq), len(loc))
            s = (np.array([self.E(l) for l in lv]) // n)[Q]
            P = np.empty((len(Q), 3), dtype=np.int64)
            for a in range(3):
                ca = np.tile(cl[a], self.nq)
                if arr == a:
                    P[:, a] = (bb[Q, a] * n + ca - g) * s
                else:
                    P[:, a] = (bb[Q, a] * n + ca - g) * s + s // 2
            dst = Q * per + np.tile(loc, self.nq)
            if arr == "cells":
                W = self._domain(P, s)
                tl, tq = self._lookup(W)
                st = (np.array([self.E(l) for l in range(self.L + 1)]) // n)[tl]
                base_b = bb[tq]
                src = np.zeros((len(Q), 8), dtype=np.int64)
                w = np.zeros((len(Q), 8))
                finer = st < s
                li = lambda pts, a: pts[:, a] // st - base_b[:, a] * n + g
                flat = lambda i, j, k: tq * per + (k * NN + j) * NN + i
                f0 = flat(li(W, 0), li(W, 1), li(W, 2))
                src[:] = f0[:, None]
                w[:, 0] = np.where(finer, 0.125, 1.0)
                for t_ in range(1, 8):
                    off = np.array([t_ & 1, (t_ >> 1) & 1, t_ >> 2])
                    Pc = W - (s // 2)[:, None] + off[None, :] * st[:, None]
                    Pb = W - (s // 2)[:, None]
                    f = flat(li(Pc, 0), li(Pc, 1), li(Pc, 2))
                    src[finer, t_] = f[finer]
                    w[finer, t_] = 0.125
                # the finer case's first source is the (0,0,0) finer cell
                fb = flat(li(Pb, 0), li(Pb, 1), li(Pb, 2))
                src[finer, 0] = fb[finer]
            else:
                d = arr
                W = P.copy()
                top = np.zeros(len(W), bool)
                for a in range(3):
                    if self.periodic[a]:
                        W[:, a] %= self.N[a]
                    elif a == d:
                        top = W[:, a] >= self.N[a]
                        W[:, a] = np.clip(W[:, a], 0, self.N[a])
                    else:
                        W[:, a] = np.clip(W[:, a], s // 2, self.N[a] - s // 2)
                Wl = W.copy()
                Wl[top, d] -= 1  # the cell below a face on the upper boundary
                tl, tq = self._lookup(Wl)
                st = (np.array([self.E(l) for l in range(self.L + 1)]) // n)[tl]
                base_b = bb[tq]
                fd = W[:, d] - base_b[:, d] * n * st
                lo_f = fd // st
                frac = (fd - lo_f * st) / st
                o1, o2 = ODIR[d]

                def flatf(i3):
                    ext = list(shp)
                    return tq * per + (i3[2] * ext[1] + i3[1]) * ext[0] + i3[0]

                i3 = [None] * 3
                i3[d] = lo_f + g
                for a in (o1, o2):
                    i3[a] = W[:, a] // st - base_b[:, a] * n + g
                f0 = flatf(i3)
                src = np.repeat(f0[:, None], 8, axis=1)
                w = np.zeros((len(Q), 8))
                w[:, 0] = 1.0
                interp = (st > s) & (frac > 0)
                j3 = list(i3)
                j3[d] = lo_f + g + 1
                f1 = flatf(j3)
                w[interp, 0] = 1.0 - frac[interp]
                src[interp, 1] = f1[interp]
                w[interp, 1] = frac[interp]
                finer = st < s
                for t_ in range(4):
                    k3 = [None] * 3
                    k3[d] = lo_f + g
                    for u, a in enumerate((o1, o2)):
                        pa = W[:, a] - s // 2 + (((t_ >> u) & 1) * st)
                        k3[a] = pa // st - base_b[:, a] * n + g
                    fk = flatf(k3)
                    src[finer, t_] = fk[finer]
                    w[finer, t_] = 0.25
            out[arr] = self._pack(arr, dst, src, w, per)
        self._gmaps = out
        return out

    @staticmethod
    def _pack(arr, dst, src, w, per):
        """The maps in the library's format (grb_gather): element offsets of
        variable 0 of the target array (the state holds N_EVOL_VARS
        variables per block), slot-major sources and weights, the number of
        used slots per entry."""
        def off(f):
            if arr != "cells":
                return f
            return (f // per) * (abi.N_EVOL_VARS * per) + f % per
        cnt = np.maximum(1, np.sum(w != 0.0, axis=1)).astype(np.int8)
        # used slots first (they are, by construction), unused ones weight 0
        return {"cnt": cnt, "dst": off(dst), "src": np.ascontiguousarray(off(src).T),
                "w": np.ascontiguousarray(w.T), "vstride": per}

    @staticmethod
    def _apply(flat, m, v):
        """One map on variable v of a flat array: w0 v0 + w1 v1 + ... over
        the used slots, accumulated in slot order, one product and one sum
        rounded at a time (as grb_fill_ghosts_gather does)."""
        o = v * m["vstride"]
        src, w, cnt = m["src"], m["w"], m["cnt"]
        acc = w[0] * flat[src[0] + o]
        for k in range(1, 8):
            use = cnt > k
            if not np.any(use):
                break
            acc = np.where(use, acc + w[k] * flat[np.where(use, src[k], src[0]) + o], acc)
        flat[m["dst"] + o] = acc

    def fill_ghosts(self, state, bx, by, bz, nvars=abi.N_HRSC):
        """Composite ghost fill of the first nvars state variables and face B
        (host numpy arrays in the library layout), in place, with the maps of
        gather_maps (the device fill, grb_fill_ghosts_gather, gives the same
        bits).  Sources are interior cells and faces only."""
        M = self.gather_maps()
        flat = state.reshape(-1)
        for v in range(nvars):
            self._apply(flat, M["cells"], v)
        for d, arr in enumerate((bx, by, bz)):
            self._apply(arr.reshape(-1), M[d], 0)
