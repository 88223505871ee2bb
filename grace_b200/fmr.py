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
        leaves.sort(key=lambda t: (t[0], t[1][2], t[1][1], t[1][0]))
        self.leaves = leaves
        self.index = {t: q for q, t in enumerate(leaves)}
        self.nq = len(leaves)
        # finest-cell lattice: a level-l block spans E(l) finest cells
        self.N = tuple(self.nb0[a] * self.n * 2 ** self.L for a in range(3))
        self._check_balance()

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
                p = [b[a] * E + (E if d[a] > 0 else (-1 if d[a] < 0 else E // 2)) for a in range(3)]
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

    # ---- composite ghost fill (host harness) ---------------------------------
    def _maps(self):
        """Per block: for every cell of the ghosted block a gather recipe
        (source block, flat source cell indices, weight), built once."""
        if hasattr(self, "_cell_maps"):
            return self._cell_maps, self._face_maps
        n, g = self.n, self.ngz
        NN = n + 2 * g
        self._cell_maps = []
        self._face_maps = [[], [], []]
        r = np.arange(NN)
        for q, (l, b) in enumerate(self.leaves):
            E = self.E(l)
            s = E // n  # finest cells per cell of this level
            K, J, I = np.meshgrid(r, r, r, indexing="ij")
            ghost = (I < g) | (I >= n + g) | (J < g) | (J >= n + g) | (K < g) | (K >= n + g)
            cells = []
            for k, j, i in zip(K[ghost], J[ghost], I[ghost]):
                # finest-lattice centre of this cell
                p = [(b[0] * n + i - g) * s + s // 2, (b[1] * n + j - g) * s + s // 2, (b[2] * n + k - g) * s + s // 2]
                t = self.leaf_at(p)
                if t is None:
                    cells.append((i, j, k, None))
                    continue
                cells.append((i, j, k, self._cell_source(t, p, s)))
            self._cell_maps.append(cells)
            for d in range(3):
                shp = [NN, NN, NN]
                shp[2 - d] += 1
                KK, JJ, II = np.meshgrid(*[np.arange(x) for x in shp], indexing="ij")
                idx = [II, JJ, KK]
                gh = np.zeros(KK.shape, bool)
                for a in range(3):
                    hi = n + g + (1 if a == d else 0)
                    gh |= (idx[a] < g) | (idx[a] >= hi)
                faces = []
                for k, j, i in zip(KK[gh], JJ[gh], II[gh]):
                    c = (i, j, k)
                    p = [(b[a] * n + c[a] - g) * s + (0 if a == d else s // 2) for a in range(3)]
                    faces.append((i, j, k, self._face_source(d, p, s)))
                self._face_maps[d].append(faces)
        return self._cell_maps, self._face_maps

    def _cell_source(self, t, p, s):
        lt, bt = t
        n, g = self.n, self.ngz
        st = self.E(lt) // n
        w = self.wrap(p)
        qs = self.index[t]
        if st == s:
            return qs, [tuple(w[a] // st - bt[a] * n + g for a in range(3))], 1.0
        if st > s:  # coarser: the containing cell
            return qs, [tuple(w[a] // st - bt[a] * n + g for a in range(3))], 1.0
        # finer: the 8 cells of the finer level inside this cell
        base = [w[a] - s // 2 for a in range(3)]
        cs = []
        for dz in (0, 1):
            for dy in (0, 1):
                for dx_ in (0, 1):
                    off = (dx_, dy, dz)
                    cs.append(tuple((base[a] + off[a] * st) // st - bt[a] * n + g for a in range(3)))
        return qs, cs, 0.125

    def _face_source(self, d, p, s):
        """Face of axis d at finest-lattice point p (on the face plane)."""
        n, g = self.n, self.ngz
        # the leaf owning the cell on the upper side of the face (or lower
        # side at the domain's upper end)
        t = self.leaf_at(p)
        if t is None:
            pm = list(p)
            pm[d] -= 1
            t = self.leaf_at(pm)
            if t is None:
                return None
        lt, bt = t
        st = self.E(lt) // n
        w = self.wrap(p)
        if w is None:
            pm = list(p)
            pm[d] -= 1
            w = list(self.wrap(pm))
            w[d] += 1
        qs = self.index[t]
        local = lambda x, a: x // st - bt[a] * n + g
        if st == s:
            return qs, [tuple(local(w[a], a) if a != d else (w[a] - bt[a] * n * st) // st + g for a in range(3))], [1.0]
        if st > s:  # coarser: on a coarse face plane take it, else interpolate between the two
            fd = (w[d] - bt[d] * n * st)
            lo_f = fd // st
            frac = (fd - lo_f * st) / st
            c = [local(w[a], a) if a != d else lo_f + g for a in range(3)]
            if frac == 0:
                return qs, [tuple(c)], [1.0]
            c2 = list(c)
            c2[d] += 1
            return qs, [tuple(c), tuple(c2)], [1.0 - frac, frac]
        # finer: the 4 finer faces inside this face
        o1, o2 = ODIR[d]
        base = list(w)
        base[o1] -= s // 2
        base[o2] -= s // 2
        cs = []
        for b2 in (0, 1):
            for b1 in (0, 1):
                pp = list(base)
                pp[o1] += b1 * st
                pp[o2] += b2 * st
                cs.append(tuple(local(pp[a], a) if a != d else (pp[a] - bt[a] * n * st) // st + g for a in range(3)))
        return qs, cs, [0.25] * 4

    def fill_ghosts(self, state, bx, by, bz, nvars=abi.N_HRSC):
        """Composite ghost fill of the first nvars state variables and face B
        (host numpy arrays in the library layout), in place.  Sources are
        read from the interiors (the fill reads the arrays as they were)."""
        cm, fm = self._maps()
        src = state.copy()
        for q, cells in enumerate(cm):
            for i, j, k, rec in cells:
                if rec is None:
                    continue
                qs, cs, w = rec
                acc = 0.0
                for (ci, cj, ck) in cs:
                    acc = acc + src[qs, :nvars, ck, cj, ci]
                state[q, :nvars, k, j, i] = acc * w if len(cs) > 1 else acc
        for d, arr in enumerate((bx, by, bz)):
            srcb = arr.copy()
            for q, faces in enumerate(fm[d]):
                for i, j, k, rec in faces:
                    if rec is None:
                        continue
                    qs, cs, ws = rec
                    if len(cs) == 1:
                        arr[q, k, j, i] = srcb[qs, cs[0][2], cs[0][1], cs[0][0]]
                    elif len(cs) == 2:
                        arr[q, k, j, i] = ws[0] * srcb[qs, cs[0][2], cs[0][1], cs[0][0]] + \
                            ws[1] * srcb[qs, cs[1][2], cs[1][1], cs[1][0]]
                    else:
                        s_ = 0.0
                        for c in cs:
                            s_ += srcb[qs, c[2], c[1], c[0]]
                        arr[q, k, j, i] = 0.25 * s_
