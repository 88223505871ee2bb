// FMR restriction into coarse buffers (GRACE's ghost-zone restriction,
// include/grace/amr/ghostzone_kernels/restrict_kernels.hh:42-165 with the
// operators of pr_helpers.hh:47-64, 187-322 and the coefficient table of
// pr_ho_coeffs.hh:33-60 that src/amr/amr_ghosts.cpp:136 passes).
//
// Every fine quadrant in the list writes the coarse-resolution image of its
// interior into its coarse buffer: cell variables by the pair-symmetric
// 8-cell average (low-order list) or the 5-point Lagrange restriction
// (high-order list, stencils chosen per axis by the block edge and by the
// quadrant's half of its parent, from its Morton child id), face B by the
// average of the 4 fine faces inside each coarse face (divergence
// preserving).  The second half of the file holds the prolongation into
// ghost zones (the ghost-zone prolongation of prolongation_kernels.hh with
// the operators of pr_helpers.hh:73-185): the face, edge and corner ghost
// elements of fine quadrants filled from their coarse buffers.  Every
// product and sum is rounded on its own (__dmul_rn, __dadd_rn), as the
// reference writes them, so the results do not depend on how the compiler
// would contract them.
#pragma once
#include "stage_kernels.cuh"

namespace grb {

// The 4 stencils x 5 weights of the 5-point restriction.
__constant__ double c_restrict5[20] = {
    -5.0 / 128.0, 7.0 / 32.0,   -35.0 / 64.0, 35.0 / 32.0,  35.0 / 128.0,
    3.0 / 128.0,  -5.0 / 32.0,  45.0 / 64.0,  15.0 / 32.0,  -5.0 / 128.0,
    -5.0 / 128.0, 15.0 / 32.0,  45.0 / 64.0,  -5.0 / 32.0,  3.0 / 128.0,
    35.0 / 128.0, 35.0 / 32.0,  -35.0 / 64.0, 7.0 / 32.0,   -5.0 / 128.0};

__device__ __forceinline__ double contract5_rn(const double* c, const double u[5]) {
  const double so = __dadd_rn(__dmul_rn(c[0], u[0]), __dmul_rn(c[4], u[4]));
  const double si = __dadd_rn(__dmul_rn(c[1], u[1]), __dmul_rn(c[3], u[3]));
  return __dadd_rn(__dadd_rn(so, si), __dmul_rn(c[2], u[2]));
}
__device__ __forceinline__ int lag4_offset(int pos, int n, int ngz, int half) {
  const int lb = pos - ngz, ub = n + ngz - pos - 1;
  if (ub == 1) return 0;
  if (lb == 0) return 3;
  if (ub == 2) return 1;
  return half ? 1 : 2;
}

// One list of restriction work: var list (up to 23 state variables).
struct RestrictVars {
  int n;
  int v[GRB_N_EVOL_VARS];
};
// V.v[i] by an unrolled select: a dynamic index into a kernel parameter
// would copy the whole list to local memory.
__device__ __forceinline__ int list_var(const RestrictVars& V, int i) {
  int v = V.v[0];
#pragma unroll
  for (int t = 1; t < GRB_N_EVOL_VARS; ++t) v = i == t ? V.v[t] : v;
  return v;
}

// Cell variables.  box: (n/2)^3 coarse cells x (nvars_in_list x nquads)
// folded into the box's block index (variable fastest).  kHigh: the 5-point
// Lagrange operator, else the 8-cell average.
template <bool kHigh>
__global__ void __launch_bounds__(128) k_restrict_cells(Geo G, Box box, RestrictVars V, FastDiv dnv,
                                                        const double* __restrict__ src, double* __restrict__ dst,
                                                        const int64_t* __restrict__ src_q,
                                                        const int64_t* __restrict__ dst_q,
                                                        const uint8_t* __restrict__ child) {
  int i, j, k;
  int64_t t;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, t)) return;
  const uint32_t iq = fast_div((uint32_t)t, dnv);
  const int v = list_var(V, (int)((uint32_t)t - iq * (uint32_t)V.n));
  const int N0 = G.NX, N1 = G.NY;
  const double* u = src + (src_q[iq] * GRB_N_EVOL_VARS + v) * G.cells;
  auto at = [&](int x, int y, int z) { return u[((int64_t)z * N1 + y) * N0 + x]; };
  const int fi = 2 * i + G.g, fj = 2 * j + G.g, fk = 2 * k + G.g;
  double r;
  if (!kHigh) {
    const double q00 = __dadd_rn(at(fi, fj, fk), at(fi + 1, fj, fk));
    const double q10 = __dadd_rn(at(fi, fj + 1, fk), at(fi + 1, fj + 1, fk));
    const double q01 = __dadd_rn(at(fi, fj, fk + 1), at(fi + 1, fj, fk + 1));
    const double q11 = __dadd_rn(at(fi, fj + 1, fk + 1), at(fi + 1, fj + 1, fk + 1));
    r = __dmul_rn(0.125, __dadd_rn(__dadd_rn(q00, q10), __dadd_rn(q01, q11)));
  } else {
    const uint8_t cid = child[iq];
    const int ox = lag4_offset(fi, G.nx, G.g, cid & 1);
    const int oy = lag4_offset(fj, G.ny, G.g, (cid >> 1) & 1);
    const int oz = lag4_offset(fk, G.nz, G.g, (cid >> 2) & 1);
    const double* cx = c_restrict5 + 5 * ox;
    const double* cy = c_restrict5 + 5 * oy;
    const double* cz = c_restrict5 + 5 * oz;
    double Sy[5];
#pragma unroll
    for (int dk = 0; dk < 5; ++dk) {
      double col[5];
#pragma unroll
      for (int dj = 0; dj < 5; ++dj) {
        double line[5];
#pragma unroll
        for (int di = 0; di < 5; ++di) line[di] = at(fi + di + ox - 3, fj + dj + oy - 3, fk + dk + oz - 3);
        col[dj] = contract5_rn(cx, line);
      }
      Sy[dk] = contract5_rn(cy, col);
    }
    r = contract5_rn(cz, Sy);
  }
  dst[(dst_q[iq] * GRB_N_EVOL_VARS + v) * G.cells + ((int64_t)(k + G.g) * N1 + (j + G.g)) * N0 + (i + G.g)] = r;
}

// High-order list, one thread per (i, j) column of coarse cells and
// variable, walking the column along z: each fine plane's contractions along
// x and y (with the column's x and y stencils) are computed once and the
// last five kept in registers; coarse cell k takes the z contraction of the
// five planes of its stencil (fk + oz - 3 .. fk + oz + 1) when the walk has
// reached the last of them.  Stencil windows never move back along z (the
// edge and half-dependent offsets keep their ends non-decreasing), so one
// pass over the fine planes ngz .. nz + ngz - 1 serves every cell.  The
// operands and their order are those of k_restrict_cells<true>, bit for
// bit.  box: (nx/2, ny/2, 1) x (nvars_in_list x nquads), variable fastest.
__global__ void __launch_bounds__(128) k_restrict_lag_zcol(Geo G, Box box, RestrictVars V, FastDiv dnv,
                                                           const double* __restrict__ src, double* __restrict__ dst,
                                                           const int64_t* __restrict__ src_q,
                                                           const int64_t* __restrict__ dst_q,
                                                           const uint8_t* __restrict__ child) {
  int i, j, k_;
  int64_t t;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k_, t)) return;
  const uint32_t iq = fast_div((uint32_t)t, dnv);
  const int v = list_var(V, (int)((uint32_t)t - iq * (uint32_t)V.n));
  const int N0 = G.NX, N1 = G.NY, g = G.g;
  const double* u = src + (src_q[iq] * GRB_N_EVOL_VARS + v) * G.cells;
  double* o = dst + (dst_q[iq] * GRB_N_EVOL_VARS + v) * G.cells;
  const uint8_t cid = child[iq];
  const int fi = 2 * i + g, fj = 2 * j + g, hz = (cid >> 2) & 1;
  const int ox = lag4_offset(fi, G.nx, g, cid & 1), oy = lag4_offset(fj, G.ny, g, (cid >> 1) & 1);
  const double* cx = c_restrict5 + 5 * ox;
  const double* cy = c_restrict5 + 5 * oy;
  const int x0 = fi + ox - 3, y0 = fj + oy - 3;
  double ring[5];
  int k = 0;
  int oz = lag4_offset(g, G.nz, g, hz);
  for (int z = g; z < G.nz + g; ++z) {
#pragma unroll
    for (int q = 0; q < 4; ++q) ring[q] = ring[q + 1];
    const double* plane = u + (int64_t)z * N1 * N0;
    double col[5];
#pragma unroll
    for (int dj = 0; dj < 5; ++dj) {
      const double* l = plane + (int64_t)(y0 + dj) * N0 + x0;
      const double line[5] = {l[0], l[1], l[2], l[3], l[4]};
      col[dj] = contract5_rn(cx, line);
    }
    ring[4] = contract5_rn(cy, col);
    // every coarse cell whose stencil ends at this plane
    while (k < G.nz / 2 && 2 * k + g + oz + 1 == z) {
      o[((int64_t)(k + g) * N1 + (j + g)) * N0 + (i + g)] = contract5_rn(c_restrict5 + 5 * oz, ring);
      ++k;
      if (k < G.nz / 2) oz = lag4_offset(2 * k + g, G.nz, g, hz);
    }
  }
}

// Face B staggered along dir: box (n/2 + (dir == 0), n/2 + (dir == 1),
// n/2 + (dir == 2)) x nquads.
template <int dir>
__global__ void __launch_bounds__(128) k_restrict_faces(Geo G, Box box, const double* __restrict__ src,
                                                        double* __restrict__ dst, const int64_t* __restrict__ src_q,
                                                        const int64_t* __restrict__ dst_q) {
  int i, j, k;
  int64_t iq;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, iq)) return;
  const int N0 = G.NX + (dir == 0), N1 = G.NY + (dir == 1), N2 = G.NZ + (dir == 2);
  const int64_t sz = (int64_t)N0 * N1 * N2;
  const double* u = src + src_q[iq] * sz;
  double val = 0.0;
#pragma unroll
  for (int ii = 0; ii <= (dir != 0); ++ii)
#pragma unroll
    for (int jj = 0; jj <= (dir != 1); ++jj)
#pragma unroll
      for (int kk = 0; kk <= (dir != 2); ++kk)
        val = __dadd_rn(val, u[((int64_t)(2 * k + G.g + kk) * N1 + (2 * j + G.g + jj)) * N0 + (2 * i + G.g + ii)]);
  dst[dst_q[iq] * sz + ((int64_t)(k + G.g) * N1 + (j + G.g)) * N0 + (i + G.g)] = __dmul_rn(0.25, val);
}

// ---------------------------------------------------------------------------
// FMR prolongation into ghost zones (GRACE's prolong_op and
// div_free_prolong_op, include/grace/amr/ghostzone_kernels/
// prolongation_kernels.hh:46-399, with the index maps of index_helpers.hh
// and the operators of pr_helpers.hh:73-185).  The ghost elements of one
// kind (faces, edges or corners of fine quadrants whose neighbour is
// coarser) are filled from each quadrant's coarse buffer: coarse cell
// ngz + t covers fine cells ngz + 2t, ngz + 2t + 1, and the low coarse
// ghosts start at ngz/2.

// Along axis d of ghost element e of one kind: where its ghost region lies
// (0 below the interior, 1 above it, 2 spanning it) and which of the
// launch's three loop indices runs along that axis (the index maps of
// compute_ghost_indices_{face,edge,corner}, index_helpers.hh:84-356).  A
// face (e = 2 axis + side) runs its normal axis over loop index 0 and its
// tangential axes over 1, 2; an edge (e = 4 axis + sides) its two fixed
// axes over 0, 1 (the sides in bits 0, 1 of e) and its own axis over 2; a
// corner axis d over d (the side in bit d of e).
template <int kKind>
__host__ __device__ __forceinline__ void ghost_axis(int e, int d, int& where, int& loop) {
  if (kKind == GRB_ELEM_FACE) {
    const int ax = e >> 1;
    where = d == ax ? (e & 1) : 2;
    loop = d == ax ? 0 : (d < ax ? d + 1 : d);
  } else if (kKind == GRB_ELEM_EDGE) {
    const int ax = e >> 2;
    const int f1 = ax == 0 ? 1 : 0;
    loop = d == ax ? 2 : (d == f1 ? 0 : 1);
    where = d == ax ? 2 : ((e >> loop) & 1);
  } else {
    where = (e >> d) & 1;
    loop = d;
  }
}
__host__ __device__ __forceinline__ int ghost_idx(int where, int n, int g, int goff, int t) {
  return where == 2 ? g + t : (where ? n + g + t : goff + t);
}
__device__ __forceinline__ int pick3(int l, int a, int b, int c) { return l == 0 ? a : (l == 1 ? b : c); }

// The 5-point prolongation weights, lower fine half then upper.
__constant__ double c_prolong5[10] = {-45.0 / 2048.0, 105.0 / 512.0, 945.0 / 1024.0, -63.0 / 512.0, 35.0 / 2048.0,
                                      35.0 / 2048.0,  -63.0 / 512.0, 945.0 / 1024.0, 105.0 / 512.0, -45.0 / 2048.0};

// Low-order list, one thread per coarse cell of an element and variable:
// the minmod slope-limited operator for the element's 8 fine cells inside
// that coarse cell (the three limited slopes shared).  box: the kind's
// ghost extent halved, (ngz/2, n/2 | ngz/2, n/2 | ngz/2) x (nvars_in_list x
// nelems), variable fastest.  The two children along x are adjacent doubles
// at an even fine index and leave as one 16-byte store.
template <int kKind>
__global__ void __launch_bounds__(128) k_prolong_cells(Geo G, Box box, RestrictVars V, FastDiv dnv,
                                                       const double* __restrict__ cbuf, double* __restrict__ fine,
                                                       const int64_t* __restrict__ fine_q,
                                                       const int64_t* __restrict__ cbuf_q,
                                                       const uint8_t* __restrict__ elem) {
  int a, b, c;
  int64_t t;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, a, b, c, t)) return;
  const uint32_t iq = fast_div((uint32_t)t, dnv);
  const int v = list_var(V, (int)((uint32_t)t - iq * (uint32_t)V.n));
  const int e = elem[iq];
  int f[3], k[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int w, lp;
    ghost_axis<kKind>(e, d, w, lp);
    const int l = pick3(lp, a, b, c);
    f[d] = ghost_idx(w, G.nx, G.g, 0, 2 * l);  // the lower child; even
    k[d] = ghost_idx(w, G.nx / 2, G.g, G.g / 2, l);
  }
  const int N0 = G.NX, N1 = G.NY;
  const double* u = cbuf + (cbuf_q[iq] * GRB_N_EVOL_VARS + v) * G.cells;
  auto at = [&](int x, int y, int z) { return u[((int64_t)z * N1 + y) * N0 + x]; };
  const double u0 = at(k[0], k[1], k[2]);
  double lim[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int dx = d == 0, dy = d == 1, dz = d == 2;
    const double sl = __dsub_rn(u0, at(k[0] - dx, k[1] - dy, k[2] - dz));
    const double sr = __dsub_rn(at(k[0] + dx, k[1] + dy, k[2] + dz), u0);
    lim[d] = lim_minmod(sl, sr);
  }
  double* o = fine + (fine_q[iq] * GRB_N_EVOL_VARS + v) * G.cells;
#pragma unroll
  for (int pz = 0; pz < 2; ++pz)
#pragma unroll
    for (int py = 0; py < 2; ++py) {
      double r[2];
#pragma unroll
      for (int px = 0; px < 2; ++px) {
        double acc = 0.0;
        acc = __dadd_rn(acc, __dmul_rn(px ? 0.25 : -0.25, lim[0]));
        acc = __dadd_rn(acc, __dmul_rn(py ? 0.25 : -0.25, lim[1]));
        acc = __dadd_rn(acc, __dmul_rn(pz ? 0.25 : -0.25, lim[2]));
        r[px] = __dadd_rn(u0, acc);
      }
      *reinterpret_cast<double2*>(o + ((int64_t)(f[2] + pz) * N1 + (f[1] + py)) * N0 + f[0]) =
          make_double2(r[0], r[1]);
    }
}

// High-order list, one thread per (x, y) column of an element's coarse
// region and variable, walking the column along z: each z plane's x sums
// (both x halves) and y sums (the 4 (x, y) halves) are computed once and the
// last five planes' y sums kept in registers, from which every coarse cell
// of the column gets its 8 fine cells (the z sum).  The operands and their
// order are those of lagrange_prolong_op<4>, so the results are its bits;
// against one thread per coarse cell it saves the loads and sums that
// neighbouring cells along z share.  box: (the kind's largest number of
// columns, 1, 1) x (nvars_in_list x nelems), variable fastest; threads past
// the element's columns return.
template <int kKind>
__global__ void __launch_bounds__(128) k_prolong_lag_zcol(Geo G, Box box, RestrictVars V, FastDiv dnv,
                                                          const double* __restrict__ cbuf, double* __restrict__ fine,
                                                          const int64_t* __restrict__ fine_q,
                                                          const int64_t* __restrict__ cbuf_q,
                                                          const uint8_t* __restrict__ elem) {
  int col, b_, c_;
  int64_t t;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, col, b_, c_, t)) return;
  const uint32_t iq = fast_div((uint32_t)t, dnv);
  const int v = list_var(V, (int)((uint32_t)t - iq * (uint32_t)V.n));
  const int e = elem[iq];
  const int n = G.nx, g = G.g;
  int r[3], k0[3], f0[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int w, lp;
    ghost_axis<kKind>(e, d, w, lp);
    r[d] = w == 2 ? n / 2 : g / 2;
    k0[d] = ghost_idx(w, n / 2, g, g / 2, 0);
    f0[d] = ghost_idx(w, n, g, 0, 0);
  }
  if (col >= r[0] * r[1]) return;
  const int x = col % r[0], y = col / r[0];
  const int kx = k0[0] + x, ky = k0[1] + y;
  const int N0 = G.NX, N1 = G.NY;
  const double* u = cbuf + (cbuf_q[iq] * GRB_N_EVOL_VARS + v) * G.cells;
  double* o = fine + (fine_q[iq] * GRB_N_EVOL_VARS + v) * G.cells;
  double ring[4][5];  // [2 px + py][plane], plane 4 the newest
  for (int zz = -2; zz < r[2] + 2; ++zz) {
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) ring[p][q] = ring[p][q + 1];
    const double* plane = u + (int64_t)(k0[2] + zz) * N1 * N0;
    double Sx[2][5];
#pragma unroll
    for (int dj = 0; dj < 5; ++dj) {
      const double* l = plane + (int64_t)(ky + dj - 2) * N0 + kx - 2;
      const double line[5] = {l[0], l[1], l[2], l[3], l[4]};
      Sx[0][dj] = contract5_rn(c_prolong5, line);
      Sx[1][dj] = contract5_rn(c_prolong5 + 5, line);
    }
#pragma unroll
    for (int px = 0; px < 2; ++px) {
      ring[2 * px][4] = contract5_rn(c_prolong5, Sx[px]);
      ring[2 * px + 1][4] = contract5_rn(c_prolong5 + 5, Sx[px]);
    }
    if (zz >= 2) {
      const int z = zz - 2;
#pragma unroll
      for (int pz = 0; pz < 2; ++pz)
#pragma unroll
        for (int py = 0; py < 2; ++py) {
          const double lo = contract5_rn(c_prolong5 + 5 * pz, ring[py]);
          const double hi = contract5_rn(c_prolong5 + 5 * pz, ring[2 + py]);
          *reinterpret_cast<double2*>(o + ((int64_t)(f0[2] + 2 * z + pz) * N1 + (f0[1] + 2 * y + py)) * N0 + f0[0] +
                                      2 * x) = make_double2(lo, hi);
        }
    }
  }
}

// One block's face array staggered along d.
struct FaceBlk {
  double* p;
  int N0, N1;
  __device__ __forceinline__ double& operator()(int i, int j, int k) const {
    return p[((int64_t)k * N1 + j) * N0 + i];
  }
};

// Phase 1 at coarse point c / fine point f: the fine faces of array d lying
// on the coarse face through c get the coarse value plus minmod slopes along
// the face's two tangential axes (Toth & Roe 2002, eqs. 4-5).
__device__ __forceinline__ void prolong_coarse_face(int d, const FaceBlk& F, const FaceBlk& C, const int c[3],
                                                    const int f[3]) {
  const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
  const double U0 = C(c[0], c[1], c[2]);
  double sl[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int ax = h == 0 ? t1 : t2;
    const int o0 = ax == 0, o1 = ax == 1, o2 = ax == 2;
    const double dl = __dsub_rn(U0, C(c[0] - o0, c[1] - o1, c[2] - o2));
    const double dr = __dsub_rn(C(c[0] + o0, c[1] + o1, c[2] + o2), U0);
    sl[h] = __dmul_rn(0.25, lim_minmod(dl, dr));
  }
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      int o[3] = {f[0], f[1], f[2]};
      o[t1] += p;
      o[t2] += q;
      F(o[0], o[1], o[2]) = __dadd_rn(__dadd_rn(U0, p ? sl[0] : -sl[0]), q ? sl[1] : -sl[1]);
    }
}

// Face B, one phase.  box: the kind's ghost extent halved x nelems; each
// point is one coarse cell of the element.  have_fine[6 i + 2 axis + side]:
// the neighbour across that side of element i's region holds fine data.
// Phase 1 writes the fine faces on coarse faces, phase 2 (a separate launch,
// as it reads phase 1's faces around each coarse cell) those inside coarse
// cells (Toth & Roe 2002, eqs. 8-12).
template <int kKind, int kPhase>
__global__ void __launch_bounds__(128) k_prolong_faces(Geo G, Box box, double* __restrict__ bx,
                                                       double* __restrict__ by, double* __restrict__ bz,
                                                       const double* __restrict__ cbx, const double* __restrict__ cby,
                                                       const double* __restrict__ cbz,
                                                       const int64_t* __restrict__ fine_q,
                                                       const int64_t* __restrict__ cbuf_q,
                                                       const uint8_t* __restrict__ elem,
                                                       const int8_t* __restrict__ have_fine) {
  int a, b, c;
  int64_t iq;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, a, b, c, iq)) return;
  const int e = elem[iq];
  const int n = G.nx, g = G.g;
  int f[3], wh[3], l[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int lp;
    ghost_axis<kKind>(e, d, wh[d], lp);
    l[d] = pick3(lp, a, b, c);
    f[d] = ghost_idx(wh[d], n, g, 0, 2 * l[d]);
  }
  const int N = G.NX;
  const int64_t sz = (int64_t)(N + 1) * N * N;
  const FaceBlk u{bx + fine_q[iq] * sz, N + 1, N}, v{by + fine_q[iq] * sz, N, N + 1}, w{bz + fine_q[iq] * sz, N, N};
  if (kPhase == 1) {
    const int64_t cq = cbuf_q[iq];
    const FaceBlk C[3] = {{const_cast<double*>(cbx) + cq * sz, N + 1, N},
                          {const_cast<double*>(cby) + cq * sz, N, N + 1},
                          {const_cast<double*>(cbz) + cq * sz, N, N}};
    const FaceBlk F[3] = {u, v, w};
    const int8_t* hf = have_fine + 6 * iq;
    int k[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) k[d] = ghost_idx(wh[d], n / 2, g, g / 2, l[d]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int first = wh[d] == 2 ? g : (wh[d] ? n + g : 0);
      const int last = wh[d] == 2 ? n + g - 2 : (wh[d] ? n + 2 * g - 2 : g - 2);
      if (!(f[d] == first && hf[2 * d])) prolong_coarse_face(d, F[d], C[d], k, f);
      if (f[d] == last && !hf[2 * d + 1]) {
        int k1[3] = {k[0], k[1], k[2]}, f1[3] = {f[0], f[1], f[2]};
        k1[d] += 1;
        f1[d] += 2;
        prolong_coarse_face(d, F[d], C[d], k1, f1);
      }
    }
  } else {
    const int i = f[0], j = f[1], kk0 = f[2];
    double Uxx = 0, Vyy = 0, Wzz = 0, Uxyz = 0, Vxyz = 0, Wxyz = 0;
#pragma unroll
    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
      for (int jj = 0; jj < 2; ++jj)
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
          const bool sij = (ii ^ jj) == 0, sik = (ii ^ kk) == 0, sjk = (jj ^ kk) == 0, sijk = ((ii ^ jj ^ kk) & 1) == 1;
          const double vu = v(i + ii, j + 2 * jj, kk0 + kk), wu = w(i + ii, j + jj, kk0 + 2 * kk);
          const double uu = u(i + 2 * ii, j + jj, kk0 + kk);
          Uxx = __dadd_rn(Uxx, __dadd_rn(sij ? vu : -vu, sik ? wu : -wu));
          Vyy = __dadd_rn(Vyy, __dadd_rn(sij ? uu : -uu, sjk ? wu : -wu));
          Wzz = __dadd_rn(Wzz, __dadd_rn(sik ? uu : -uu, sjk ? vu : -vu));
          Uxyz = __dadd_rn(Uxyz, sijk ? uu : -uu);
          Vxyz = __dadd_rn(Vxyz, sijk ? vu : -vu);
          Wxyz = __dadd_rn(Wxyz, sijk ? wu : -wu);
        }
    Uxx = __dmul_rn(Uxx, 0.125);
    Vyy = __dmul_rn(Vyy, 0.125);
    Wzz = __dmul_rn(Wzz, 0.125);
    Uxyz = __dmul_rn(Uxyz, 0.0625);
    Vxyz = __dmul_rn(Vxyz, 0.0625);
    Wxyz = __dmul_rn(Wxyz, 0.0625);
#pragma unroll
    for (int jj = 0; jj < 2; ++jj)
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        const double sj = jj ? 1.0 : -1.0, sk = kk ? 1.0 : -1.0;
        const double mu = __dmul_rn(0.5, __dadd_rn(u(i, j + jj, kk0 + kk), u(i + 2, j + jj, kk0 + kk)));
        const double mv = __dmul_rn(0.5, __dadd_rn(v(i + jj, j, kk0 + kk), v(i + jj, j + 2, kk0 + kk)));
        const double mw = __dmul_rn(0.5, __dadd_rn(w(i + jj, j + kk, kk0), w(i + jj, j + kk, kk0 + 2)));
        u(i + 1, j + jj, kk0 + kk) = __dadd_rn(__dadd_rn(__dadd_rn(mu, Uxx), sk * Vxyz), sj * Wxyz);
        v(i + jj, j + 1, kk0 + kk) = __dadd_rn(__dadd_rn(__dadd_rn(mv, Vyy), sj * Wxyz), sk * Uxyz);
        w(i + jj, j + kk, kk0 + 1) = __dadd_rn(__dadd_rn(__dadd_rn(mw, Wzz), sk * Uxyz), sj * Vxyz);
      }
  }
}

// Ghost fill by gather maps (grb_fill_ghosts_gather): entry e writes
// sum over its cnt[e] used slots k of w[k n + e] * a[src[k n + e] + v vs]
// into a[dst[e] + v vs] for variable v = blockIdx.y (vs the offset between
// variables), accumulated in slot order with every product and sum rounded
// on its own.  Sources are never destinations (interior cells and faces).
__global__ void __launch_bounds__(256) k_ghost_gather(int64_t n, int64_t vstride, const int8_t* __restrict__ cnt,
                                                      const int64_t* __restrict__ dst,
                                                      const int64_t* __restrict__ src,
                                                      const double* __restrict__ w, double* __restrict__ a) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int64_t vo = (int64_t)blockIdx.y * vstride;
  const int c = cnt[e];
  double acc = __dmul_rn(w[e], a[src[e] + vo]);
  for (int k = 1; k < c; ++k) acc = __dadd_rn(acc, __dmul_rn(w[k * n + e], a[src[k * n + e] + vo]));
  a[dst[e] + vo] = acc;
}

}  // namespace grb
