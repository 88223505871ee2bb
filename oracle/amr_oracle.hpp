// CPU oracle — test infrastructure only, never linked into the CUDA library.
//
// FMR restriction into coarse buffers (GRACE's ghost-zone restriction,
// include/grace/amr/ghostzone_kernels/restrict_kernels.hh and
// pr_helpers.hh), restated:
//   * restrict_op (restrict_kernels.hh:42-109): every fine quadrant iq
//     writes the coarse-resolution copy of its interior into its coarse
//     buffer: dest(i+g, j+g, k+g, v, dst_q) = op(u, 2i+g, 2j+g, 2k+g,
//     half_x, half_y, half_z) for i, j, k in [0, n/2), the half flags being
//     the bits of the quadrant's Morton child id;
//   * op = second_order_restrict_op (pr_helpers.hh:187-213), the
//     pair-symmetric 8-cell average, for the low-order variable list, and
//     lagrange_restrict_op<4> (pr_helpers.hh:216-322), the 5-point Lagrange
//     restriction with per-axis stencil selection (edges and parent half)
//     and pair-symmetric contractions (pr_helpers.hh:47-64), for the
//     high-order list, with the coefficient table of
//     fill_fifth_order_restriction_coefficients (pr_ho_coeffs.hh:33-60), the
//     one GRACE passes (src/amr/amr_ghosts.cpp:136);
//   * div_free_restrict_op<d> (restrict_kernels.hh:118-165) for the face
//     arrays: the average of the 4 fine faces inside each coarse face, over
//     i in [0, n/2 + (d == 0)) etc., accumulated in (ii, jj, kk) order.
// Compiled with -ffp-contract=off, so every product and sum is rounded on
// its own, as the reference's operators are written.
#pragma once
#include <cmath>
#include <cstdint>

namespace orc_amr {

// The 4 stencils x 5 weights of the 5-point restriction (stencils L2, L1,
// CENTER, R1 as compute_offset numbers them).
inline const double* restrict5_coeffs() {
  static const double c[20] = {
      -5.0 / 128.0, 7.0 / 32.0,   -35.0 / 64.0, 35.0 / 32.0,  35.0 / 128.0,
      3.0 / 128.0,  -5.0 / 32.0,  45.0 / 64.0,  15.0 / 32.0,  -5.0 / 128.0,
      -5.0 / 128.0, 15.0 / 32.0,  45.0 / 64.0,  -5.0 / 32.0,  3.0 / 128.0,
      35.0 / 128.0, 35.0 / 32.0,  -35.0 / 64.0, 7.0 / 32.0,   -5.0 / 128.0};
  return c;
}

// Read access to variable v of block q of a LayoutLeft (N0, N1, N2, nv, nq)
// array.
struct Acc {
  const double* a;
  int N0, N1, N2;
  int64_t off;  // offset of (0, 0, 0, v, q)
  double operator()(int i, int j, int k) const { return a[off + ((int64_t)k * N1 + j) * N0 + i]; }
};

inline double restrict2(const Acc& u, int i, int j, int k) {
  const double q00 = u(i, j, k) + u(i + 1, j, k);
  const double q10 = u(i, j + 1, k) + u(i + 1, j + 1, k);
  const double q01 = u(i, j, k + 1) + u(i + 1, j, k + 1);
  const double q11 = u(i, j + 1, k + 1) + u(i + 1, j + 1, k + 1);
  const double r0 = q00 + q10;
  const double r1 = q01 + q11;
  return 0.125 * (r0 + r1);
}

inline int lag4_offset(int pos, int n, int ngz, int half) {
  const int lb = pos - ngz;
  const int ub = n + ngz - pos - 1;
  if (ub == 1) return 0;
  if (lb == 0) return 3;
  if (ub == 2) return 1;
  return half ? 1 : 2;
}

inline double contract5(const double c[5], const double u[5]) {
  const double s_outer = c[0] * u[0] + c[4] * u[4];
  const double s_inner = c[1] * u[1] + c[3] * u[3];
  const double s_ctr = c[2] * u[2];
  return (s_outer + s_inner) + s_ctr;
}

inline double restrict_lag4(const Acc& u, int n, int ngz, int i, int j, int k, int hx, int hy, int hz) {
  const double* co = restrict5_coeffs();
  const int ox = lag4_offset(i, n, ngz, hx), oy = lag4_offset(j, n, ngz, hy), oz = lag4_offset(k, n, ngz, hz);
  const int cx = ox - 3, cy = oy - 3, cz = oz - 3;
  double Sx[5][5];
  for (int dk = 0; dk < 5; ++dk)
    for (int dj = 0; dj < 5; ++dj) {
      double line[5];
      for (int di = 0; di < 5; ++di) line[di] = u(i + di + cx, j + dj + cy, k + dk + cz);
      Sx[dj][dk] = contract5(co + 5 * ox, line);
    }
  double Sy[5];
  for (int dk = 0; dk < 5; ++dk) {
    double line[5];
    for (int dj = 0; dj < 5; ++dj) line[dj] = Sx[dj][dk];
    Sy[dk] = contract5(co + 5 * oy, line);
  }
  return contract5(co + 5 * oz, Sy);
}

// The two per-point operators of this restatement.
struct OrcOps {
  double lo(const Acc& u, int i, int j, int k) const { return restrict2(u, i, j, k); }
  double hi(const Acc& u, int n, int ngz, int i, int j, int k, int hx, int hy, int hz) const {
    return restrict_lag4(u, n, ngz, i, j, k, hx, hy, hz);
  }
};

// Cell variables: src (fine blocks) and dst (coarse buffers) are LayoutLeft
// (N, N, N, nvars, .) arrays with N = n + 2 ngz.  Ops: the per-point
// operators (this restatement's, or the reference's own compiled in place).
template <class Ops>
inline void restrict_cells(const Ops& ops, int n, int ngz, int nvars, const double* src, double* dst,
                           int64_t nquads, const int64_t* src_q, const int64_t* dst_q, const uint8_t* child,
                           const int* vlo, int nlo, const int* vhi, int nhi) {
  const int N = n + 2 * ngz;
  const int64_t cells = (int64_t)N * N * N;
  for (int64_t iq = 0; iq < nquads; ++iq) {
    const int hx = child[iq] & 1, hy = (child[iq] >> 1) & 1, hz = (child[iq] >> 2) & 1;
    for (int pass = 0; pass < 2; ++pass) {
      const int* vl = pass == 0 ? vlo : vhi;
      const int nl = pass == 0 ? nlo : nhi;
      for (int t = 0; t < nl; ++t) {
        const int v = vl[t];
        const Acc u{src, N, N, N, (src_q[iq] * nvars + v) * cells};
        double* d = dst + (dst_q[iq] * nvars + v) * cells;
        for (int k = 0; k < n / 2; ++k)
          for (int j = 0; j < n / 2; ++j)
            for (int i = 0; i < n / 2; ++i) {
              const int fi = 2 * i + ngz, fj = 2 * j + ngz, fk = 2 * k + ngz;
              d[((int64_t)(k + ngz) * N + (j + ngz)) * N + (i + ngz)] =
                  pass == 0 ? ops.lo(u, fi, fj, fk) : ops.hi(u, n, ngz, fi, fj, fk, hx, hy, hz);
            }
      }
    }
  }
}

// One face array staggered along dir: (N + (dir == 0), N + (dir == 1),
// N + (dir == 2), 1, .).
inline void restrict_faces(int dir, int n, int ngz, const double* src, double* dst, int64_t nquads,
                           const int64_t* src_q, const int64_t* dst_q) {
  const int N = n + 2 * ngz;
  const int N0 = N + (dir == 0), N1 = N + (dir == 1), N2 = N + (dir == 2);
  const int64_t sz = (int64_t)N0 * N1 * N2;
  for (int64_t iq = 0; iq < nquads; ++iq) {
    const Acc u{src, N0, N1, N2, src_q[iq] * sz};
    double* d = dst + dst_q[iq] * sz;
    for (int k = 0; k < n / 2 + (dir == 2); ++k)
      for (int j = 0; j < n / 2 + (dir == 1); ++j)
        for (int i = 0; i < n / 2 + (dir == 0); ++i) {
          double val = 0;
          for (int ii = 0; ii <= (dir != 0); ++ii)
            for (int jj = 0; jj <= (dir != 1); ++jj)
              for (int kk = 0; kk <= (dir != 2); ++kk)
                val += u(2 * i + ngz + ii, 2 * j + ngz + jj, 2 * k + ngz + kk);
          d[((int64_t)(k + ngz) * N1 + (j + ngz)) * N0 + (i + ngz)] = 0.25 * val;
        }
  }
}

// ---------------------------------------------------------------------------
// FMR prolongation into ghost zones (GRACE's prolong_op and
// div_free_prolong_op, include/grace/amr/ghostzone_kernels/
// prolongation_kernels.hh:46-399, driven per element kind by
// prolongation_task_factories.hh:70-230, index maps of index_helpers.hh),
// restated.  A ghost element of a fine quadrant (one of its 6 faces, 12
// edges or 8 corners) whose neighbour is coarser is filled from the
// quadrant's coarse buffer, which holds the coarse data around the
// quadrant's volume: coarse cell ngz + t covers fine cells ngz + 2t and
// ngz + 2t + 1.
//   * the element's ghost cells (ghost_indices below restates
//     compute_ghost_indices_{face,edge,corner}, index_helpers.hh:84-356):
//     a face spans (ngz, n, n) points, an edge (ngz, ngz, n), a corner
//     ngz^3; fine point (a, b, c) reads coarse point (a/2, b/2, c/2) of the
//     half-size block with the low ghosts shifted by ngz/2;
//   * low-order variables: slope_limited_prolong_op<minmod>
//     (pr_helpers.hh:73-103), u0 + sum_d (+-1/4) minmod(dL, dR), the sign
//     by the fine index's parity (odd = upper half);
//   * high-order variables: lagrange_prolong_op<4> (pr_helpers.hh:105-185),
//     5-point stencils (i-2 .. i+2) with the coefficients of
//     fill_fifth_order_prolongation_coefficients (pr_ho_coeffs.hh:60-75),
//     weights 0..4 for the lower half, 5..9 for the upper, pair-symmetric
//     contractions;
//   * face B: the Toth-Roe divergence-preserving prolongation
//     (div_free_prolong_op, prolongation_kernels.hh:110-399): phase 1 gives
//     the fine faces lying on coarse faces the coarse value plus minmod
//     slopes (skipping the first face of an axis where the neighbour has fine
//     data, adding the last one where it has not), phase 2 the faces inside
//     coarse cells from the phase-1 faces around them.
enum { ORC_ELEM_FACE = 0, ORC_ELEM_EDGE = 1, ORC_ELEM_CORNER = 2 };

// Index of loop point (a, b, c) of element e of a kind, in a block of n
// cells per side with ngz ghosts whose low ghost region starts at goff.
inline void ghost_indices(int kind, int e, int n, int ngz, int goff, int a, int b, int c, int out[3]) {
  auto side = [&](int high, int t) { return high ? n + ngz + t : goff + t; };
  if (kind == ORC_ELEM_FACE) {
    const int ax = e / 2;
    const int t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
    out[ax] = side(e % 2, a);
    out[t1] = ngz + b;
    out[t2] = ngz + c;
  } else if (kind == ORC_ELEM_EDGE) {
    const int ax = e / 4;
    const int f1 = ax == 0 ? 1 : 0, f2 = ax == 2 ? 1 : 2;
    out[f1] = side(e & 1, a);
    out[f2] = side((e >> 1) & 1, b);
    out[ax] = ngz + c;
  } else {
    out[0] = side(e & 1, a);
    out[1] = side((e >> 1) & 1, b);
    out[2] = side((e >> 2) & 1, c);
  }
}

// First and last even fine index along axis d of element e
// (_get_{first,last}_iter_index_*, index_helpers.hh:110-355).
inline void ghost_first_last(int kind, int e, int d, int n, int ngz, int& first, int& last) {
  int where;  // 0 below the interior, 1 above it, 2 spanning it
  if (kind == ORC_ELEM_FACE) {
    where = d == e / 2 ? e % 2 : 2;
  } else if (kind == ORC_ELEM_EDGE) {
    const int ax = e / 4;
    const int f1 = ax == 0 ? 1 : 0;
    where = d == ax ? 2 : (d == f1 ? (e & 1) : ((e >> 1) & 1));
  } else {
    where = (e >> d) & 1;
  }
  first = where == 2 ? ngz : (where ? n + ngz : 0);
  last = where == 2 ? n + ngz - 2 : (where ? n + 2 * ngz - 2 : ngz - 2);
}

inline void ghost_extents(int kind, int n, int ngz, int e[3]) {
  e[0] = ngz;
  e[1] = kind == ORC_ELEM_FACE ? n : ngz;
  e[2] = kind == ORC_ELEM_CORNER ? ngz : n;
}

inline double minmod(double l, double r) {
  const double m = std::fabs(l) < std::fabs(r) ? std::fabs(l) : std::fabs(r);
  return 0.5 * (std::copysign(1.0, l) + std::copysign(1.0, r)) * m;
}

inline const double* prolong5_coeffs() {
  static const double c[10] = {-45.0 / 2048.0, 105.0 / 512.0, 945.0 / 1024.0, -63.0 / 512.0, 35.0 / 2048.0,
                               35.0 / 2048.0,  -63.0 / 512.0, 945.0 / 1024.0, 105.0 / 512.0, -45.0 / 2048.0};
  return c;
}

// s[d]: 1 for the upper fine half of the coarse cell along d, else 0.
inline double prolong_slope(const Acc& u, const int c[3], const int s[3]) {
  const double u0 = u(c[0], c[1], c[2]);
  double acc = 0.0;
  for (int d = 0; d < 3; ++d) {
    const int dx = d == 0, dy = d == 1, dz = d == 2;
    const double eta = (s[d] ? 1.0 : -1.0) * 0.25;
    const double sl = u0 - u(c[0] - dx, c[1] - dy, c[2] - dz);
    const double sr = u(c[0] + dx, c[1] + dy, c[2] + dz) - u0;
    acc += eta * minmod(sl, sr);
  }
  return u0 + acc;
}

inline double prolong_lag4(const Acc& u, const int c[3], const int s[3]) {
  const double* co = prolong5_coeffs();
  const double *cx = co + 5 * s[0], *cy = co + 5 * s[1], *cz = co + 5 * s[2];
  double Sy[5];
  for (int dk = 0; dk < 5; ++dk) {
    double col[5];
    for (int dj = 0; dj < 5; ++dj) {
      double line[5];
      for (int di = 0; di < 5; ++di) line[di] = u(c[0] + di - 2, c[1] + dj - 2, c[2] + dk - 2);
      col[dj] = contract5(cx, line);
    }
    Sy[dk] = contract5(cy, col);
  }
  return contract5(cz, Sy);
}

// Cell variables of the elements of one kind.  fine / cbuf: LayoutLeft
// (N, N, N, nvars, .) arrays, N = n + 2 ngz.
inline void prolong_cells(int kind, int n, int ngz, int nvars, double* fine, const double* cbuf, int64_t nelems,
                          const int64_t* fine_q, const int64_t* cbuf_q, const uint8_t* elem, const int* vlo,
                          int nlo, const int* vhi, int nhi) {
  const int N = n + 2 * ngz;
  const int64_t cells = (int64_t)N * N * N;
  int ext[3];
  ghost_extents(kind, n, ngz, ext);
  for (int64_t iq = 0; iq < nelems; ++iq)
    for (int pass = 0; pass < 2; ++pass) {
      const int* vl = pass == 0 ? vlo : vhi;
      const int nl = pass == 0 ? nlo : nhi;
      for (int t = 0; t < nl; ++t) {
        const int v = vl[t];
        const Acc u{cbuf, N, N, N, (cbuf_q[iq] * nvars + v) * cells};
        double* d = fine + (fine_q[iq] * nvars + v) * cells;
        for (int c = 0; c < ext[2]; ++c)
          for (int b = 0; b < ext[1]; ++b)
            for (int a = 0; a < ext[0]; ++a) {
              int f[3], cc[3], s[3];
              ghost_indices(kind, elem[iq], n, ngz, 0, a, b, c, f);
              ghost_indices(kind, elem[iq], n / 2, ngz, ngz / 2, a / 2, b / 2, c / 2, cc);
              for (int q = 0; q < 3; ++q) s[q] = f[q] & 1;
              d[((int64_t)f[2] * N + f[1]) * N + f[0]] = pass == 0 ? prolong_slope(u, cc, s) : prolong_lag4(u, cc, s);
            }
      }
    }
}

// Read/write access to one face array of one block.
struct FaceArr {
  double* a;
  int N0, N1;
  double& operator()(int i, int j, int k) const { return a[((int64_t)k * N1 + j) * N0 + i]; }
};

// Phase 1 at coarse point c / fine point f: the fine faces on the coarse
// faces through c's lower corner, for the arrays whose flag is set.
inline void fill_coarse_faces(const FaceArr F[3], const FaceArr C[3], const int c[3], const int f[3],
                              const bool fill[3]) {
  for (int d = 0; d < 3; ++d) {
    if (!fill[d]) continue;
    const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;  // the face's tangential axes
    int cm[3] = {c[0], c[1], c[2]}, cp[3] = {c[0], c[1], c[2]};
    const double U0 = C[d](c[0], c[1], c[2]);
    double sl[2];
    for (int h = 0; h < 2; ++h) {
      const int ax = h == 0 ? t1 : t2;
      cm[ax] -= 1;
      cp[ax] += 1;
      sl[h] = 0.25 * minmod(U0 - C[d](cm[0], cm[1], cm[2]), C[d](cp[0], cp[1], cp[2]) - U0);
      cm[ax] += 1;
      cp[ax] -= 1;
    }
    for (int p = 0; p < 2; ++p)
      for (int q = 0; q < 2; ++q) {
        int o[3] = {f[0], f[1], f[2]};
        o[t1] += p;
        o[t2] += q;
        F[d](o[0], o[1], o[2]) = U0 + (p ? 1.0 : -1.0) * sl[0] + (q ? 1.0 : -1.0) * sl[1];
      }
  }
}

// Face B of the elements of one kind.  fx, fy, fz: fine face arrays
// (N+1, N, N, 1, .), (N, N+1, N, 1, .), (N, N, N+1, 1, .); cx, cy, cz the
// coarse buffers of the same shapes.  have_fine[6 i + 2 axis + side]: the
// neighbour across that side of element i's region holds fine data.
inline void prolong_faces(int kind, int n, int ngz, double* fx, double* fy, double* fz, const double* cx,
                          const double* cy, const double* cz, int64_t nelems, const int64_t* fine_q,
                          const int64_t* cbuf_q, const uint8_t* elem, const int8_t* have_fine) {
  const int N = n + 2 * ngz;
  const int64_t szf[3] = {(int64_t)(N + 1) * N * N, (int64_t)N * (N + 1) * N, (int64_t)N * N * (N + 1)};
  double* fa[3] = {fx, fy, fz};
  const double* ca[3] = {cx, cy, cz};
  int ext[3];
  ghost_extents(kind, n, ngz, ext);
  for (int d = 0; d < 3; ++d) ext[d] /= 2;
  for (int64_t iq = 0; iq < nelems; ++iq) {
    const int e = elem[iq];
    FaceArr F[3], C[3];
    for (int d = 0; d < 3; ++d) {
      F[d] = FaceArr{fa[d] + fine_q[iq] * szf[d], N + (d == 0), N + (d == 1)};
      C[d] = FaceArr{const_cast<double*>(ca[d]) + cbuf_q[iq] * szf[d], N + (d == 0), N + (d == 1)};
    }
    const int8_t* hf = have_fine + 6 * iq;
    int first[3], last[3];
    for (int d = 0; d < 3; ++d) ghost_first_last(kind, e, d, n, ngz, first[d], last[d]);
    for (int c = 0; c < ext[2]; ++c)
      for (int b = 0; b < ext[1]; ++b)
        for (int a = 0; a < ext[0]; ++a) {
          int f[3], cc[3];
          ghost_indices(kind, e, n, ngz, 0, 2 * a, 2 * b, 2 * c, f);
          ghost_indices(kind, e, n / 2, ngz, ngz / 2, a, b, c, cc);
          bool fill[3];
          for (int d = 0; d < 3; ++d) fill[d] = !(f[d] == first[d] && hf[2 * d]);
          fill_coarse_faces(F, C, cc, f, fill);
          for (int d = 0; d < 3; ++d)
            if (f[d] == last[d] && !hf[2 * d + 1]) {
              int c1[3] = {cc[0], cc[1], cc[2]}, f1[3] = {f[0], f[1], f[2]};
              c1[d] += 1;
              f1[d] += 2;
              bool only[3] = {d == 0, d == 1, d == 2};
              fill_coarse_faces(F, C, c1, f1, only);
            }
        }
    for (int c = 0; c < ext[2]; ++c)
      for (int b = 0; b < ext[1]; ++b)
        for (int a = 0; a < ext[0]; ++a) {
          int f[3];
          ghost_indices(kind, e, n, ngz, 0, 2 * a, 2 * b, 2 * c, f);
          const int i = f[0], j = f[1], k = f[2];
          const FaceArr &u = F[0], &v = F[1], &w = F[2];
          double Uxx = 0, Vyy = 0, Wzz = 0, Uxyz = 0, Vxyz = 0, Wxyz = 0;
          for (int ii = 0; ii < 2; ++ii)
            for (int jj = 0; jj < 2; ++jj)
              for (int kk = 0; kk < 2; ++kk) {
                const double is = ii ? 1 : -1, js = jj ? 1 : -1, ks = kk ? 1 : -1;
                Uxx += is * js * v(i + ii, j + 2 * jj, k + kk) + is * ks * w(i + ii, j + jj, k + 2 * kk);
                Vyy += is * js * u(i + 2 * ii, j + jj, k + kk) + js * ks * w(i + ii, j + jj, k + 2 * kk);
                Wzz += is * ks * u(i + 2 * ii, j + jj, k + kk) + js * ks * v(i + ii, j + 2 * jj, k + kk);
                Uxyz += is * js * ks * u(i + 2 * ii, j + jj, k + kk);
                Vxyz += is * js * ks * v(i + ii, j + 2 * jj, k + kk);
                Wxyz += is * js * ks * w(i + ii, j + jj, k + 2 * kk);
              }
          Uxx *= 0.125;
          Vyy *= 0.125;
          Wzz *= 0.125;
          Uxyz *= 0.0625;
          Vxyz *= 0.0625;
          Wxyz *= 0.0625;
          for (int jj = 0; jj < 2; ++jj)
            for (int kk = 0; kk < 2; ++kk) {
              const double js = jj ? 1 : -1, ks = kk ? 1 : -1;
              u(i + 1, j + jj, k + kk) = 0.5 * (u(i, j + jj, k + kk) + u(i + 2, j + jj, k + kk)) + Uxx + ks * Vxyz + js * Wxyz;
              v(i + jj, j + 1, k + kk) = 0.5 * (v(i + jj, j, k + kk) + v(i + jj, j + 2, k + kk)) + Vyy + js * Wxyz + ks * Uxyz;
              w(i + jj, j + kk, k + 1) = 0.5 * (w(i + jj, j + kk, k) + w(i + jj, j + kk, k + 2)) + Wzz + ks * Uxyz + js * Vxyz;
            }
        }
  }
}

}  // namespace orc_amr
