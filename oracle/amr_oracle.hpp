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

}  // namespace orc_amr
