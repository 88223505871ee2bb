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
// preserving).  Every product and sum is rounded on its own (__dmul_rn,
// __dadd_rn), as the reference writes them, so the results do not depend on
// how the compiler would contract them.
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
  const int v = V.v[(uint32_t)t - iq * (uint32_t)V.n];
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

}  // namespace grb
