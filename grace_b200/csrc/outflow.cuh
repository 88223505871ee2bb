// Mass outflux through the outer domain boundary (GRACE's
// boundary_outflow_t::accumulate, include/grace/evolution/boundary_outflow.hh:
// 79-180): for each listed (quadrant, face) on a non-periodic outer boundary,
// the DENS face flux summed over the face's interior cells, times the face's
// outward sign, the cell face area and the substep weight dt * dtfact, added
// to one device scalar.  It reads the face fluxes the last substep left in
// the stage scratch (after the FOFC correction, before they were applied),
// the ones the reference integrates.
#pragma once
#include "stage_kernels.cuh"

namespace grb {

constexpr int kOutflowThreads = 128;

// One CTA per listed face.  face: 2 axis + side (side 1 = upper).  dx: the
// (3, nq) cell spacings, dx[d + 3 q].
__global__ void __launch_bounds__(kOutflowThreads) k_boundary_outflow(Geo G, const double* __restrict__ flux,
                                                                      const int64_t* __restrict__ quad,
                                                                      const uint8_t* __restrict__ face,
                                                                      const double* __restrict__ dx, double weight,
                                                                      double* __restrict__ out) {
  const int64_t q = quad[blockIdx.x];
  const int f = face[blockIdx.x];
  const int axis = f >> 1;
  const int n[3] = {G.nx, G.ny, G.nz};
  const int na = axis == 0 ? G.ny : G.nx, nb = axis == 2 ? G.ny : G.nz;
  const int plane = (f & 1) ? n[axis] + G.g : G.g;
  double acc = 0.0;
  for (int lin = threadIdx.x; lin < na * nb; lin += kOutflowThreads) {
    const int a = G.g + lin % na, b = G.g + lin / na;
    const int i = axis == 0 ? plane : a;
    const int j = axis == 1 ? plane : (axis == 0 ? a : b);
    const int k = axis == 2 ? plane : b;
    acc += flux[flx(G, i, j, k, 0, axis, q)];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double part[kOutflowThreads / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kOutflowThreads / 32; ++w) s += part[w];
    const double d0 = dx[3 * q], d1 = dx[3 * q + 1], d2 = dx[3 * q + 2];
    const double dA = axis == 0 ? d1 * d2 : (axis == 1 ? d0 * d2 : d0 * d1);
    atomicAdd(out, ((f & 1) ? 1.0 : -1.0) * weight * dA * s);
  }
}

}  // namespace grb
