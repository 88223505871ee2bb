// Face fluxes from shared-memory tiles staged by TMA (tuned mode).
//
// Same arithmetic as getflux<dir> + mhd_fluxes<dir> (grmhd.hh:551-970) on the
// tuned face ranges; what changes is where the stencil comes from.  One CTA
// takes W x R faces of one block: W consecutive faces (x) across the warp
// lanes, R rows of them along the "row" axis, one index along the third.
// Thread 0 issues two 5-D TMA loads (cp.async.bulk.tensor, no multicast)
// into shared memory: the 10 reconstructed aux variables (RHO .. ENTROPY,
// aux variables 0..9) and the 10 metric variables (GXX .. BETAZ, state
// variables 7..16) of every cell the tile's stencils touch, the full x
// extent of the block (boxes start at x = 0, so every copy is 16-byte
// aligned).  Rows past the end of the block are zero-filled by the copy and
// feed only idle threads.  All threads wait on one mbarrier (bounded), then
// each reconstructs its face from shared memory: a cell read by six faces
// comes from DRAM once per tile.
#pragma once
#include <cuda.h>

#include "stage_kernels.cuh"

namespace grb {

// Tile geometry of one direction (host-computed).
struct FluxTile {
  int lo[3], n[3];  // face box of the tuned range
  int R;            // face rows per CTA
  int BY, BZ;       // box extent along y and z (cells)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void tma_load5(uint32_t dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3,
                                          int c4, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
      :
      : "r"(dst), "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(mbar)
      : "memory");
}
// Bounded wait for phase `parity` of an mbarrier; false after `limit` tries.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int limit) {
  for (int it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// getflux<dir> on a staged stencil.  A, M: aux / metric tile at stencil
// cell 0 (the cell three before the face) of variable 0; vs: variable
// stride; st: stencil stride (cells along dir).
template <int dir>
__device__ __forceinline__ void getflux_tile(const DevParams& P, int recon, bool rusanov, const double* A,
                                             const double* M, int vs, int st, double bface, double f[7],
                                             double vb[4]) {
  const double alpl = M[(GRB_ALP - GRB_GXX) * vs + 2 * st];
  const double alpr = M[(GRB_ALP - GRB_GXX) * vs + 3 * st];
  double gm[10];
#pragma unroll
  for (int a = 0; a < 10; ++a) {
    const double* p = M + a * vs;
    gm[a] = face4(p[st], p[2 * st], p[3 * st], p[4 * st]);
  }
  const Met m = make_met<true>(gm, gm + 7, gm[6]);
  const int av[10] = {GRB_RHO, GRB_ZVECX, GRB_ZVECY, GRB_ZVECZ, GRB_YE, GRB_TEMP, GRB_ENTROPY, GRB_BX, GRB_BY, GRB_BZ};
  const int pv[10] = {GRB_P_RHO, GRB_P_ZX, GRB_P_ZY, GRB_P_ZZ, GRB_P_YE, GRB_P_TEMP, GRB_P_ENT, GRB_P_BX, GRB_P_BY, GRB_P_BZ};
  double pl[13], pr[13];
  const bool donor = (alpl <= P.alp_ex || alpr <= P.alp_ex);
  if (!donor && recon == GRB_RECON_WENOZ) {
    // two variables per division: their four WENO-Z states through div_quad
#pragma unroll
    for (int r = 0; r < 10; r += 2) {
      double u0[6], u1[6], n[4], d[4], q[4];
#pragma unroll
      for (int o = 0; o < 6; ++o) {
        u0[o] = A[av[r] * vs + o * st];
        u1[o] = A[av[r + 1] * vs + o * st];
      }
      weno_z_nd(u0, n[0], d[0], n[1], d[1]);
      weno_z_nd(u1, n[2], d[2], n[3], d[3]);
      div_quad(n, d, q);
      pl[pv[r]] = q[0];
      pr[pv[r]] = q[1];
      pl[pv[r + 1]] = q[2];
      pr[pv[r + 1]] = q[3];
    }
  } else {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
      const double* p = A + av[r] * vs;
      if (donor) {
        pl[pv[r]] = p[2 * st];
        pr[pv[r]] = p[3 * st];
      } else {
        double u[6];
#pragma unroll
        for (int o = 0; o < 6; ++o) u[o] = p[o * st];
        recon6_fast(recon, u, pl[pv[r]], pr[pv[r]]);
      }
    }
  }
  const double bn = bface * m.isqrtg;
  pl[GRB_P_BX + dir] = bn;
  pr[GRB_P_BX + dir] = bn;
  eos_PT_pair_f(P.eos, pl, pr);
  mhd_fluxes<dir, true>(P, rusanov, pl, pr, m, f, vb);
}

constexpr int kTmaWaitLimit = 1 << 22;

// Shared memory of one CTA: aux tile and metric tile, each
// [10 vars][BZ][BY][NX] doubles, the metric tile starting on a 128-byte
// boundary, then the mbarrier and one more word (the persistent form's
// current tile).
__host__ __device__ inline int flux_tile_doubles(const Geo& G, const FluxTile& T) {
  return (10 * T.BY * T.BZ * G.NX + 15) / 16 * 16;
}
__host__ __device__ inline size_t flux_tile_smem(const Geo& G, const FluxTile& T) {
  return 2 * sizeof(double) * (size_t)flux_tile_doubles(G, T) + 16;
}

// The face of this thread in a staged tile (box origin oy, oz of block q):
// lanes along x, rows along the tile's row axis; threads past the tile's
// faces do nothing.
template <int dir>
__device__ __forceinline__ void flux_tile_face(const DevParams& P, const Geo& G, const FluxTile& T,
                                               const double* sa, const double* sm, int vs, int oy, int oz,
                                               int64_t q, const double* __restrict__ bface, const StageBufs& B) {
  const int W = T.n[0];
  const int w = threadIdx.x % W, r = threadIdx.x / W;
  if (r >= T.R) return;
  const int i = T.lo[0] + w;
  int j, k, base, st;
  if (dir == 0) {
    j = oy + r; k = oz;
    if (j >= T.lo[1] + T.n[1]) return;
    base = r * G.NX + i - 3; st = 1;
  } else if (dir == 1) {
    j = oy + 3 + r; k = oz;
    if (j >= T.lo[1] + T.n[1]) return;
    base = r * G.NX + i; st = G.NX;
  } else {
    j = oy; k = oz + 3 + r;
    if (k >= T.lo[2] + T.n[2]) return;
    base = r * G.NX + i; st = G.NX;
  }
  const int64_t bi = dir == 0 ? bxi(G, i, j, k, q) : dir == 1 ? byi(G, i, j, k, q) : bzi(G, i, j, k, q);
  double f[7], vb[4];
  getflux_tile<dir>(P, P.recon, P.riemann == GRB_RIEMANN_LLF, sa + base, sm + base, vs, st, __ldg(bface + bi), f, vb);
  store_face(G, B, P.emf, dir, i, j, k, q, f, vb);
}

// grid: (ceil(n_row / R), n_other, nq); NT threads (128 or 256); W = n[0]
// <= NT; R = NT / W rows (a 256-thread tile re-reads the 5-row stencil halo
// of the y and z directions over twice as many rows).
//   dir 0: lanes i (faces), rows j, other k; box rows j (BY = R, BZ = 1)
//   dir 1: lanes i, rows j (faces), other k; box rows j - 3 .. (BY = R + 5)
//   dir 2: lanes i, rows k (faces), other j; box rows k - 3 .. (BZ = R + 5)
template <int dir, int MINB, int NT = 128>
__global__ void __launch_bounds__(NT, MINB) k_flux_tma(DevParams P, Geo G, FluxTile T,
                                                      const __grid_constant__ CUtensorMap tm_aux,
                                                      const __grid_constant__ CUtensorMap tm_met,
                                                      const double* __restrict__ bface, StageBufs B) {
  extern __shared__ __align__(128) unsigned char sm_raw[];
  const int vs = T.BY * T.BZ * G.NX;  // variable stride in the tile
  const int td = flux_tile_doubles(G, T);
  double* sa = reinterpret_cast<double*>(sm_raw);
  double* sm = sa + td;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + td);
  const int tile = blockIdx.x, other = blockIdx.y;
  const int64_t q = blockIdx.z;
  // box origin in cells (x always 0)
  int oy, oz;
  if (dir == 0) { oy = T.lo[1] + tile * T.R; oz = T.lo[2] + other; }
  else if (dir == 1) { oy = T.lo[1] + tile * T.R - 3; oz = T.lo[2] + other; }
  else { oy = T.lo[1] + other; oz = T.lo[2] + tile * T.R - 3; }
  const uint32_t mb = smem_u32(mbar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  // both destinations start on 128-byte boundaries (checked: no copy is
  // issued otherwise, and the wait below then gives up)
  const bool aligned = ((smem_u32(sa) | smem_u32(sm)) & 127u) == 0;
  if (threadIdx.x == 0 && aligned) {
    const uint32_t bytes = (uint32_t)(2 * 10 * vs * sizeof(double));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
    tma_load5(smem_u32(sa), &tm_aux, 0, oy, oz, 0, (int)q, mb);
    tma_load5(smem_u32(sm), &tm_met, 0, oy, oz, GRB_GXX, (int)q, mb);
  }
  if (!aligned) {
    if (threadIdx.x == 0) atomicOr(B.flags, GRB_FLAG_WAIT_TIMEOUT);
    return;
  }
  if (!mbar_wait(mb, 0, kTmaWaitLimit)) {
    if (threadIdx.x == 0) atomicOr(B.flags, GRB_FLAG_WAIT_TIMEOUT);
    return;
  }
  flux_tile_face<dir>(P, G, T, sa, sm, vs, oy, oz, q, bface, B);
}

// The same as a persistent launch (tuned candidate): one wave of CTAs, each
// taking tiles, numbered tile row fastest, then the other index, then the
// block, from the device work queue *queue (zeroed before the launch) until
// they run out; per tile the same two TMA loads into the same shared
// memory, the mbarrier's phase alternating from tile to tile.  Every thread
// reaches every barrier; a wait that gives up sets the flag and ends the
// CTA.  ntx, nother: tiles along the row axis, indices along the third.
template <int dir, int MINB, int NT = 128>
__global__ void __launch_bounds__(NT, MINB) k_flux_tma_queue(DevParams P, Geo G, FluxTile T,
                                                            const __grid_constant__ CUtensorMap tm_aux,
                                                            const __grid_constant__ CUtensorMap tm_met,
                                                            const double* __restrict__ bface, StageBufs B,
                                                            unsigned long long* __restrict__ queue, int ntx,
                                                            int nother) {
  extern __shared__ __align__(128) unsigned char sm_raw[];
  const int vs = T.BY * T.BZ * G.NX;
  const int td = flux_tile_doubles(G, T);
  double* sa = reinterpret_cast<double*>(sm_raw);
  double* sm = sa + td;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + td);
  // the tile taken from the queue, in the second word after the mbarrier
  unsigned long long& item = *reinterpret_cast<unsigned long long*>(mbar + 1);
  const uint32_t mb = smem_u32(mbar);
  // both destinations start on 128-byte boundaries (the same for every
  // thread, so the CTA leaves as a whole otherwise)
  if (((smem_u32(sa) | smem_u32(sm)) & 127u) != 0) {
    if (threadIdx.x == 0) atomicOr(B.flags, GRB_FLAG_WAIT_TIMEOUT);
    return;
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  const unsigned long long ntiles = (unsigned long long)ntx * (unsigned long long)nother * (unsigned long long)G.nq;
  const uint32_t bytes = (uint32_t)(2 * 10 * vs * sizeof(double));
  uint32_t parity = 0;
  for (;;) {
    // every thread is done with the previous tile's shared memory here
    __syncthreads();
    if (threadIdx.x == 0) item = atomicAdd(queue, 1ull);
    __syncthreads();
    const unsigned long long t = item;
    if (t >= ntiles) break;
    const int tile = (int)(t % (unsigned long long)ntx);
    const unsigned long long rest = t / (unsigned long long)ntx;
    const int other = (int)(rest % (unsigned long long)nother);
    const int64_t q = (int64_t)(rest / (unsigned long long)nother);
    int oy, oz;
    if (dir == 0) { oy = T.lo[1] + tile * T.R; oz = T.lo[2] + other; }
    else if (dir == 1) { oy = T.lo[1] + tile * T.R - 3; oz = T.lo[2] + other; }
    else { oy = T.lo[1] + other; oz = T.lo[2] + tile * T.R - 3; }
    if (threadIdx.x == 0) {
      // the async proxy overwrites what the generic proxy just read
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
      tma_load5(smem_u32(sa), &tm_aux, 0, oy, oz, 0, (int)q, mb);
      tma_load5(smem_u32(sm), &tm_met, 0, oy, oz, GRB_GXX, (int)q, mb);
    }
    const bool ok = mbar_wait(mb, parity, kTmaWaitLimit);
    parity ^= 1u;
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(B.flags, GRB_FLAG_WAIT_TIMEOUT);
      return;
    }
    flux_tile_face<dir>(P, G, T, sa, sm, vs, oy, oz, q, bface, B);
  }
}

}  // namespace grb
