// Learned bracket for the Kastaun c2p.
//
// A 12 -> 64 -> 64 -> 64 -> 1 ReLU network predicts y = asinh(L / L0) with
// L = log(mu0 / mu) and L0 = 1e-4: mu is the root of the Kastaun master
// function f(mu) = mu - 1/(hbw + rbar^2 mu) (kastaun_c2p.hh:245-290), mu0 the
// top of the plain bracket (kastaun_c2p.hh:355-369, an EOS-free Newton solve
// the plain path runs anyway).  L spans 1e-10..3; the asinh keeps small gaps
// linear and large ones logarithmic, so no tail dominates the squared error.  Features: the Kastaun scalars of the state (kastaun_c2p.hh:306-337:
// D, q = tau/D, |r|, |B~|^2, cos^2(r, B~)) and log mu0, normalised, each
// split into a BF16 high part and a BF16 remainder (12 inputs).  Hidden
// layers run on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32
// accumulation); the output layer is FP32 on the BF16-rounded activations.
// The unchanged FP64 Brent iteration then starts from
// [mu0 e^(-L0 sinh(y+delta)), min(mu0 e^(-L0 sinh(y-delta)), mu0)] when f
// changes sign there, and from the plain [0, mu0] otherwise, so the network
// only moves where the iteration starts.
//
// Training (all on the GPU): labels come from the roots of the plain FP64
// c2p on the caller's states; k_mlp_grad runs the same tensor-core forward on
// 64 states per CTA, keeps the BF16-rounded activations in shared memory and
// back-propagates in FP32 (straight-through for the BF16 rounding), writing
// one partial gradient per CTA; k_mlp_adam sums the partials in a fixed order
// (bitwise reproducible) and applies Adam.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "c2p.cuh"

namespace grb {

constexpr int kMlpIn = 6;    // features; inputs 0..5 high parts, 6..11 remainders
constexpr int kMlpK0 = 16;   // input width padded to one MMA k-chunk
constexpr int kMlpH = 64;    // hidden width
constexpr double kMlpL0 = 1e-4;  // scale of the asinh target
// FP32 parameter block, in this order: W1[64][16], b1[64], W2[64][64], b2[64],
// W3[64][64], b3[64], w4[64], b4 (trainable), then the normalisation
// fmu[6], fsd[6], tmu, tsd and the bracket half-width delta (in y).
constexpr int kMlpOffW1 = 0;
constexpr int kMlpOffB1 = kMlpOffW1 + kMlpH * kMlpK0;
constexpr int kMlpOffW2 = kMlpOffB1 + kMlpH;
constexpr int kMlpOffB2 = kMlpOffW2 + kMlpH * kMlpH;
constexpr int kMlpOffW3 = kMlpOffB2 + kMlpH;
constexpr int kMlpOffB3 = kMlpOffW3 + kMlpH * kMlpH;
constexpr int kMlpOffW4 = kMlpOffB3 + kMlpH;
constexpr int kMlpOffB4 = kMlpOffW4 + kMlpH;
constexpr int kMlpNumWeights = kMlpOffB4 + 1;
constexpr int kMlpOffNorm = kMlpNumWeights;
constexpr int kMlpNumParams = kMlpOffNorm + 2 * kMlpIn + 3;
// shared-memory row pitches (BF16 elements) that make the B-fragment and
// A-fragment loads bank-conflict free: 8 rows x 4 words land on 32 banks
constexpr int kP1 = 24;   // W1 rows
constexpr int kPH = 72;   // W2, W3 rows
constexpr int kXP = 24;   // input tile rows

struct MlpNorm {
  float fmu[kMlpIn], fsd[kMlpIn], tmu, tsd, delta;
};

// ---- features of one state ------------------------------------------------
// c: densitized conserved variables with densitized cell-centred B, as
// conservs_to_prims receives them (c2p.cpp:188-230); mu0: top of the plain
// Kastaun bracket of the state.  FP64 scalars, FP32 logs.
GRB_HD void mlp_features(const double c[10], const Met& m, double mu0, float f[kMlpIn]) {
  const double isg = 1.0 / m.sqrtg;
  const double D = fmax(c[0] * isg, 1e-30);
  const double iD = 1.0 / D;
  const double q = c[4] * isg * iD;
  const double r[3] = {c[1] * isg * iD, c[2] * isg * iD, c[3] * isg * iD};
  const double isD = isg / sqrt(D);
  const double Bt[3] = {c[7] * isD, c[8] * isD, c[9] * isD};
  const double r2 = sqs(m.gi, r);
  const double b2 = sqs(m.g, Bt);
  const double rb = r[0] * Bt[0] + r[1] * Bt[1] + r[2] * Bt[2];
  f[0] = log10f((float)D);
  f[1] = log10f((float)fmax(q, 1e-30));
  f[2] = 0.5f * log10f((float)(r2 + 1e-30));
  f[3] = log10f((float)(b2 + 1e-30));
  f[4] = (float)fmin(1.0, fmax(0.0, rb * rb / (r2 * b2 + 1e-300)));
  f[5] = (float)log(fmax(mu0, 1e-300));
}

// Top of the plain Kastaun bracket from the densitized cons, by the same
// operations as conservs_to_prims + kastaun_c2p_t::invert (so bit-identical
// to the value the plain solve computes when limit_conservatives leaves the
// state unchanged); 0 for D <= 0.
GRB_HD double plain_mu0(const DevEos& e, const Met& m, const double c[10]) {
  double cc[10];
#pragma unroll
  for (int v = 0; v < 10; ++v) cc[v] = c[v] / m.sqrtg;
  if (!(cc[0] > 0.0)) return 0.0;
  const KSc k = kscalars(e, m, cc);
  return kastaun_mu0(k);
}

// ---- tensor-core helpers ----------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// D(16x8) += A(16x16, row) * B(16x8, col); BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Network in shared memory: BF16 weights (padded rows), FP32 rest.
struct MlpSmem {
  __nv_bfloat16 W1[kMlpH * kP1];
  __nv_bfloat16 W2[kMlpH * kPH];
  __nv_bfloat16 W3[kMlpH * kPH];
  float b1[kMlpH], b2[kMlpH], b3[kMlpH], w4[kMlpH];
  float b4;
  MlpNorm nrm;
};

// Cooperative load: FP32 master parameters -> BF16 weights.  The caller
// synchronises the CTA before use.
__device__ __forceinline__ void mlp_load_smem(MlpSmem& s, const float* __restrict__ P) {
  for (int t = threadIdx.x; t < kMlpH * kMlpK0; t += blockDim.x)
    s.W1[(t >> 4) * kP1 + (t & 15)] = __float2bfloat16_rn(P[kMlpOffW1 + t]);
  for (int t = threadIdx.x; t < kMlpH * kMlpH; t += blockDim.x) {
    s.W2[(t >> 6) * kPH + (t & 63)] = __float2bfloat16_rn(P[kMlpOffW2 + t]);
    s.W3[(t >> 6) * kPH + (t & 63)] = __float2bfloat16_rn(P[kMlpOffW3 + t]);
  }
  for (int t = threadIdx.x; t < kMlpH; t += blockDim.x) {
    s.b1[t] = P[kMlpOffB1 + t];
    s.b2[t] = P[kMlpOffB2 + t];
    s.b3[t] = P[kMlpOffB3 + t];
    s.w4[t] = P[kMlpOffW4 + t];
  }
  if (threadIdx.x == 0) {
    s.b4 = P[kMlpOffB4];
    for (int k = 0; k < kMlpIn; ++k) {
      s.nrm.fmu[k] = P[kMlpOffNorm + k];
      s.nrm.fsd[k] = P[kMlpOffNorm + kMlpIn + k];
    }
    s.nrm.tmu = P[kMlpOffNorm + 2 * kMlpIn];
    s.nrm.tsd = P[kMlpOffNorm + 2 * kMlpIn + 1];
    s.nrm.delta = P[kMlpOffNorm + 2 * kMlpIn + 2];
  }
}

// Network inputs: normalised features split into BF16 high parts (inputs
// 0..5) and BF16 remainders (6..11), 16-bit significands in total; 12..15 zero.
__device__ __forceinline__ void mlp_inputs(const MlpNorm& nrm, const float f[kMlpIn], __nv_bfloat16 x[kMlpK0]) {
#pragma unroll
  for (int k = 0; k < kMlpIn; ++k) {
    const float v = __fdiv_rn(f[k] - nrm.fmu[k], nrm.fsd[k]);
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    x[k] = hi;
    x[kMlpIn + k] = __float2bfloat16_rn(v - __bfloat162float(hi));
  }
#pragma unroll
  for (int k = 2 * kMlpIn; k < kMlpK0; ++k) x[k] = __float2bfloat16_rn(0.f);
}

// B fragment of W^T for W row-major [out][in] with pitch ld: element (k, n)
// = W[n0 + n][k0 + k]; b0 holds k = 2(lane%4)+{0,1}, b1 k+8, n = lane/4.
__device__ __forceinline__ void frag_b_wt(const __nv_bfloat16* W, int ld, int n0, int k0, uint32_t b[2]) {
  const int lane = threadIdx.x & 31;
  const __nv_bfloat16* p = W + (n0 + (lane >> 2)) * ld + k0 + 2 * (lane & 3);
  b[0] = *reinterpret_cast<const uint32_t*>(p);
  b[1] = *reinterpret_cast<const uint32_t*>(p + 8);
}

// One warp, 16 states (rows of xs, BF16, pitch kXP).  The D fragment of
// output tile nt is exactly the A fragment of k-chunk nt/2 of the next
// layer, so activations stay in registers between layers.  Returns the
// network outputs of rows lane/4 (lo) and lane/4 + 8 (hi) in every lane.
// kStore: also write the BF16-rounded activations to H[layer][col][row0 + row]
// (FP32, pitch sp) for the backward pass.
template <bool kStore>
__device__ __forceinline__ void mlp_tile16(const MlpSmem& s, const __nv_bfloat16* xs, float& out_lo,
                                           float& out_hi, float* H, int row0, int sp) {
  const int lane = threadIdx.x & 31;
  const int r = lane >> 2, c = 2 * (lane & 3);
  uint32_t a[4][4];
  {
    uint32_t x[4];
    x[0] = *reinterpret_cast<const uint32_t*>(xs + r * kXP + c);
    x[1] = *reinterpret_cast<const uint32_t*>(xs + (r + 8) * kXP + c);
    x[2] = *reinterpret_cast<const uint32_t*>(xs + r * kXP + c + 8);
    x[3] = *reinterpret_cast<const uint32_t*>(xs + (r + 8) * kXP + c + 8);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      uint32_t b[2];
      frag_b_wt(s.W1, kP1, nt * 8, 0, b);
      mma_bf16(d, x, b);
      const float bb0 = s.b1[nt * 8 + c], bb1 = s.b1[nt * 8 + c + 1];
      const float h0 = fmaxf(d[0] + bb0, 0.f), h1 = fmaxf(d[1] + bb1, 0.f);
      const float h2 = fmaxf(d[2] + bb0, 0.f), h3 = fmaxf(d[3] + bb1, 0.f);
      a[nt >> 1][(nt & 1) ? 2 : 0] = pack_bf16(h0, h1);
      a[nt >> 1][(nt & 1) ? 3 : 1] = pack_bf16(h2, h3);
      if (kStore) {
        float* Hc = H + (nt * 8 + c) * sp + row0;
        Hc[r] = bf16_round(h0);
        Hc[sp + r] = bf16_round(h1);
        Hc[r + 8] = bf16_round(h2);
        Hc[sp + r + 8] = bf16_round(h3);
      }
    }
  }
#pragma unroll
  for (int layer = 0; layer < 2; ++layer) {
    const __nv_bfloat16* W = layer == 0 ? s.W2 : s.W3;
    const float* bias = layer == 0 ? s.b2 : s.b3;
    float* Hl = kStore ? H + (layer + 1) * kMlpH * sp : nullptr;
    uint32_t an[4][4];
    float acc_lo = 0.f, acc_hi = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kc = 0; kc < 4; ++kc) {
        uint32_t b[2];
        frag_b_wt(W, kPH, nt * 8, kc * 16, b);
        mma_bf16(d, a[kc], b);
      }
      const float bb0 = bias[nt * 8 + c], bb1 = bias[nt * 8 + c + 1];
      const float h0 = fmaxf(d[0] + bb0, 0.f), h1 = fmaxf(d[1] + bb1, 0.f);
      const float h2 = fmaxf(d[2] + bb0, 0.f), h3 = fmaxf(d[3] + bb1, 0.f);
      if (layer == 0) {
        an[nt >> 1][(nt & 1) ? 2 : 0] = pack_bf16(h0, h1);
        an[nt >> 1][(nt & 1) ? 3 : 1] = pack_bf16(h2, h3);
      }
      const float r0 = bf16_round(h0), r1 = bf16_round(h1), r2 = bf16_round(h2), r3 = bf16_round(h3);
      if (layer == 1) {
        const float w0 = s.w4[nt * 8 + c], w1 = s.w4[nt * 8 + c + 1];
        acc_lo += r0 * w0 + r1 * w1;
        acc_hi += r2 * w0 + r3 * w1;
      }
      if (kStore) {
        float* Hc = Hl + (nt * 8 + c) * sp + row0;
        Hc[r] = r0;
        Hc[sp + r] = r1;
        Hc[r + 8] = r2;
        Hc[sp + r + 8] = r3;
      }
    }
    if (layer == 0) {
#pragma unroll
      for (int kc = 0; kc < 4; ++kc)
#pragma unroll
        for (int e = 0; e < 4; ++e) a[kc][e] = an[kc][e];
    } else {
      acc_lo += __shfl_xor_sync(0xffffffffu, acc_lo, 1);
      acc_lo += __shfl_xor_sync(0xffffffffu, acc_lo, 2);
      acc_hi += __shfl_xor_sync(0xffffffffu, acc_hi, 1);
      acc_hi += __shfl_xor_sync(0xffffffffu, acc_hi, 2);
      out_lo = acc_lo + s.b4;
      out_hi = acc_hi + s.b4;
    }
  }
}

// Whole warp, one state per lane: network inputs in, network output
// (normalised y) of the lane's own state out.  xs: per-warp shared buffer of
// 32 rows x kXP BF16.  All 32 lanes must call.
__device__ __forceinline__ float mlp_warp32(const MlpSmem& s, __nv_bfloat16* xs, const __nv_bfloat16 x[kMlpK0]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kMlpK0; ++k) xs[lane * kXP + k] = x[k];
  __syncwarp();
  float lo0, hi0, lo1, hi1;
  mlp_tile16<false>(s, xs, lo0, hi0, nullptr, 0, 0);
  mlp_tile16<false>(s, xs + 16 * kXP, lo1, hi1, nullptr, 0, 0);
  __syncwarp();
  // state `lane` is row lane%16 of tile lane/16, held by lane 4*(row%8)
  const int row = lane & 15;
  const int src = 4 * (row & 7);
  const float v0 = __shfl_sync(0xffffffffu, lo0, src);
  const float v1 = __shfl_sync(0xffffffffu, hi0, src);
  const float v2 = __shfl_sync(0xffffffffu, lo1, src);
  const float v3 = __shfl_sync(0xffffffffu, hi1, src);
  return lane >= 16 ? (row >= 8 ? v3 : v2) : (row >= 8 ? v1 : v0);
}

// Learned bracket of one state from the network output and the plain mu0.
__device__ __forceinline__ Guess mlp_bracket(const MlpNorm& nrm, float out, double mu0) {
  const float y = fmaf(out, nrm.tsd, nrm.tmu);
  const float Llo = (float)kMlpL0 * sinhf(y - nrm.delta);
  const float Lhi = (float)kMlpL0 * sinhf(y + nrm.delta);
  Guess g;
  g.lo = mu0 * (double)expf(-Lhi);
  g.hi = fmin(mu0 * (double)expf(-Llo), mu0);
  g.valid = mu0 > 0.0 && g.lo > 0.0 && g.hi > g.lo && isfinite(g.hi);
  g.mu0 = mu0;
  g.has_mu0 = mu0 > 0.0;
  return g;
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  // splitmix64 finaliser (Steele, Lea, Flood 2014)
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ Met batch_metric(const double* __restrict__ metric, int64_t n, int64_t t) {
  double g[6] = {1, 0, 0, 1, 0, 1}, b[3] = {0, 0, 0}, alp = 1.0;
  if (metric) {
#pragma unroll
    for (int a = 0; a < 6; ++a) g[a] = metric[a * n + t];
#pragma unroll
    for (int a = 0; a < 3; ++a) b[a] = metric[(6 + a) * n + t];
    alp = metric[9 * n + t];
  }
  return make_met(g, b, alp);
}

// ---- batched c2p, plain or with the learned bracket ------------------------
struct C2PDiagDev {
  int32_t* iters;      // Brent iterations
  int8_t* guess_used;  // learned bracket held the root
  double* mu;          // Kastaun root (0 where the solve did not run)
  double* bracket;     // [2][n] learned bracket (lo, hi); 0 where none
};

constexpr int kC2PThreads = 128;
struct C2PLearnedSmem {
  MlpSmem net;
  __nv_bfloat16 xs[kC2PThreads / 32][32 * kXP];
};
static_assert(sizeof(MlpSmem) % 16 == 0, "the packed network is copied in 16-byte words");

// Packs the FP32 parameter block into the shared-memory image of the network
// (BF16 weights in padded rows), once per model; c2p CTAs copy the image.
__global__ void __launch_bounds__(256) k_mlp_pack(const float* __restrict__ P, MlpSmem* __restrict__ out) {
  mlp_load_smem(*out, P);
}

// One state per thread.  With the learned bracket every lane of a warp takes
// part in the network (lanes past n with neutral inputs), then returns.
// kFast: the tuned-mode c2p arithmetic (same functions up to rounding).
template <bool kLearned, bool kFast = false>
__global__ void __launch_bounds__(kC2PThreads) k_c2p_batch(DevParams P, int64_t n, const double* __restrict__ cons,
                                                          const double* __restrict__ metric,
                                                          double* __restrict__ prims, double* __restrict__ cons_out,
                                                          uint32_t* __restrict__ err, C2PDiagDev diag,
                                                          const MlpSmem* __restrict__ net, uint32_t* flags) {
  __shared__ __align__(16) unsigned char smraw[kLearned ? sizeof(C2PLearnedSmem) : 16];
  C2PLearnedSmem& S = *reinterpret_cast<C2PLearnedSmem*>(smraw);
  if (kLearned) {
    const uint4* src = reinterpret_cast<const uint4*>(net);
    uint4* dst = reinterpret_cast<uint4*>(&S.net);
    for (int w = threadIdx.x; w < (int)(sizeof(MlpSmem) / 16); w += kC2PThreads) dst[w] = src[w];
    __syncthreads();
  }
  {
    const int64_t t = (int64_t)blockIdx.x * kC2PThreads + threadIdx.x;
    const bool active = t < n;
    const int64_t ts = active ? t : 0;
    const Met m = batch_metric(metric, n, ts);
    double c[10], pr[13];
#pragma unroll
    for (int v = 0; v < 10; ++v) c[v] = active ? cons[v * n + t] : 0.0;
    Guess gs = no_guess();
    if (kLearned) {
      float f[kMlpIn];
      __nv_bfloat16 x[kMlpK0];
      const double mu0 = active ? plain_mu0(P.eos, m, c) : 0.0;
      if (active) mlp_features(c, m, mu0, f);
      else {
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) f[k] = S.net.nrm.fmu[k];
      }
      mlp_inputs(S.net.nrm, f, x);
      const float out = mlp_warp32(S.net, S.xs[threadIdx.x >> 5], x);
      gs = mlp_bracket(S.net.nrm, out, mu0);
    }
    if (!active) return;
    const C2POut o = c2p<kFast>(c, pr, m, P, 0.0, false, P.alp_bh_thresh, gs);
    if (o.fatal) atomicOr(flags, o.fatal);
    pr[GRB_P_CS2] = 0.0;
#pragma unroll
    for (int v = 0; v < 13; ++v) prims[v * n + t] = pr[v];
    if (cons_out) {
#pragma unroll
      for (int v = 0; v < 10; ++v) cons_out[v * n + t] = c[v];
    }
    if (err) err[t] = o.err;
    if (diag.iters) diag.iters[t] = o.iters;
    if (diag.guess_used) diag.guess_used[t] = o.guess_used ? 1 : 0;
    if (diag.mu) diag.mu[t] = o.mu;
    if (diag.bracket) {
      diag.bracket[t] = gs.valid ? gs.lo : 0.0;
      diag.bracket[n + t] = gs.valid ? gs.hi : 0.0;
    }
  }
}

// ---- batched c2p with the entropy backup deferred ------------------------------
// The states whose Kastaun result is distrusted (failed, eps too low, or
// beta = 2P/b^2 <= beta_fallback) take the entropy-based backup solve.  In
// a batch of mixed states nearly every warp holds some, so a one-pass
// kernel runs both solves on every warp.  k_c2p_batch_front runs each
// state up to that decision and finishes the trusted ones; the distrusted
// ones are appended (warp-aggregated) to a list with their intermediate
// state, and k_c2p_batch_backup runs the backup and the rest of the policy
// on the listed states only, every warp of it busy with backups.  Each
// state sees the same operations in the same order as in c2p(): only the
// order in which states are processed changes.
struct C2PDeferred {
  double c[10];
  double pr[13];
  C2PState F;
  int64_t t;
};

template <bool kLearned, bool kFast>
__global__ void __launch_bounds__(kC2PThreads) k_c2p_batch_front(DevParams P, int64_t n,
                                                                const double* __restrict__ cons,
                                                                const double* __restrict__ metric,
                                                                double* __restrict__ prims,
                                                                double* __restrict__ cons_out,
                                                                uint32_t* __restrict__ err, C2PDiagDev diag,
                                                                const MlpSmem* __restrict__ net, uint32_t* flags,
                                                                C2PDeferred* __restrict__ defer,
                                                                unsigned long long* __restrict__ ndefer) {
  __shared__ __align__(16) unsigned char smraw[kLearned ? sizeof(C2PLearnedSmem) : 16];
  C2PLearnedSmem& S = *reinterpret_cast<C2PLearnedSmem*>(smraw);
  if (kLearned) {
    const uint4* src = reinterpret_cast<const uint4*>(net);
    uint4* dst = reinterpret_cast<uint4*>(&S.net);
    for (int w = threadIdx.x; w < (int)(sizeof(MlpSmem) / 16); w += kC2PThreads) dst[w] = src[w];
    __syncthreads();
  }
  const int64_t t = (int64_t)blockIdx.x * kC2PThreads + threadIdx.x;
  const bool active = t < n;
  const int64_t ts = active ? t : 0;
  const Met m = batch_metric(metric, n, ts);
  double c[10], pr[13];
#pragma unroll
  for (int v = 0; v < 10; ++v) c[v] = active ? cons[v * n + t] : 0.0;
  Guess gs = no_guess();
  if (kLearned) {
    float f[kMlpIn];
    __nv_bfloat16 x[kMlpK0];
    const double mu0 = active ? plain_mu0(P.eos, m, c) : 0.0;
    if (active) mlp_features(c, m, mu0, f);
    else {
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) f[k] = S.net.nrm.fmu[k];
    }
    mlp_inputs(S.net.nrm, f, x);
    const float out = mlp_warp32(S.net, S.xs[threadIdx.x >> 5], x);
    gs = mlp_bracket(S.net.nrm, out, mu0);
  }
  C2PState F{};
  if (active) F = c2p_front<kFast>(c, pr, m, P, false, P.alp_bh_thresh, gs);
  const bool later = active && !F.done && F.backup;
  // one slot per deferred lane, one atomic per warp
  const unsigned mask = __ballot_sync(0xffffffffu, later);
  unsigned long long base = 0;
  const int lane = threadIdx.x & 31;
  if (lane == 0 && mask) base = atomicAdd(ndefer, (unsigned long long)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (!active) return;
  if (diag.iters) diag.iters[t] = F.o.iters;
  if (diag.guess_used) diag.guess_used[t] = F.o.guess_used ? 1 : 0;
  if (diag.mu) diag.mu[t] = F.o.mu;
  if (diag.bracket) {
    diag.bracket[t] = gs.valid ? gs.lo : 0.0;
    diag.bracket[n + t] = gs.valid ? gs.hi : 0.0;
  }
  if (later) {
    C2PDeferred& d = defer[base + __popc(mask & ((1u << lane) - 1u))];
#pragma unroll
    for (int v = 0; v < 10; ++v) d.c[v] = c[v];
#pragma unroll
    for (int v = 0; v < 13; ++v) d.pr[v] = pr[v];
    d.F = F;
    d.t = t;
    return;
  }
  if (!F.done) c2p_back<kFast>(F, c, pr, m, P, 0.0);
  if (F.o.fatal) atomicOr(flags, F.o.fatal);
  pr[GRB_P_CS2] = 0.0;
#pragma unroll
  for (int v = 0; v < 13; ++v) prims[v * n + t] = pr[v];
  if (cons_out) {
#pragma unroll
    for (int v = 0; v < 10; ++v) cons_out[v * n + t] = c[v];
  }
  if (err) err[t] = F.o.err;
}

// The listed states: the entropy backup and the rest of the policy
// (grid-stride over the count the front kernel left).
template <bool kFast>
__global__ void __launch_bounds__(kC2PThreads) k_c2p_batch_backup(DevParams P, int64_t n,
                                                                 const double* __restrict__ metric,
                                                                 double* __restrict__ prims,
                                                                 double* __restrict__ cons_out,
                                                                 uint32_t* __restrict__ err, uint32_t* flags,
                                                                 const C2PDeferred* __restrict__ defer,
                                                                 const unsigned long long* __restrict__ ndefer) {
  const int64_t nd = (int64_t)*ndefer;
  for (int64_t e = (int64_t)blockIdx.x * kC2PThreads + threadIdx.x; e < nd; e += (int64_t)gridDim.x * kC2PThreads) {
    const C2PDeferred& d = defer[e];
    double c[10], pr[13];
#pragma unroll
    for (int v = 0; v < 10; ++v) c[v] = d.c[v];
#pragma unroll
    for (int v = 0; v < 13; ++v) pr[v] = d.pr[v];
    C2PState F = d.F;
    const int64_t t = d.t;
    const Met m = batch_metric(metric, n, t);
    c2p_backup(F, c, pr, m, P);
    c2p_back<kFast>(F, c, pr, m, P, 0.0);
    if (F.o.fatal) atomicOr(flags, F.o.fatal);
    pr[GRB_P_CS2] = 0.0;
#pragma unroll
    for (int v = 0; v < 13; ++v) prims[v * n + t] = pr[v];
    if (cons_out) {
#pragma unroll
      for (int v = 0; v < 10; ++v) cons_out[v * n + t] = c[v];
    }
    if (err) err[t] = F.o.err;
  }
}

// ---- training data ----------------------------------------------------------
// Raw features [6][n] and target y = asinh(log(mu0 / mu) / L0) [n] (NaN where
// the plain c2p did not reach the Kastaun solve) from the states and the
// plain roots.
__global__ void __launch_bounds__(256) k_mlp_labels(DevParams P, int64_t n, const double* __restrict__ cons,
                                                    const double* __restrict__ metric,
                                                    const double* __restrict__ mu, float* __restrict__ feat,
                                                    float* __restrict__ tgt) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const Met m = batch_metric(metric, n, t);
    double c[10];
#pragma unroll
    for (int v = 0; v < 10; ++v) c[v] = cons[v * n + t];
    const double mu0 = plain_mu0(P.eos, m, c);
    float f[kMlpIn];
    mlp_features(c, m, mu0, f);
    bool ok = mu0 > 0.0;
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) {
      feat[k * n + t] = f[k];
      ok = ok && isfinite(f[k]);
    }
    const double u = mu ? mu[t] : 0.0;
    tgt[t] = (ok && u > 0.0 && isfinite(u)) ? (float)asinh((log(mu0) - log(u)) / kMlpL0)
                                            : __int_as_float(0x7fc00000);
  }
}

// Per-CTA sums of features, squares, targets and counts over valid samples
// (fixed grid, reduced on the host in CTA order: reproducible).
constexpr int kStatN = 2 * kMlpIn + 3;
constexpr int kStatBlocks = 256;
__global__ void __launch_bounds__(256) k_mlp_stats(int64_t n, const float* __restrict__ feat,
                                                   const float* __restrict__ tgt, double* __restrict__ part) {
  double acc[kStatN];
#pragma unroll
  for (int a = 0; a < kStatN; ++a) acc[a] = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const float y = tgt[t];
    if (!isfinite(y)) continue;
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) {
      const double f = feat[k * n + t];
      acc[k] += f;
      acc[kMlpIn + k] += f * f;
    }
    acc[2 * kMlpIn] += y;
    acc[2 * kMlpIn + 1] += (double)y * y;
    acc[2 * kMlpIn + 2] += 1.0;
  }
  __shared__ double red[kStatN][8];
#pragma unroll
  for (int a = 0; a < kStatN; ++a) {
    double v = acc[a];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[a][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < kStatN) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
    part[blockIdx.x * kStatN + threadIdx.x] = v;
  }
}

// ---- gradient of the batch loss -------------------------------------------
// loss = sum_s w_s (y_s - t_s)^2 with w_s = inv_count for valid samples,
// y and t normalised.
constexpr int kGradRows = 64;            // states per CTA
constexpr int kGradThreads = 256;
constexpr int kSP = kGradRows + 1;       // pitch of the [feature][state] arrays
constexpr int kPW = kMlpNumWeights + 1;  // partial row: gradient, then loss

struct MlpGradSmem {
  MlpSmem net;
  __nv_bfloat16 xs[kGradRows * kXP];
  float X[kMlpK0 * kSP];
  float H[3 * kMlpH * kSP];
  float DA[kMlpH * kSP], DB[kMlpH * kSP];
  float y[kGradRows], g[kGradRows], l[kGradRows];
};

// dW[o][i] = sum_s D[o][s] Hp[i][s], db[o] = sum_s D[o][s]; thread -> (o, 16 i)
__device__ __forceinline__ void mlp_wgrad64(const float* D, const float* Hp, float* gW, float* gb) {
  const int o = threadIdx.x >> 2, q = threadIdx.x & 3;
  float acc[16], db = 0.f;
#pragma unroll
  for (int j = 0; j < 16; ++j) acc[j] = 0.f;
  for (int s = 0; s < kGradRows; ++s) {
    const float d = D[o * kSP + s];
    db += d;
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[j] = fmaf(d, Hp[(q + 4 * j) * kSP + s], acc[j]);
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) gW[o * kMlpH + q + 4 * j] = acc[j];
  if (q == 0) gb[o] = db;
}
__device__ __forceinline__ void mlp_wgrad16(const float* D, const float* X, float* gW, float* gb) {
  const int o = threadIdx.x >> 2, q = threadIdx.x & 3;
  float acc[4], db = 0.f;
#pragma unroll
  for (int j = 0; j < 4; ++j) acc[j] = 0.f;
  for (int s = 0; s < kGradRows; ++s) {
    const float d = D[o * kSP + s];
    db += d;
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j] = fmaf(d, X[(q + 4 * j) * kSP + s], acc[j]);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) gW[o * kMlpK0 + q + 4 * j] = acc[j];
  if (q == 0) gb[o] = db;
}
// Dout[i][s] = [Hp[i][s] > 0] sum_o W[o][i] D[o][s]; thread -> (s, 16 i)
__device__ __forceinline__ void mlp_backdelta(const __nv_bfloat16* W, const float* D, const float* Hp, float* Dout) {
  const int s = threadIdx.x & (kGradRows - 1), i0 = (threadIdx.x >> 6) * 16;
  float acc[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) acc[j] = 0.f;
  for (int o = 0; o < kMlpH; ++o) {
    const float d = D[o * kSP + s];
    const __nv_bfloat162* w2 = reinterpret_cast<const __nv_bfloat162*>(W + o * kPH + i0);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float2 w = __bfloat1622float2(w2[j]);
      acc[2 * j] = fmaf(w.x, d, acc[2 * j]);
      acc[2 * j + 1] = fmaf(w.y, d, acc[2 * j + 1]);
    }
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int i = i0 + j;
    Dout[i * kSP + s] = Hp[i * kSP + s] > 0.f ? acc[j] : 0.f;
  }
}

// One CTA: kGradRows states -> one partial gradient row part[blockIdx.x][kPW].
// identity != 0: state j of the batch is sample j (gradient checks);
// otherwise sample hash(seed, step, j) mod n, drawn with replacement.
__global__ void __launch_bounds__(kGradThreads) k_mlp_grad(const float* __restrict__ P, int64_t n,
                                                           const float* __restrict__ feat,
                                                           const float* __restrict__ tgt, int64_t nbatch,
                                                           uint64_t seed, int64_t step, int identity,
                                                           float inv_count, float* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smraw[];
  MlpGradSmem& S = *reinterpret_cast<MlpGradSmem*>(smraw);
  const int tid = threadIdx.x;
  mlp_load_smem(S.net, P);
  __syncthreads();
  if (tid < kGradRows) {
    const int64_t j = (int64_t)blockIdx.x * kGradRows + tid;
    int64_t gi = -1;
    if (j < nbatch)
      gi = identity ? j
                    : (int64_t)(mix64(seed ^ mix64((uint64_t)step * 0x100000001B3ull + (uint64_t)j)) %
                                (uint64_t)n);
    const float t = (gi >= 0 && gi < n) ? tgt[gi] : __int_as_float(0x7fc00000);
    const bool ok = isfinite(t);
    float f[kMlpIn];
    __nv_bfloat16 x[kMlpK0];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) f[k] = ok ? feat[k * n + gi] : S.net.nrm.fmu[k];
    mlp_inputs(S.net.nrm, f, x);
#pragma unroll
    for (int k = 0; k < kMlpK0; ++k) {
      S.xs[tid * kXP + k] = x[k];
      S.X[k * kSP + tid] = __bfloat162float(x[k]);
    }
    S.g[tid] = ok ? 1.f : 0.f;
    S.y[tid] = ok ? __fdiv_rn(t - S.net.nrm.tmu, S.net.nrm.tsd) : 0.f;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  if (warp < kGradRows / 16) {
    float lo, hi;
    mlp_tile16<true>(S.net, S.xs + warp * 16 * kXP, lo, hi, S.H, warp * 16, kSP);
    if ((lane & 3) == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int R = warp * 16 + (lane >> 2) + 8 * h;
        const float out = h ? hi : lo;
        const bool ok = S.g[R] != 0.f;
        const float e = out - S.y[R];
        S.g[R] = ok ? 2.f * inv_count * e : 0.f;
        S.l[R] = ok ? inv_count * e * e : 0.f;
      }
    }
  }
  __syncthreads();
  float* pg = part + (int64_t)blockIdx.x * kPW;
  const float* H1 = S.H;
  const float* H2 = S.H + kMlpH * kSP;
  const float* H3 = S.H + 2 * kMlpH * kSP;
  for (int e = tid; e < kMlpH * kGradRows; e += kGradThreads) {
    const int o = e >> 6, s = e & (kGradRows - 1);
    S.DA[o * kSP + s] = H3[o * kSP + s] > 0.f ? S.g[s] * S.net.w4[o] : 0.f;
  }
  if (tid < kMlpH) {
    float a = 0.f;
    for (int s = 0; s < kGradRows; ++s) a = fmaf(S.g[s], H3[tid * kSP + s], a);
    pg[kMlpOffW4 + tid] = a;
  } else if (tid == kMlpH) {
    float a = 0.f;
    for (int s = 0; s < kGradRows; ++s) a += S.g[s];
    pg[kMlpOffB4] = a;
  } else if (tid == kMlpH + 1) {
    float a = 0.f;
    for (int s = 0; s < kGradRows; ++s) a += S.l[s];
    pg[kMlpNumWeights] = a;
  }
  __syncthreads();
  mlp_wgrad64(S.DA, H2, pg + kMlpOffW3, pg + kMlpOffB3);
  mlp_backdelta(S.net.W3, S.DA, H2, S.DB);
  __syncthreads();
  mlp_wgrad64(S.DB, H1, pg + kMlpOffW2, pg + kMlpOffB2);
  mlp_backdelta(S.net.W2, S.DB, H1, S.DA);
  __syncthreads();
  mlp_wgrad16(S.DA, S.X, pg + kMlpOffW1, pg + kMlpOffB1);
}

// Sum of the partial rows in CTA order -> grad[kPW] (gradient, then loss).
__global__ void __launch_bounds__(256) k_mlp_reduce(const float* __restrict__ part, int nparts,
                                                    float* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kPW) return;
  float g = 0.f;
  for (int c = 0; c < nparts; ++c) g += part[(int64_t)c * kPW + p];
  grad[p] = g;
}

// Adam (Kingma & Ba 2015) on the trainable block; the loss of the step goes
// to loss_hist[step].  bc1, bc2: bias corrections 1 - beta^t.
__global__ void __launch_bounds__(256) k_mlp_adam(float* __restrict__ P, float* __restrict__ m1,
                                                  float* __restrict__ m2, const float* __restrict__ part,
                                                  int nparts, float lr, float bc1, float bc2,
                                                  float* __restrict__ loss_hist, int64_t step) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kPW) return;
  float g = 0.f;
  for (int c = 0; c < nparts; ++c) g += part[(int64_t)c * kPW + p];
  if (p == kMlpNumWeights) {
    if (loss_hist) loss_hist[step] = g;
    return;
  }
  const float a = 0.9f * m1[p] + 0.1f * g;
  const float b = 0.999f * m2[p] + 0.001f * g * g;
  m1[p] = a;
  m2[p] = b;
  P[p] -= lr * (a / bc1) / (sqrtf(b / bc2) + 1e-8f);
}

// Network outputs (y, denormalised) for n raw feature rows [6][n].
__global__ void __launch_bounds__(kC2PThreads) k_mlp_eval(const float* __restrict__ P, int64_t n,
                                                          const float* __restrict__ feat, float* __restrict__ out) {
  __shared__ __align__(16) C2PLearnedSmem S;
  mlp_load_smem(S.net, P);
  __syncthreads();
  for (int64_t base = (int64_t)blockIdx.x * kC2PThreads; base < n; base += (int64_t)gridDim.x * kC2PThreads) {
    const int64_t t = base + threadIdx.x;
    float f[kMlpIn];
    __nv_bfloat16 x[kMlpK0];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) f[k] = t < n ? feat[k * n + t] : S.net.nrm.fmu[k];
    mlp_inputs(S.net.nrm, f, x);
    const float y = mlp_warp32(S.net, S.xs[threadIdx.x >> 5], x);
    if (t < n) out[t] = fmaf(y, S.net.nrm.tsd, S.net.nrm.tmu);
  }
}

}  // namespace grb
