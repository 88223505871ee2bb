// CPU oracle of the learned c2p bracket network — test infrastructure only.
//
// The network has no counterpart in the reference; what the reference fixes
// is its input and its label: the Kastaun scalars (kastaun_c2p.hh:306-337),
// the top mu0 of the plain bracket (kastaun_c2p.hh:355-369) and the root mu
// of the Kastaun master function (kastaun_c2p.hh:245-290), all from
// c2p_oracle.hpp's restatement.  The label is L = log(mu0/mu).  This file
// restates the library's forward pass and its gradient in FP64:
//   * emulate_bf16 = 1: the rounding points of the tensor-core forward
//     (normalised inputs split into a BF16 high part and a BF16 remainder,
//     W1..W3 and the three hidden activations rounded to BF16
//     round-to-nearest-even; the gradient passes straight through the
//     rounding), for GPU-vs-CPU checks;
//   * emulate_bf16 = 0: plain FP64 arithmetic (the high part is the
//     normalised input, the remainder zero), whose gradient the tests pin by
//     central finite differences.
// Parameter layout: W1[64][16] b1[64] W2[64][64] b2[64] W3[64][64] b3[64]
// w4[64] b4, then fmu[6] fsd[6] tmu tsd delta.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "c2p_oracle.hpp"

namespace orc {
namespace mlp {

constexpr int kIn = 6, kK0 = 16, kH = 64;
constexpr int oW1 = 0, oB1 = oW1 + kH * kK0, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH * kH, oW4 = oB3 + kH, oB4 = oW4 + kH, kNW = oB4 + 1, oNorm = kNW,
              kNP = oNorm + 2 * kIn + 3;

// float -> bfloat16 -> float, round to nearest even (finite inputs)
inline float bf16(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  u &= 0xFFFF0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// Top of the plain Kastaun bracket of a state (densitized cons), 0 for D <= 0.
inline double plain_mu0(const Eos& e, const Metric& m, const double c[10]) {
  double cc[10];
  for (int v = 0; v < 10; ++v) cc[v] = c[v] / m.sqrtg;
  if (!(cc[0] > 0.0)) return 0.0;
  const KScalars k = kastaun_setup(e, m, cc);
  return kastaun_mu0(k);
}

// Features of one state from densitized cons (as the c2p receives them).
inline void features(const double c[10], const Metric& m, double mu0, float f[kIn]) {
  const double isg = 1.0 / m.sqrtg;
  const double D = std::fmax(c[0] * isg, 1e-30);
  const double iD = 1.0 / D;
  const double q = c[4] * isg * iD;
  const double r[3] = {c[1] * isg * iD, c[2] * isg * iD, c[3] * isg * iD};
  const double isD = isg / std::sqrt(D);
  const double Bt[3] = {c[7] * isD, c[8] * isD, c[9] * isD};
  const double r2 = sq_sym(m.ginv, r);
  const double b2 = sq_sym(m.g, Bt);
  const double rb = r[0] * Bt[0] + r[1] * Bt[1] + r[2] * Bt[2];
  f[0] = std::log10((float)D);
  f[1] = std::log10((float)std::fmax(q, 1e-30));
  f[2] = 0.5f * std::log10((float)(r2 + 1e-30));
  f[3] = std::log10((float)(b2 + 1e-30));
  f[4] = (float)std::fmin(1.0, std::fmax(0.0, rb * rb / (r2 * b2 + 1e-300)));
  f[5] = (float)std::log(std::fmax(mu0, 1e-300));
}

struct Net {
  // weights as the forward uses them (rounded when emulating BF16)
  std::vector<double> W1, W2, W3, b1, b2, b3, w4;
  double b4;
  float fmu[kIn], fsd[kIn], tmu, tsd;
  bool emu;
  Net(const float* P, bool emulate) : W1(kH * kK0), W2(kH * kH), W3(kH * kH), b1(kH), b2(kH), b3(kH), w4(kH),
                                      emu(emulate) {
    auto w = [&](float v) { return (double)(emu ? bf16(v) : v); };
    for (int t = 0; t < kH * kK0; ++t) W1[t] = w(P[oW1 + t]);
    for (int t = 0; t < kH * kH; ++t) { W2[t] = w(P[oW2 + t]); W3[t] = w(P[oW3 + t]); }
    for (int t = 0; t < kH; ++t) {
      b1[t] = P[oB1 + t]; b2[t] = P[oB2 + t]; b3[t] = P[oB3 + t]; w4[t] = P[oW4 + t];
    }
    b4 = P[oB4];
    for (int k = 0; k < kIn; ++k) { fmu[k] = P[oNorm + k]; fsd[k] = P[oNorm + kIn + k]; }
    tmu = P[oNorm + 2 * kIn];
    tsd = P[oNorm + 2 * kIn + 1];
  }
  double act(double a) const {
    const double h = a > 0 ? a : 0.0;
    return emu ? (double)bf16((float)h) : h;
  }
  // forward of one sample; x[16], h1..h3[64] out; returns normalised output
  double forward(const float f[kIn], double x[kK0], double h1[kH], double h2[kH], double h3[kH]) const {
    for (int k = 0; k < kK0; ++k) x[k] = 0.0;
    for (int k = 0; k < kIn; ++k) {
      const float d = f[k] - fmu[k];
      const float v = d / fsd[k];
      if (emu) {
        const float hi = bf16(v);
        x[k] = hi;
        x[kIn + k] = bf16(v - hi);
      } else {
        x[k] = v;
      }
    }
    for (int o = 0; o < kH; ++o) {
      double a = 0.0;
      for (int k = 0; k < kK0; ++k) a += W1[o * kK0 + k] * x[k];
      h1[o] = act(a + b1[o]);
    }
    for (int o = 0; o < kH; ++o) {
      double a = 0.0;
      for (int i = 0; i < kH; ++i) a += W2[o * kH + i] * h1[i];
      h2[o] = act(a + b2[o]);
    }
    for (int o = 0; o < kH; ++o) {
      double a = 0.0;
      for (int i = 0; i < kH; ++i) a += W3[o * kH + i] * h2[i];
      h3[o] = act(a + b3[o]);
    }
    double y = b4;
    for (int o = 0; o < kH; ++o) y += w4[o] * h3[o];
    return y;
  }
};

// Mean-squared-error loss over n samples (NaN targets contribute nothing but
// count in the mean) and its gradient grad[kNW] with respect to the
// trainable parameters; returns the loss.
inline double loss_grad(const float* P, int64_t n, const float* feat, const float* tgt, int emulate,
                        double* grad) {
  const Net net(P, emulate != 0);
  if (grad)
    for (int p = 0; p < kNW; ++p) grad[p] = 0.0;
  double loss = 0.0;
  const double inv = 1.0 / (double)n;
  double x[kK0], h1[kH], h2[kH], h3[kH], d1[kH], d2[kH], d3[kH];
  for (int64_t s = 0; s < n; ++s) {
    if (!std::isfinite(tgt[s])) continue;
    float f[kIn];
    for (int k = 0; k < kIn; ++k) f[k] = feat[k * n + s];
    const double y = net.forward(f, x, h1, h2, h3);
    const float tn = (tgt[s] - net.tmu) / net.tsd;
    const double e = y - (double)tn;
    loss += inv * e * e;
    if (!grad) continue;
    const double g = 2.0 * inv * e;
    grad[oB4] += g;
    for (int o = 0; o < kH; ++o) {
      grad[oW4 + o] += g * h3[o];
      d3[o] = h3[o] > 0 ? g * net.w4[o] : 0.0;
      grad[oB3 + o] += d3[o];
      for (int i = 0; i < kH; ++i) grad[oW3 + o * kH + i] += d3[o] * h2[i];
    }
    for (int i = 0; i < kH; ++i) {
      double a = 0.0;
      for (int o = 0; o < kH; ++o) a += net.W3[o * kH + i] * d3[o];
      d2[i] = h2[i] > 0 ? a : 0.0;
    }
    for (int o = 0; o < kH; ++o) {
      grad[oB2 + o] += d2[o];
      for (int i = 0; i < kH; ++i) grad[oW2 + o * kH + i] += d2[o] * h1[i];
    }
    for (int i = 0; i < kH; ++i) {
      double a = 0.0;
      for (int o = 0; o < kH; ++o) a += net.W2[o * kH + i] * d2[o];
      d1[i] = h1[i] > 0 ? a : 0.0;
    }
    for (int o = 0; o < kH; ++o) {
      grad[oB1 + o] += d1[o];
      for (int k = 0; k < kK0; ++k) grad[oW1 + o * kK0 + k] += d1[o] * x[k];
    }
  }
  return loss;
}

}  // namespace mlp
}  // namespace orc

extern "C" {

int orc_mlp_num_params() { return orc::mlp::kNP; }

// features [6][n] of n states (metric [10][n] or NULL = flat)
void orc_mlp_features(const grb_params* p, int64_t n, const double* cons, const double* metric, float* feat) {
  const orc::Eos eos = orc::make_eos(p->eos);
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < n; ++t) {
    double g[6] = {1, 0, 0, 1, 0, 1}, b[3] = {0, 0, 0}, alp = 1.0;
    if (metric) {
      for (int a = 0; a < 6; ++a) g[a] = metric[a * n + t];
      for (int a = 0; a < 3; ++a) b[a] = metric[(6 + a) * n + t];
      alp = metric[9 * n + t];
    }
    const orc::Metric m = orc::make_metric(g, b, alp);
    double c[10];
    for (int v = 0; v < 10; ++v) c[v] = cons[v * n + t];
    float f[orc::mlp::kIn];
    orc::mlp::features(c, m, orc::mlp::plain_mu0(eos, m, c), f);
    for (int k = 0; k < orc::mlp::kIn; ++k) feat[k * n + t] = f[k];
  }
}

// network output L (denormalised) of n feature rows
void orc_mlp_forward(const float* P, int64_t n, const float* feat, int32_t emulate, double* out) {
  const orc::mlp::Net net(P, emulate != 0);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < n; ++s) {
    double x[orc::mlp::kK0], h1[orc::mlp::kH], h2[orc::mlp::kH], h3[orc::mlp::kH];
    float f[orc::mlp::kIn];
    for (int k = 0; k < orc::mlp::kIn; ++k) f[k] = feat[k * n + s];
    out[s] = net.forward(f, x, h1, h2, h3) * (double)net.tsd + (double)net.tmu;
  }
}

double orc_mlp_loss_grad(const float* P, int64_t n, const float* feat, const float* tgt, int32_t emulate,
                         double* grad) {
  return orc::mlp::loss_grad(P, n, feat, tgt, emulate, grad);
}

// conservs_to_prims with a per-state starting bracket [lo[t], hi[t]]
// (lo[t] <= 0: no bracket); iters, guess_used, mu out (each may be NULL).
int orc_c2p_batch_guess(const grb_params* p, int64_t n, const double* cons, const double* metric,
                        const double* lo, const double* hi, double* prims, double* cons_out, uint32_t* err,
                        int32_t* iters, int8_t* guess_used, double* mu) {
  const orc::Eos eos = orc::make_eos(p->eos);
  const orc::C2PParams cp = orc::make_c2p_params(*p);
  int fatal_all = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : fatal_all)
  for (int64_t t = 0; t < n; ++t) {
    double g[6] = {1, 0, 0, 1, 0, 1}, b[3] = {0, 0, 0}, alp = 1.0;
    if (metric) {
      for (int a = 0; a < 6; ++a) g[a] = metric[a * n + t];
      for (int a = 0; a < 3; ++a) b[a] = metric[(6 + a) * n + t];
      alp = metric[9 * n + t];
    }
    const orc::Metric m = orc::make_metric(g, b, alp);
    double c[10], pr[13] = {0};
    for (int v = 0; v < 10; ++v) c[v] = cons[v * n + t];
    orc::BracketGuess gs;
    gs.valid = lo && hi && lo[t] > 0.0 && hi[t] > lo[t];
    gs.lo = gs.valid ? lo[t] : 0.0;
    gs.hi = gs.valid ? hi[t] : 0.0;
    orc::C2PStats st;
    uint32_t e = 0;
    int fat = 0;
    orc::conservs_to_prims(c, pr, m, eos, cp, 0.0, e, false, fat, &st, &gs);
    fatal_all |= fat;
    for (int v = 0; v < 13; ++v) prims[v * n + t] = pr[v];
    if (cons_out)
      for (int v = 0; v < 10; ++v) cons_out[v * n + t] = c[v];
    if (err) err[t] = e;
    if (iters) iters[t] = st.brent_iters;
    if (guess_used) guess_used[t] = (int8_t)st.guess_used;
    if (mu) mu[t] = st.mu;
  }
  return fatal_all;
}

}  // extern "C"
