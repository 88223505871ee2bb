// Device-side GRMHD numerics for sm_100a (FP64 throughout).
//
// Per-cell physics of GRACE's Cowling GRMHD path, written for the GPU: all
// state lives in registers, structs are passed by value, and the EOS is a
// runtime switch instead of a template.  References (paths relative to the
// GRACE source tree):
//   EOS .............. include/grace/physics/eos/{hybrid,ideal_gas,piecewise_polytropic}_eos.hh
//   metric ........... include/grace/utils/metric_utils.hh:48-82
//   W, b^mu, vtilde .. include/grace/physics/grmhd_subexpressions.hh:10-57
//   char. speeds ..... include/grace/physics/grmhd_subexpressions.hh:59-95
//   cons / fluxes .... include/grace/physics/grmhd_subexpressions.hh:97-156, 294-331
//   sources .......... include/grace/physics/grmhd_subexpressions.hh:158-292
//   WENO-Z, limiters . include/grace/utils/{weno_reconstruction,reconstruction,limiters}.hh
//   HLLE ............. include/grace/utils/riemann_solvers.hh:60-70
//   Brent, Newton .... include/grace/utils/rootfinding.hh:73-306
//   Kastaun c2p ...... include/grace/physics/eos/kastaun_c2p.hh:44-402
//   entropy backup ... include/grace/physics/eos/ent_based_c2p.hh:44-260
//   c2p policy ....... src/physics/eos/c2p.cpp:40-455, include/grace/physics/eos/c2p.hh:124-316
// Branch decisions (clamps, signal bits, acceptance tests) follow the
// reference step by step; the algebra is written from the standard GRMHD
// formulas and agrees with the reference to rounding.
#pragma once
#include <cstdint>

#include "grace_b200.h"

namespace grb {

#define GRB_HD __device__ __forceinline__

// ---- bit layouts (c2p.hh:44-121, eos_base.hh:40-54) -----------------------
enum : uint32_t {
  SIG_EPS_HIGH = 1u << 0, SIG_EPS_LOW = 1u << 1, SIG_RHO_HIGH = 1u << 4,
  SIG_RHO_LOW = 1u << 5, SIG_ENT_LOW = 1u << 6, SIG_ENT_HIGH = 1u << 7,
  SIG_VEL_HIGH = 1u << 8, SIG_SIGMA_HIGH = 1u << 9
};
enum : uint32_t {
  ERR_RESET_DENS = 1u << 0, ERR_RESET_TAU = 1u << 1, ERR_RESET_STILDE = 1u << 2,
  ERR_RESET_ENTROPY = 1u << 3, ERR_RESET_YE = 1u << 4,
  ERR_SIG_RHO_LOW = 1u << 5, ERR_SIG_RHO_HIGH = 1u << 6, ERR_SIG_EPS_LOW = 1u << 7,
  ERR_SIG_EPS_HIGH = 1u << 8, ERR_SIG_ENT_LOW = 1u << 11, ERR_SIG_ENT_HIGH = 1u << 12,
  ERR_SIG_TEMP_LOW = 1u << 13, ERR_SIG_TEMP_HIGH = 1u << 14, ERR_SIG_PRESS_LOW = 1u << 15,
  ERR_SIG_PRESS_HIGH = 1u << 16, ERR_SIG_VEL_HIGH = 1u << 17, ERR_SIG_SIGMA_HIGH = 1u << 18,
  ERR_ENT_BACKUP = 1u << 19, ERR_ATMO = 1u << 20, ERR_T_FLOORED = 1u << 21
};
enum : uint32_t {
  EOS_RHO_HIGH = 1u << 0, EOS_RHO_LOW = 1u << 1, EOS_EPS_HIGH = 1u << 2, EOS_EPS_LOW = 1u << 3,
  EOS_TEMP_LOW = 1u << 6, EOS_TEMP_HIGH = 1u << 7, EOS_ENT_LOW = 1u << 8, EOS_ENT_HIGH = 1u << 9,
  EOS_PRESS_LOW = 1u << 10, EOS_PRESS_HIGH = 1u << 11
};
constexpr uint32_t ERR_ALL_RESETS =
    ERR_RESET_DENS | ERR_RESET_TAU | ERR_RESET_STILDE | ERR_RESET_ENTROPY | ERR_RESET_YE;

// ---- parameters as the kernels see them -----------------------------------
struct DevEos {
  int kind, n;
  double rhomax, rhomin, tempmax, yemax, eps_max, h_min;
  double gm1, g, ggm1, ent_min;        // ideal gas
  double gthm1, entropy_min;           // hybrid thermal part
  double igm1, ih0;                    // 1/gm1 (ideal gas), 1/h_min
  double K[GRB_MAX_PIECES], G[GRB_MAX_PIECES], R[GRB_MAX_PIECES], E[GRB_MAX_PIECES];
};
struct DevParams {
  DevEos eos;
  double rho_fl, ye_fl, temp_fl, atmo_tol;
  int excise_by_radius;
  double r_ex, alp_ex;
  double tol, max_w, max_sigma, beta_fallback, alp_bh_thresh;
  int use_ent_backup;
  double rusanov_c_limit;
  int fofc, dmp_enable;
  double dmp_M;
  int recon, riemann, emf;
};

// ---- metric ---------------------------------------------------------------
// isqrtg, ialp: 1/sqrt(gamma) and 1/alpha, set by make_met<true> (tuned
// mode) only.
struct Met {
  double g[6], beta[3], alp, gi[6], sqrtg, isqrtg, ialp;
};
// FAST (tuned mode): 1/sqrt(gamma) = rsqrt(det), sqrt(gamma) = det / sqrt(det)
// and 1/det = (1/sqrt(gamma))^2, so no square root and one division (1/alpha).
template <bool FAST = false>
GRB_HD Met make_met(const double g[6], const double b[3], double alp) {
  Met m;
#pragma unroll
  for (int a = 0; a < 6; ++a) m.g[a] = g[a];
#pragma unroll
  for (int a = 0; a < 3; ++a) m.beta[a] = b[a];
  m.alp = alp;
  const double c0 = g[3] * g[5] - g[4] * g[4];
  const double c1 = g[2] * g[4] - g[1] * g[5];
  const double c2 = g[1] * g[4] - g[2] * g[3];
  const double det = g[0] * c0 + g[1] * c1 + g[2] * c2;
  double id, isg = 0.0;
  if (FAST) {
    isg = rsqrt(det);
    id = isg * isg;
    m.ialp = 1.0 / alp;
  } else {
    id = 1.0 / det;
    m.ialp = 0.0;
  }
  m.gi[0] = c0 * id;
  m.gi[1] = c1 * id;
  m.gi[2] = c2 * id;
  m.gi[3] = (g[0] * g[5] - g[2] * g[2]) * id;
  m.gi[4] = (g[1] * g[2] - g[0] * g[4]) * id;
  m.gi[5] = (g[0] * g[3] - g[1] * g[1]) * id;
  m.sqrtg = FAST ? det * isg : sqrt(det);
  m.isqrtg = isg;
  return m;
}
GRB_HD double sqs(const double s[6], const double v[3]) {
  return s[0] * v[0] * v[0] + s[3] * v[1] * v[1] + s[5] * v[2] * v[2] +
         2. * (s[1] * v[0] * v[1] + s[2] * v[0] * v[2] + s[4] * v[1] * v[2]);
}
GRB_HD void mvs(const double s[6], const double v[3], double o[3]) {
  o[0] = s[0] * v[0] + s[1] * v[1] + s[2] * v[2];
  o[1] = s[1] * v[0] + s[3] * v[1] + s[4] * v[2];
  o[2] = s[2] * v[0] + s[4] * v[1] + s[5] * v[2];
}

// ---- EOS ------------------------------------------------------------------
GRB_HD int pw_idx(const DevEos& e, double& rho) {
  rho = fmax(e.rhomin, fmin(e.rhomax, rho));
  for (int ii = 0; ii < e.n - 1; ++ii)
    if (rho > e.R[ii] && rho <= e.R[ii + 1]) return ii;
  return e.n - 1;
}
// rho^G of the cold polytrope.  G = 2 (the usual neutron-star index) and
// G = 1 are exact products, rho*rho being the correctly rounded square;
// other indices call pow.  The branch is uniform: G is a run constant.
GRB_HD double pw_pow(double rho, double G) {
  if (G == 2.0) return rho * rho;
  if (G == 1.0) return rho;
  return pow(rho, G);
}
GRB_HD double pw_cold(const DevEos& e, double& ec, double& rho) {
  const int i = pw_idx(e, rho);
  const double pc = e.K[i] * pw_pow(rho, e.G[i]);
  ec = e.E[i] + pc / (rho * (e.G[i] - 1.));
  return pc;
}
GRB_HD double pw_dpdrho(const DevEos& e, double& rho) {
  const int i = pw_idx(e, rho);
  return e.G[i] * (e.K[i] * pw_pow(rho, e.G[i])) / rho;
}
GRB_HD void hy_rho(const DevEos& e, double& rho, uint32_t& q) {
  if (rho < e.rhomin) { q |= EOS_RHO_LOW; rho = e.rhomin; }
  if (rho > e.rhomax) { q |= EOS_RHO_HIGH; rho = e.rhomax; }
}
GRB_HD void hy_temp(const DevEos& e, double& t, uint32_t& q) {
  if (t < 0.0) { q |= EOS_TEMP_LOW; t = 0.0; }
  if (t > e.tempmax) { q |= EOS_TEMP_HIGH; t = e.tempmax; }
}
GRB_HD void hy_eps(const DevEos& e, double& eps, double ec, uint32_t& q) {
  const double lo = fmin(ec, e.eps_max);
  if (eps < lo) { q |= EOS_EPS_LOW; eps = lo; }
  if (eps > e.eps_max) { q |= EOS_EPS_HIGH; eps = e.eps_max; }
}
GRB_HD double hy_ent(const DevEos& e, double eth, double rho) {
  return log(fmax(eth, e.entropy_min) * pow(rho, -e.gthm1)) / e.gthm1;
}
GRB_HD void id_eps(const DevEos& e, double& eps, uint32_t& q) {
  if (eps > e.eps_max) { q |= EOS_EPS_HIGH; eps = e.eps_max; }
  if (eps < 0.0) { q |= EOS_EPS_LOW; eps = 0.0; }
}
GRB_HD void id_temp(const DevEos& e, double& t, uint32_t& q) {
  const double tmax = e.eps_max * e.gm1;
  if (t < 0.0) { t = 0.0; q |= EOS_TEMP_LOW; }
  if (t > tmax) { q |= EOS_TEMP_HIGH; t = tmax; }
}
GRB_HD double id_ent(const DevEos& e, double eps, double rho) { return log(eps) / e.gm1 - log(rho); }

// P, eps, cs2 (and optionally s) from (T, rho): hybrid_eos.hh:224-291,
// ideal_gas_eos.hh:233-288.  T and rho are clamped in place.
GRB_HD double eos_PT(const DevEos& e, double& eps, double& cs2, double* ent, double& t,
                     double& rho, uint32_t& q) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_temp(e, t, q);
    eps = t / e.gm1;
    const double p = e.gm1 * eps * rho;
    cs2 = e.ggm1 * eps / (1.0 + e.g * eps);
    if (ent) *ent = id_ent(e, eps, rho);
    return p;
  }
  hy_rho(e, rho, q);
  hy_temp(e, t, q);
  double ec;
  const double pc = pw_cold(e, ec, rho);
  const double eth = fmax(0.0, t / e.gthm1);
  const double p = pc + eth * rho * e.gthm1;
  eps = ec + eth;
  const double h = 1. + eps + p / rho;
  cs2 = (pw_dpdrho(e, rho) + e.gthm1 * (e.gthm1 + 1) * eth) / h;
  if (ent) *ent = hy_ent(e, eth, rho);
  return p;
}
// eos_PT for the two reconstructed states of a face (tuned mode; states
// in the local primitive layout, no entropy): for the ideal gas
// eps = T * (1/(Gamma-1)) and both sound speeds from one reciprocal of
// (1 + Gamma eps_l)(1 + Gamma eps_r) (both >= 1); the hybrid EOS calls
// eos_PT per state.
GRB_HD void eos_PT_pair_f(const DevEos& e, double* pl, double* pr) {
  uint32_t q0 = 0;
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_temp(e, pl[GRB_P_TEMP], q0);
    id_temp(e, pr[GRB_P_TEMP], q0);
    const double el = pl[GRB_P_TEMP] * e.igm1, er = pr[GRB_P_TEMP] * e.igm1;
    pl[GRB_P_EPS] = el;
    pr[GRB_P_EPS] = er;
    pl[GRB_P_PRESS] = e.gm1 * el * pl[GRB_P_RHO];
    pr[GRB_P_PRESS] = e.gm1 * er * pr[GRB_P_RHO];
    const double dl = 1.0 + e.g * el, dr = 1.0 + e.g * er;
    const double r = 1.0 / (dl * dr);
    pl[GRB_P_CS2] = e.ggm1 * el * dr * r;
    pr[GRB_P_CS2] = e.ggm1 * er * dl * r;
    return;
  }
  pl[GRB_P_PRESS] = eos_PT(e, pl[GRB_P_EPS], pl[GRB_P_CS2], nullptr, pl[GRB_P_TEMP], pl[GRB_P_RHO], q0);
  pr[GRB_P_PRESS] = eos_PT(e, pr[GRB_P_EPS], pr[GRB_P_CS2], nullptr, pr[GRB_P_TEMP], pr[GRB_P_RHO], q0);
}
// cs2 from (T, rho) as press_h_csnd2__temp_rho_ye computes it
// (hybrid_eos.hh:227-240, ideal_gas_eos.hh:224-234: h summed as
// 1 + eps_cold + eps_th + P/rho); rho and T clamped in place
GRB_HD double eos_cs2_T(const DevEos& e, double& t, double& rho, uint32_t& q) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_temp(e, t, q);
    const double eps = t / e.gm1;
    return e.ggm1 * eps / (1.0 + e.g * eps);
  }
  hy_rho(e, rho, q);
  hy_temp(e, t, q);
  double ec;
  const double pc = pw_cold(e, ec, rho);
  const double eth = fmax(0.0, t / e.gthm1);
  const double p = pc + eth * rho * e.gthm1;
  const double h = 1. + ec + eth + p / rho;
  return (pw_dpdrho(e, rho) + e.gthm1 * (e.gthm1 + 1) * eth) / h;
}
// P from (eps, rho): hybrid_eos.hh:78-85, ideal_gas_eos.hh:88-92
GRB_HD double eos_Peps(const DevEos& e, double& eps, double& rho, uint32_t& q) {
  if (e.kind == GRB_EOS_IDEAL_GAS) { id_eps(e, eps, q); return e.gm1 * eps * rho; }
  hy_rho(e, rho, q);
  double ec;
  const double pc = pw_cold(e, ec, rho);
  hy_eps(e, eps, ec, q);
  return pc + (eps - ec) * rho * e.gthm1;
}
// P, T, s from (eps, rho): hybrid_eos.hh:241-257, ideal_gas_eos.hh:247-258
GRB_HD double eos_Peps_full(const DevEos& e, double& temp, double& ent, double& eps,
                            double& rho, uint32_t& q) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_eps(e, eps, q);
    temp = eps * e.gm1;
    ent = id_ent(e, eps, rho);
    return e.gm1 * eps * rho;
  }
  hy_rho(e, rho, q);
  double ec;
  const double pc = pw_cold(e, ec, rho);
  hy_eps(e, eps, ec, q);
  const double eth = eps - ec;
  ent = hy_ent(e, eth, rho);
  temp = fmax(0.0, eth * e.gthm1);
  return pc + eth * rho * e.gthm1;
}
// P, T, eps from (s, rho): hybrid_eos.hh:293-308 (+ check_entropy_range
// 404-417), ideal_gas_eos.hh:291-302.  ent is clamped in place.
GRB_HD double eos_Pent(const DevEos& e, double& temp, double& eps, double& ent, double& rho,
                       uint32_t& q) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    const double smin = id_ent(e, e.ent_min, rho), smax = id_ent(e, e.eps_max, rho);
    if (ent < smin) { ent = smin; q |= EOS_ENT_LOW; }
    if (ent > smax) { ent = smax; q |= EOS_ENT_HIGH; }
    eps = exp(e.gm1 * (ent + log(rho)));
    temp = eps * e.gm1;
    return e.gm1 * eps * rho;
  }
  hy_rho(e, rho, q);
  {
    double r = rho;
    hy_rho(e, r, q);
    double ecr;
    pw_cold(e, ecr, r);
    const double smin = hy_ent(e, e.entropy_min, r), smax = hy_ent(e, e.eps_max - ecr, r);
    if (ent < smin) { q |= EOS_ENT_LOW; ent = smin; }
    if (ent > smax) { q |= EOS_ENT_HIGH; ent = smax; }
  }
  double ec;
  const double pc = pw_cold(e, ec, rho);
  const double eth = exp(e.gthm1 * ent) * pow(rho, e.gthm1);
  temp = fmax(0.0, eth * e.gthm1);
  eps = ec + eth;
  return pc + eth * rho * e.gthm1;
}
GRB_HD void eos_eps_range(const DevEos& e, double& lo, double& hi, double rho) {
  if (e.kind == GRB_EOS_IDEAL_GAS) { lo = 0; hi = e.eps_max; return; }
  uint32_t q = 0;
  hy_rho(e, rho, q);
  double ec;
  pw_cold(e, ec, rho);
  lo = fmin(ec, e.eps_max);
  hi = e.eps_max;
}

// ---- GRMHD algebra --------------------------------------------------------
GRB_HD double lorentz(const double g[6], const double z[3]) { return sqrt(1. + sqs(g, z)); }
// b^mu and b^2 (grmhd_subexpressions.hh:20-42)
GRB_HD void comoving_b(double alp, const double beta[3], const double g[6], const double B[3],
                       const double z[3], double W, double b[4], double& b2) {
  double zl[3];
  mvs(g, z, zl);
  const double Bz = B[0] * zl[0] + B[1] * zl[1] + B[2] * zl[2];
  const double b0 = Bz / alp;
  const double iW = 1.0 / W;
  b[0] = b0;
#pragma unroll
  for (int i = 0; i < 3; ++i) b[i + 1] = (B[i] + alp * b0 * (z[i] - W * beta[i] / alp)) * iW;
  b2 = (sqs(g, B) + Bz * Bz) * iW * iW;
}
GRB_HD void vtilde(double alp, const double beta[3], const double z[3], double W, double vt[3]) {
  const double aw = alp / W;
#pragma unroll
  for (int i = 0; i < 3; ++i) vt[i] = aw * z[i] - beta[i];
}
// fast magnetosonic speeds (grmhd_subexpressions.hh:59-95)
GRB_HD void char_speeds(double alp, double betad, double rho, double press, double eps,
                        double cs2, double W, double b2, double vtd, double guu_dd, double& cm,
                        double& cp) {
  const double va2 = b2 / (b2 + rho * (1. + eps) + press);
  const double c2 = va2 + cs2 * (1. - va2);
  const double ia2 = 1. / (alp * alp);
  const double u0 = W / alp;
  const double ud = W * vtd / alp;
  const double A = (1. - c2) * u0 * u0 + c2 * ia2;
  const double B = -2. * (1. - c2) * u0 * ud + 2. * c2 * betad * ia2;
  const double C = (1. - c2) * ud * ud - c2 * (guu_dd - betad * betad * ia2);
  const double disc = sqrt(fmax(0., B * B - 4. * A * C));
  const double i2A = 0.5 / A;
  const double l1 = (-B + disc) * i2A, l2 = (-B - disc) * i2A;
  cm = fmin(l1, l2);
  cp = fmax(l1, l2);
}
// Tuned-mode forms of the three helpers above: the same expressions with the
// face's 1/alpha (ialp) and the side's 1/W (iW) computed once and multiplied
// in, instead of 5 divisions by alpha and 2 by W per side; equal up to
// rounding.
GRB_HD void comoving_b_f(double alp, double ialp, const double beta[3], const double g[6], const double B[3],
                         const double z[3], double W, double iW, double b[4], double& b2) {
  double zl[3];
  mvs(g, z, zl);
  const double Bz = B[0] * zl[0] + B[1] * zl[1] + B[2] * zl[2];
  const double b0 = Bz * ialp;
  b[0] = b0;
#pragma unroll
  for (int i = 0; i < 3; ++i) b[i + 1] = (B[i] + alp * b0 * (z[i] - W * beta[i] * ialp)) * iW;
  b2 = (sqs(g, B) + Bz * Bz) * iW * iW;
}
GRB_HD void vtilde_f(double alp, const double beta[3], const double z[3], double iW, double vt[3]) {
  const double aw = alp * iW;
#pragma unroll
  for (int i = 0; i < 3; ++i) vt[i] = aw * z[i] - beta[i];
}
// char_speeds with 1/alpha multiplied in, for the two states of a face at
// once (tuned mode): the two va^2 denominators share one reciprocal, and so
// do the two 2A (all four positive and of physical size, far from the
// double range's ends).
GRB_HD void char_speeds_f2(double ialp, double betad, double guu_dd, const double* pl, const double* pr,
                           double wl, double wr, double b2l, double b2r, double vtdl, double vtdr, double& cml,
                           double& cpl, double& cmr, double& cpr) {
  const double dl = b2l + pl[GRB_P_RHO] * (1. + pl[GRB_P_EPS]) + pl[GRB_P_PRESS];
  const double dr = b2r + pr[GRB_P_RHO] * (1. + pr[GRB_P_EPS]) + pr[GRB_P_PRESS];
  const double rd = 1.0 / (dl * dr);
  const double va2[2] = {b2l * dr * rd, b2r * dl * rd};
  const double cs2[2] = {pl[GRB_P_CS2], pr[GRB_P_CS2]};
  const double W[2] = {wl, wr}, vtd[2] = {vtdl, vtdr};
  const double ia2 = ialp * ialp;
  double A[2], B[2], C[2];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const double c2 = va2[s] + cs2[s] * (1. - va2[s]);
    const double u0 = W[s] * ialp;
    const double ud = W[s] * vtd[s] * ialp;
    A[s] = (1. - c2) * u0 * u0 + c2 * ia2;
    B[s] = -2. * (1. - c2) * u0 * ud + 2. * c2 * betad * ia2;
    C[s] = (1. - c2) * ud * ud - c2 * (guu_dd - betad * betad * ia2);
  }
  const double ra = 0.5 / (A[0] * A[1]);
  const double i2A[2] = {A[1] * ra, A[0] * ra};
  double cm[2], cp[2];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const double disc = sqrt(fmax(0., B[s] * B[s] - 4. * A[s] * C[s]));
    const double l1 = (-B[s] + disc) * i2A[s], l2 = (-B[s] - disc) * i2A[s];
    cm[s] = fmin(l1, l2);
    cp[s] = fmax(l1, l2);
  }
  cml = cm[0]; cpl = cp[0]; cmr = cm[1]; cpr = cp[1];
}
// conserved + fluxes along d (grmhd_subexpressions.hh:97-156, 294-331)
struct ConsFlux {
  double D, tau, S[3], ents, fD, ftau, fS[3], fent;
};
// ialp > 0 (tuned mode): 1/alpha, multiplied in instead of dividing.
GRB_HD ConsFlux cons_flux(double alp, const double beta[3], const double g[6], double rho,
                          double press, double eps, const double z[3], double s, double W,
                          double b2, const double b[4], const double vt[3], int d, double ialp = 0.0) {
  ConsFlux o;
  const double rhoh = rho * (1. + eps) + press + b2;
  const double pstar = press + 0.5 * b2;
  double bl[3], betal[3], zl[3], vtl[3];
  mvs(g, b + 1, bl);
  mvs(g, beta, betal);
  mvs(g, z, zl);
  mvs(g, vt, vtl);
#pragma unroll
  for (int i = 0; i < 3; ++i) bl[i] += betal[i] * b[0];
  o.D = rho * W;
  const double W2rhoh = rhoh * W * W;
  o.tau = W2rhoh - pstar - alp * alp * b[0] * b[0] - o.D;
#pragma unroll
  for (int i = 0; i < 3; ++i) o.S[i] = rhoh * W * zl[i] - alp * b[0] * bl[i];
  o.ents = s * o.D;
  o.fD = o.D * vt[d];
  o.ftau = W2rhoh * vt[d] + pstar * beta[d] - alp * alp * b[0] * b[d + 1] - o.fD;
  const double c = ialp > 0.0 ? W2rhoh * vt[d] * ialp : W2rhoh * vt[d] / alp;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    o.fS[j] = c * (betal[j] + vtl[j]) + alp * ((j == d ? pstar : 0.) - b[d + 1] * bl[j]);
  o.fent = o.ents * vt[d];
  return o;
}
// geometric sources (grmhd_subexpressions.hh:158-292)
//   S_tau = alpha [ (T00 b^i b^j + 2 T0i b^j + Tij) K_ij - (T00 b^i + T0i) d_i alpha ]
//   S_Sj  = alpha [ 1/2 T00 d_j g00 + T0i d_j g0i + 1/2 Tik d_j g_ik ]
GRB_HD void geom_sources(const Met& m, const double K[6], const double dalp[3],
                         const double dg[18], const double db[9], double rho, double press,
                         double eps, const double B[3], const double z[3], double W,
                         double& stau, double sS[3]) {
  const double alp = m.alp;
  const double* beta = m.beta;
  double b[4], b2;
  comoving_b(alp, beta, m.g, B, z, W, b, b2);
  const double rhoh = rho * (1. + eps) + press + b2;
  const double pstar = press + 0.5 * b2;
  const double ia2 = 1. / (alp * alp);
  const double u0 = W / alp;
  double u[3], T0[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) u[i] = z[i] - W * beta[i] / alp;
  const double T00 = rhoh * u0 * u0 - pstar * ia2 - b[0] * b[0];
#pragma unroll
  for (int i = 0; i < 3; ++i) T0[i] = rhoh * u0 * u[i] + pstar * beta[i] * ia2 - b[0] * b[i + 1];
  // symmetric T^ij in (xx,xy,xz,yy,yz,zz) order
  const int si[6] = {0, 0, 0, 1, 1, 2}, sj[6] = {0, 1, 2, 1, 2, 2};
  double T[6];
#pragma unroll
  for (int a = 0; a < 6; ++a)
    T[a] = rhoh * u[si[a]] * u[sj[a]] + pstar * (m.gi[a] - beta[si[a]] * beta[sj[a]] * ia2) -
           b[si[a] + 1] * b[sj[a] + 1];
  double kt = 0.;
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    const double w = (a == 0 || a == 3 || a == 5) ? 1.0 : 2.0;
    const int i = si[a], j = sj[a];
    kt += w * (T00 * beta[i] * beta[j] + T0[i] * beta[j] + T0[j] * beta[i] + T[a]) * K[a];
  }
  double at = 0.;
#pragma unroll
  for (int i = 0; i < 3; ++i) at += (T00 * beta[i] + T0[i]) * dalp[i];
  stau = alp * (kt - at);
  double betal[3];
  mvs(m.g, beta, betal);
#pragma unroll
  for (int jd = 0; jd < 3; ++jd) {
    const double* dgj = dg + 6 * jd;
    const double* dbj = db + 3 * jd;
    double dbv[3];  // beta^k d_j g_ik
    mvs(dgj, beta, dbv);
    double gdb[3];  // g_ik d_j beta^k
    mvs(m.g, dbj, gdb);
    const double dg00 = -2. * alp * dalp[jd] + (beta[0] * dbv[0] + beta[1] * dbv[1] + beta[2] * dbv[2]) +
                        2. * (betal[0] * dbj[0] + betal[1] * dbj[1] + betal[2] * dbj[2]);
    double acc = 0.5 * T00 * dg00;
#pragma unroll
    for (int i = 0; i < 3; ++i) acc += T0[i] * (dbv[i] + gdb[i]);
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      const double w = (a == 0 || a == 3 || a == 5) ? 0.5 : 1.0;
      acc += w * T[a] * dgj[a];
    }
    sS[jd] = alp * acc;
  }
}

GRB_HD double hll(double fL, double fR, double uL, double uR, double cmin, double cmax) {
  return (cmax * fL + cmin * fR - cmax * cmin * (uR - uL)) / (cmax + cmin);
}

// ---- reconstruction at face i-1/2 from cells i-3 .. i+2 -------------------
GRB_HD void weno_z(double um3, double um2, double um1, double u0, double up1, double up2,
                   double& uL, double& uR) {
  const double c13 = 13.0 / 12.0, c14 = 0.25, ep = 1.0e-42;
  {
    const double t0 = um2 + u0 - 2.0 * um1, s0 = um2 + 3.0 * u0 - 4.0 * um1;
    const double t1 = um1 + up1 - 2.0 * u0, s1 = um1 - up1;
    const double t2 = up2 + u0 - 2.0 * up1, s2 = up2 + 3.0 * u0 - 4.0 * up1;
    const double b0 = c13 * t0 * t0 + c14 * s0 * s0;
    const double b1 = c13 * t1 * t1 + c14 * s1 * s1;
    const double b2 = c13 * t2 * t2 + c14 * s2 * s2;
    const double t5 = fabs(b0 - b2);
    const double r0 = t5 / (b0 + ep), r1 = t5 / (b1 + ep), r2 = t5 / (b2 + ep);
    const double a0 = 0.1 * (1.0 + r2 * r2), a1 = 0.6 * (1.0 + r1 * r1), a2 = 0.3 * (1.0 + r0 * r0);
    const double f0 = 2.0 * up2 - 7.0 * up1 + 11.0 * u0;
    const double f1 = -up1 + 5.0 * u0 + 2.0 * um1;
    const double f2 = 2.0 * u0 + 5.0 * um1 - um2;
    uR = (f0 * a0 + f1 * a1 + f2 * a2) / (6.0 * (a0 + a1 + a2));
  }
  {
    const double t0 = um3 + um1 - 2.0 * um2, s0 = um3 + 3.0 * um1 - 4.0 * um2;
    const double t1 = um2 + u0 - 2.0 * um1, s1 = um2 - u0;
    const double t2 = up1 + um1 - 2.0 * u0, s2 = up1 + 3.0 * um1 - 4.0 * u0;
    const double b0 = c13 * t0 * t0 + c14 * s0 * s0;
    const double b1 = c13 * t1 * t1 + c14 * s1 * s1;
    const double b2 = c13 * t2 * t2 + c14 * s2 * s2;
    const double t5 = fabs(b0 - b2);
    const double r0 = t5 / (b0 + ep), r1 = t5 / (b1 + ep), r2 = t5 / (b2 + ep);
    const double a0 = 0.1 * (1.0 + r0 * r0), a1 = 0.6 * (1.0 + r1 * r1), a2 = 0.3 * (1.0 + r2 * r2);
    const double f0 = 2.0 * um3 - 7.0 * um2 + 11.0 * um1;
    const double f1 = -um2 + 5.0 * um1 + 2.0 * u0;
    const double f2 = 2.0 * um1 + 5.0 * u0 - up1;
    uL = (f0 * a0 + f1 * a1 + f2 * a2) / (6.0 * (a0 + a1 + a2));
  }
}
GRB_HD double lim_minmod(double sl, double sr) {
  return 0.5 * (copysign(1.0, sl) + copysign(1.0, sr)) * fmin(fabs(sl), fabs(sr));
}
GRB_HD double lim_mc2(double sl, double sr) {
  const double sc = 0.5 * (sr + sl);
  const double s = copysign(1.0, sr);
  return s * fmax(0., fmin(fmin(2. * fabs(sr), 2. * s * sl), s * sc));
}
GRB_HD void recon6(int kind, const double u[6], double& uL, double& uR) {
  if (kind == GRB_RECON_WENOZ) { weno_z(u[0], u[1], u[2], u[3], u[4], u[5], uL, uR); return; }
  if (kind == GRB_RECON_DONOR) { uL = u[2]; uR = u[3]; return; }
  if (kind == GRB_RECON_MC2) {
    uR = u[3] - 0.5 * lim_mc2(u[3] - u[2], u[4] - u[3]);
    uL = u[2] + 0.5 * lim_mc2(u[2] - u[1], u[3] - u[2]);
  } else {
    uR = u[3] - 0.5 * lim_minmod(u[3] - u[2], u[4] - u[3]);
    uL = u[2] + 0.5 * lim_minmod(u[2] - u[1], u[3] - u[2]);
  }
}
// HLL flux with a precomputed 1/(cmax+cmin): one division per face instead
// of one per variable (agrees with hll() to a few ulp).
GRB_HD double hll_r(double fL, double fR, double uL, double uR, double cmin, double cmax,
                    double inv_sum) {
  return (cmax * fL + cmin * fR - cmax * cmin * (uR - uL)) * inv_sum;
}

// WENO-Z with one division per side: with e_k = (beta_k + eps)^2 the
// nonlinear weights alpha_k = d_k (1 + tau^2 / e_k) are multiplied through by
// e_0 e_1 e_2, so u = sum d_k (e_k + tau^2) f_k E_k / (6 sum d_k (e_k + tau^2) E_k)
// with E_k the product of the other two e_j.  e_k >= 1e-84 (eps = 1e-42), so
// the products stay far above the subnormal range for any physical input.
GRB_HD double wz_side(double b0, double b1, double b2, double f0, double f1, double f2,
                      double d0, double d1, double d2) {
  const double ep = 1.0e-42;
  const double t5 = fabs(b0 - b2);
  const double t2 = t5 * t5;
  const double e0 = (b0 + ep) * (b0 + ep), e1 = (b1 + ep) * (b1 + ep), e2 = (b2 + ep) * (b2 + ep);
  const double w0 = d0 * (e0 + t2) * (e1 * e2);
  const double w1 = d1 * (e1 + t2) * (e0 * e2);
  const double w2 = d2 * (e2 + t2) * (e0 * e1);
  return (f0 * w0 + f1 * w1 + f2 * w2) / (6.0 * (w0 + w1 + w2));
}
// wz_side as a numerator and a positive, normal denominator (>= 6e-253).
GRB_HD void wz_side_nd(double b0, double b1, double b2, double f0, double f1, double f2, double d0, double d1,
                       double d2, double& num, double& den) {
  const double ep = 1.0e-42;
  const double t5 = fabs(b0 - b2);
  const double t2 = t5 * t5;
  const double e0 = (b0 + ep) * (b0 + ep), e1 = (b1 + ep) * (b1 + ep), e2 = (b2 + ep) * (b2 + ep);
  const double w0 = d0 * (e0 + t2) * (e1 * e2);
  const double w1 = d1 * (e1 + t2) * (e0 * e2);
  const double w2 = d2 * (e2 + t2) * (e0 * e1);
  num = f0 * w0 + f1 * w1 + f2 * w2;
  den = 6.0 * (w0 + w1 + w2);
}
// 2^-e for a nonzero normal d = +-m 2^e (m in [1, 2)), exact.
GRB_HD double inv_pow2_exponent(double d) {
#ifdef __CUDA_ARCH__
  const long long be = (__double_as_longlong(d) >> 52) & 0x7ff;
  return __longlong_as_double((2046ll - be) << 52);
#else
  int e;
  frexp(d, &e);  // d = f 2^e, f in [0.5, 1)
  return ldexp(1.0, 1 - e);
#endif
}
// n1 / d1 and n2 / d2 with one division (tuned mode): the denominators,
// nonzero and normal, are first scaled by powers of two to magnitudes in
// [1, 2) (exact), so that their product neither overflows nor underflows.
GRB_HD void div_pair(double n1, double d1, double n2, double d2, double& q1, double& q2) {
  const double s1 = inv_pow2_exponent(d1), s2 = inv_pow2_exponent(d2);
  const double a1 = d1 * s1, a2 = d2 * s2;
  const double r = 1.0 / (a1 * a2);
  q1 = (n1 * s1) * a2 * r;
  q2 = (n2 * s2) * a1 * r;
}
// WENO-Z at face i-1/2 as numerators and denominators (tuned mode): the
// states are nL / dL and nR / dR (dL, dR positive and normal).
GRB_HD void weno_z_nd(const double u[6], double& nL, double& dL, double& nR, double& dR) {
  const double um3 = u[0], um2 = u[1], um1 = u[2], u0 = u[3], up1 = u[4], up2 = u[5];
  const double c13 = 13.0 / 12.0, c14 = 0.25;
  {
    const double t0 = um2 + u0 - 2.0 * um1, s0 = um2 + 3.0 * u0 - 4.0 * um1;
    const double t1 = um1 + up1 - 2.0 * u0, s1 = um1 - up1;
    const double t2 = up2 + u0 - 2.0 * up1, s2 = up2 + 3.0 * u0 - 4.0 * up1;
    const double b0 = c13 * t0 * t0 + c14 * s0 * s0;
    const double b1 = c13 * t1 * t1 + c14 * s1 * s1;
    const double b2 = c13 * t2 * t2 + c14 * s2 * s2;
    wz_side_nd(b2, b1, b0, 2.0 * up2 - 7.0 * up1 + 11.0 * u0, -up1 + 5.0 * u0 + 2.0 * um1,
               2.0 * u0 + 5.0 * um1 - um2, 0.1, 0.6, 0.3, nR, dR);
  }
  {
    const double t0 = um3 + um1 - 2.0 * um2, s0 = um3 + 3.0 * um1 - 4.0 * um2;
    const double t1 = um2 + u0 - 2.0 * um1, s1 = um2 - u0;
    const double t2 = up1 + um1 - 2.0 * u0, s2 = up1 + 3.0 * um1 - 4.0 * u0;
    const double b0 = c13 * t0 * t0 + c14 * s0 * s0;
    const double b1 = c13 * t1 * t1 + c14 * s1 * s1;
    const double b2 = c13 * t2 * t2 + c14 * s2 * s2;
    wz_side_nd(b0, b1, b2, 2.0 * um3 - 7.0 * um2 + 11.0 * um1, -um2 + 5.0 * um1 + 2.0 * u0,
               2.0 * um1 + 5.0 * u0 - up1, 0.1, 0.6, 0.3, nL, dL);
  }
}
// n[k] / d[k], k = 0..3, with one division (tuned mode): as div_pair, the
// four denominators scaled to magnitudes in [1, 2) first.
GRB_HD void div_quad(const double n[4], const double d[4], double q[4]) {
  double s[4], a[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    s[k] = inv_pow2_exponent(d[k]);
    a[k] = d[k] * s[k];
  }
  const double p01 = a[0] * a[1], p23 = a[2] * a[3];
  const double r = 1.0 / (p01 * p23);
  const double r01 = p23 * r, r23 = p01 * r;
  q[0] = (n[0] * s[0]) * a[1] * r01;
  q[1] = (n[1] * s[1]) * a[0] * r01;
  q[2] = (n[2] * s[2]) * a[3] * r23;
  q[3] = (n[3] * s[3]) * a[2] * r23;
}
GRB_HD void weno_z_fast(double um3, double um2, double um1, double u0, double up1, double up2,
                        double& uL, double& uR) {
  const double u[6] = {um3, um2, um1, u0, up1, up2};
  double nL, dL, nR, dR;
  weno_z_nd(u, nL, dL, nR, dR);
  div_pair(nL, dL, nR, dR, uL, uR);
}
GRB_HD void recon6_fast(int kind, const double u[6], double& uL, double& uR) {
  if (kind == GRB_RECON_WENOZ) { weno_z_fast(u[0], u[1], u[2], u[3], u[4], u[5], uL, uR); return; }
  recon6(kind, u, uL, uR);
}
GRB_HD double face4(double um2, double um1, double u0, double up1) {
  return 0.5625 * (um1 + u0) + (-0.0625) * (um2 + up1);
}
// Sixth-order centred first derivative.  On the device every operation is
// rounded on its own (no contraction into fused multiply-adds), so the value
// is the same bits wherever the stencil is inlined (the stage, the
// static-metric cache) and matches a host evaluation without FMA.
GRB_HD double fd6(double m3, double m2, double m1, double p1, double p2, double p3, double h) {
#ifdef __CUDA_ARCH__
  const double s = __dadd_rn(__dsub_rn(__dmul_rn(45.0, __dsub_rn(p1, m1)), __dmul_rn(9.0, __dsub_rn(p2, m2))),
                             __dsub_rn(p3, m3));
  return __dmul_rn(__dmul_rn(1.0 / 60.0, h), s);
#else
  return (1.0 / 60.0) * h * (45.0 * (p1 - m1) - 9.0 * (p2 - m2) + (p3 - m3));
#endif
}

}  // namespace grb
