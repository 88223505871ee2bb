// CPU oracle — test infrastructure only.  Nothing in the CUDA library links,
// includes or calls this file; only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load the oracle library built from it.
//
// Restatement, in plain C++, of the per-cell numerics of GRACE's Cowling
// GRMHD path.  Every function names the reference file:line it follows
// (paths relative to the GRACE source tree).  The physics expressions
// (Lorentz factor, comoving field, characteristic speeds, fluxes, geometric
// sources) are written from the standard GRMHD formulas, not from the
// reference's SymPy-generated expression trees, so they agree with the
// reference to rounding, not bit for bit.  Control flow that decides
// branches (c2p policy, Brent, clamps, signal bits) follows the reference
// step by step, because the outcome of those decisions is part of the
// result.  Built with -ffp-contract=off.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>

#include "grace_b200.h"

namespace orc {

// ---------------------------------------------------------------------------
// bit layouts (c2p.hh:44-121, eos_base.hh:40-54)
// ---------------------------------------------------------------------------
enum SigBit : uint32_t {
  S_EPS_TOO_HIGH = 0, S_EPS_TOO_LOW, S_YE_TOO_LOW, S_YE_TOO_HIGH, S_RHO_TOO_HIGH,
  S_RHO_TOO_LOW, S_ENT_TOO_LOW, S_ENT_TOO_HIGH, S_VEL_TOO_HIGH, S_SIGMA_TOO_HIGH
};
enum ErrBit : uint32_t {
  E_RESET_DENS = 0, E_RESET_TAU, E_RESET_STILDE, E_RESET_ENTROPY, E_RESET_YE,
  E_SIG_RHO_TOO_LOW, E_SIG_RHO_TOO_HIGH, E_SIG_EPS_TOO_LOW, E_SIG_EPS_TOO_HIGH,
  E_SIG_YE_TOO_LOW, E_SIG_YE_TOO_HIGH, E_SIG_ENT_TOO_LOW, E_SIG_ENT_TOO_HIGH,
  E_SIG_TEMP_TOO_LOW, E_SIG_TEMP_TOO_HIGH, E_SIG_PRESS_TOO_LOW,
  E_SIG_PRESS_TOO_HIGH, E_SIG_VEL_TOO_HIGH, E_SIG_SIGMA_TOO_HIGH,
  E_ENT_BACKUP_USED, E_ATMO_RESET, E_T_FLOORED
};
enum EosBit : uint32_t {
  Q_RHO_TOO_HIGH = 0, Q_RHO_TOO_LOW, Q_EPS_TOO_HIGH, Q_EPS_TOO_LOW, Q_YE_TOO_LOW,
  Q_YE_TOO_HIGH, Q_TEMP_TOO_LOW, Q_TEMP_TOO_HIGH, Q_ENT_TOO_LOW, Q_ENT_TOO_HIGH,
  Q_PRESS_TOO_LOW, Q_PRESS_TOO_HIGH
};
// local cons / prims orderings (grmhd_helpers.hh:105-149)
enum { CONS_D = 0, CONS_SX, CONS_SY, CONS_SZ, CONS_TAU, CONS_YES, CONS_ENTS, CONS_BX, CONS_BY, CONS_BZ };
enum { PR_RHO = 0, PR_PRESS, PR_ZX, PR_ZY, PR_ZZ, PR_YE, PR_TEMP, PR_EPS, PR_ENT, PR_BX, PR_BY, PR_BZ, PR_CS2 };
inline void setb(uint32_t& w, uint32_t b) { w |= (1u << b); }
inline bool tstb(uint32_t w, uint32_t b) { return (w >> b) & 1u; }

// ---------------------------------------------------------------------------
// 3-metric (metric_utils.hh:48-82, 220-295)
// ---------------------------------------------------------------------------
struct Metric {
  double g[6], beta[3], alp, ginv[6], sqrtg;
};
inline Metric make_metric(const double g[6], const double b[3], double alp) {
  Metric m;
  for (int a = 0; a < 6; ++a) m.g[a] = g[a];
  for (int a = 0; a < 3; ++a) m.beta[a] = b[a];
  m.alp = alp;
  // cofactor expansion of the symmetric 3x3 matrix (xx,xy,xz,yy,yz,zz)
  const double c0 = g[3] * g[5] - g[4] * g[4];
  const double c1 = g[2] * g[4] - g[1] * g[5];
  const double c2 = g[1] * g[4] - g[2] * g[3];
  const double det = g[0] * c0 + g[1] * c1 + g[2] * c2;
  m.ginv[0] = c0 / det;
  m.ginv[1] = c1 / det;
  m.ginv[2] = c2 / det;
  m.ginv[3] = (g[0] * g[5] - g[2] * g[2]) / det;
  m.ginv[4] = (g[1] * g[2] - g[0] * g[4]) / det;
  m.ginv[5] = (g[0] * g[3] - g[1] * g[1]) / det;
  m.sqrtg = std::sqrt(det);
  return m;
}
// v^i v^j g_ij with a symmetric 6-array
inline double sq_sym(const double s[6], const double v[3]) {
  return s[0] * v[0] * v[0] + s[3] * v[1] * v[1] + s[5] * v[2] * v[2] +
         2. * (s[1] * v[0] * v[1] + s[2] * v[0] * v[2] + s[4] * v[1] * v[2]);
}
inline void mul_sym(const double s[6], const double v[3], double o[3]) {
  o[0] = s[0] * v[0] + s[1] * v[1] + s[2] * v[2];
  o[1] = s[1] * v[0] + s[3] * v[1] + s[4] * v[2];
  o[2] = s[2] * v[0] + s[4] * v[1] + s[5] * v[2];
}

// ---------------------------------------------------------------------------
// EOS (eos_base.hh, ideal_gas_eos.hh, hybrid_eos.hh,
// piecewise_polytropic_eos.hh).  Arguments passed by reference are clamped
// in place exactly where the reference clamps them.
// ---------------------------------------------------------------------------
struct Eos {
  int kind;
  // eos_base_t limits (hybrid_eos.hh:62-75, ideal_gas_eos.hh:56-86)
  double rhomax, rhomin, tempmax, tempmin, yemax, yemin, c2p_eps_min, c2p_eps_max;
  double h_min, temp_atm, ye_atm;
  // ideal gas
  double g_m1, g, gg_m1, ent_min;
  // hybrid: thermal part + cold polytrope
  double gth_m1, entropy_min;
  int n;
  double K[GRB_MAX_PIECES], G[GRB_MAX_PIECES], R[GRB_MAX_PIECES], E[GRB_MAX_PIECES];
};

inline Eos make_eos(const grb_eos_params& p) {
  Eos e{};
  e.kind = p.kind;
  e.c2p_eps_min = 0.0;
  e.c2p_eps_max = p.eps_max;
  e.temp_atm = p.temp_atm;
  e.ye_atm = 0.0;
  e.tempmin = 0.0;
  e.yemin = 0.0;
  if (p.kind == GRB_EOS_IDEAL_GAS) {
    e.rhomax = 1e100; e.rhomin = 1e-100; e.tempmax = 1e100; e.yemax = 1e100;
    e.h_min = 1. + 1e-15;
    e.g_m1 = p.gamma - 1.;
    e.g = e.g_m1 + 1.;
    e.gg_m1 = e.g * e.g_m1;
    e.ent_min = (p.temp_atm > 0.0) ? (p.temp_atm / e.g_m1) : 1e-100;
  } else {
    // eos_storage.cpp:143-150 (polytrope bounds) and :176 (h_min)
    e.rhomax = 1e10; e.rhomin = 1e-100; e.tempmax = 1e99; e.yemax = 1e99;
    e.h_min = 1. + 1e-10;
    e.gth_m1 = p.gamma_th - 1.;
    e.entropy_min = p.entropy_min;
    e.n = p.n_pieces;
    for (int i = 0; i < GRB_MAX_PIECES; ++i) {
      e.K[i] = p.pw_kappa[i]; e.G[i] = p.pw_gamma[i];
      e.R[i] = p.pw_rho[i]; e.E[i] = p.pw_eps[i];
    }
  }
  return e;
}

// --- piecewise polytrope (piecewise_polytropic_eos.hh:71-78, 128-138)
inline int pw_index(const Eos& e, double& rho) {
  rho = std::fmax(e.rhomin, std::fmin(e.rhomax, rho));
  for (int ii = 0; ii < e.n - 1; ++ii)
    if (rho > e.R[ii] && rho <= e.R[ii + 1]) return ii;
  return e.n - 1;
}
inline double pw_press_cold(const Eos& e, double& eps_cold, double& rho) {
  const int i = pw_index(e, rho);
  const double pc = e.K[i] * std::pow(rho, e.G[i]);
  eps_cold = e.E[i] + pc / (rho * (e.G[i] - 1.));
  return pc;
}
inline double pw_dpress_drho(const Eos& e, double& rho) {
  const int i = pw_index(e, rho);
  const double pc = e.K[i] * std::pow(rho, e.G[i]);
  return e.G[i] * pc / rho;
}

// --- hybrid helpers (hybrid_eos.hh:376-470)
inline void hy_check_rho(const Eos& e, double& rho, uint32_t& err) {
  if (rho < e.rhomin) { setb(err, Q_RHO_TOO_LOW); rho = e.rhomin; }
  if (rho > e.rhomax) { setb(err, Q_RHO_TOO_HIGH); rho = e.rhomax; }
}
inline void hy_check_temp(const Eos& e, double& t, uint32_t& err) {
  if (t < e.tempmin) { setb(err, Q_TEMP_TOO_LOW); t = e.tempmin; }
  if (t > e.tempmax) { setb(err, Q_TEMP_TOO_HIGH); t = e.tempmax; }
}
inline void hy_check_eps(const Eos& e, double& eps, double eps_cold, uint32_t& err) {
  const double lo = std::min(eps_cold, e.c2p_eps_max);
  if (eps < lo) { setb(err, Q_EPS_TOO_LOW); eps = lo; }
  if (eps > e.c2p_eps_max) { setb(err, Q_EPS_TOO_HIGH); eps = e.c2p_eps_max; }
}
inline double hy_entropy(const Eos& e, double eps_th, double rho) {
  const double et = std::max(eps_th, e.entropy_min);
  return std::log(et * std::pow(rho, -e.gth_m1)) / e.gth_m1;
}
inline double hy_cs2(const Eos& e, double& rho, double eps_th, double h) {
  return (pw_dpress_drho(e, rho) + e.gth_m1 * (e.gth_m1 + 1) * eps_th) / h;
}

// --- ideal-gas helpers (ideal_gas_eos.hh:360-437)
inline void id_limit_eps(const Eos& e, double& eps, uint32_t& err) {
  if (eps > e.c2p_eps_max) { setb(err, Q_EPS_TOO_HIGH); eps = e.c2p_eps_max; }
  if (eps < e.c2p_eps_min) { setb(err, Q_EPS_TOO_LOW); eps = e.c2p_eps_min; }
}
inline void id_limit_temp(const Eos& e, double& t, uint32_t& err) {
  const double tmax = e.c2p_eps_max * e.g_m1;
  if (t < e.tempmin) { t = e.tempmin; setb(err, Q_TEMP_TOO_LOW); }
  if (t > tmax) { setb(err, Q_TEMP_TOO_HIGH); t = tmax; }
}
inline double id_entropy(const Eos& e, double eps, double rho) {
  return std::log(eps) / e.g_m1 - std::log(rho);
}

// P, eps, cs2 from (T, rho): hybrid_eos.hh:224-239, ideal_gas_eos.hh:233-244
inline double press_eps_csnd2__temp_rho(const Eos& e, double& eps, double& cs2,
                                        double& temp, double& rho, uint32_t& err) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_limit_temp(e, temp, err);
    eps = temp / e.g_m1;
    const double p = e.g_m1 * eps * rho;
    const double h = 1.0 + e.g * eps;
    cs2 = e.gg_m1 * eps / h;
    return p;
  }
  hy_check_rho(e, rho, err);
  hy_check_temp(e, temp, err);
  double ec;
  const double pc = pw_press_cold(e, ec, rho);
  const double eth = std::fmax(0.0, temp / e.gth_m1);
  const double p = pc + eth * rho * e.gth_m1;
  eps = ec + eth;
  const double h = 1. + eps + p / rho;
  cs2 = hy_cs2(e, rho, eth, h);
  return p;
}
// P, h, cs2 from (T, rho): hybrid_eos.hh:227-240, ideal_gas_eos.hh:224-234
// (h summed as 1 + eps_cold + eps_th + P/rho, as the reference does there)
inline double press_h_csnd2__temp_rho(const Eos& e, double& h, double& cs2, double& temp,
                                      double& rho, uint32_t& err) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_limit_temp(e, temp, err);
    const double eps = temp / e.g_m1;
    const double p = e.g_m1 * eps * rho;
    h = 1.0 + e.g * eps;
    cs2 = e.gg_m1 * eps / h;
    return p;
  }
  hy_check_rho(e, rho, err);
  hy_check_temp(e, temp, err);
  double ec;
  const double pc = pw_press_cold(e, ec, rho);
  const double eth = std::fmax(0.0, temp / e.gth_m1);
  const double p = pc + eth * rho * e.gth_m1;
  h = 1. + ec + eth + p / rho;
  cs2 = hy_cs2(e, rho, eth, h);
  return p;
}
// P, eps, cs2, s from (T, rho): hybrid_eos.hh:276-291, ideal_gas_eos.hh:277-288
inline double press_eps_csnd2_entropy__temp_rho(const Eos& e, double& eps, double& cs2,
                                                double& ent, double& temp, double& rho,
                                                uint32_t& err) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_limit_temp(e, temp, err);
    eps = temp / e.g_m1;
    const double p = e.g_m1 * eps * rho;
    const double h = 1.0 + e.g * eps;
    cs2 = e.gg_m1 * eps / h;
    ent = id_entropy(e, eps, rho);
    return p;
  }
  hy_check_rho(e, rho, err);
  hy_check_temp(e, temp, err);
  double ec;
  const double pc = pw_press_cold(e, ec, rho);
  const double eth = std::fmax(0.0, temp / e.gth_m1);
  const double p = pc + eth * rho * e.gth_m1;
  eps = eth + ec;
  const double h = 1. + eps + p / rho;
  cs2 = hy_cs2(e, rho, eth, h);
  ent = hy_entropy(e, eth, rho);
  return p;
}
// P only from (eps, rho): hybrid_eos.hh:78-85, ideal_gas_eos.hh:88-92
inline double press__eps_rho(const Eos& e, double& eps, double& rho, uint32_t& err) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_limit_eps(e, eps, err);
    return e.g_m1 * eps * rho;
  }
  hy_check_rho(e, rho, err);
  double ec;
  const double pc = pw_press_cold(e, ec, rho);
  hy_check_eps(e, eps, ec, err);
  return pc + (eps - ec) * rho * e.gth_m1;
}
// P, h, cs2, T, s from (eps, rho): hybrid_eos.hh:241-257, ideal_gas_eos.hh:247-258
inline double press_h_csnd2_temp_entropy__eps_rho(const Eos& e, double& h, double& cs2,
                                                  double& temp, double& ent, double& eps,
                                                  double& rho, uint32_t& err) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    id_limit_eps(e, eps, err);
    const double p = e.g_m1 * eps * rho;
    h = 1.0 + e.g * eps;
    cs2 = e.gg_m1 * eps / h;
    temp = eps * e.g_m1;
    ent = id_entropy(e, eps, rho);
    return p;
  }
  hy_check_rho(e, rho, err);
  double ec;
  const double pc = pw_press_cold(e, ec, rho);
  hy_check_eps(e, eps, ec, err);
  const double eth = eps - ec;
  const double p = pc + eth * rho * e.gth_m1;
  h = 1. + eps + p / rho;
  cs2 = hy_cs2(e, rho, eth, h);
  ent = hy_entropy(e, eth, rho);
  temp = std::fmax(0.0, eth * e.gth_m1);
  return p;
}
// P, h, cs2, T, eps from (s, rho): hybrid_eos.hh:293-308, ideal_gas_eos.hh:291-302
inline double press_h_csnd2_temp_eps__entropy_rho(const Eos& e, double& h, double& cs2,
                                                  double& temp, double& eps, double& ent,
                                                  double& rho, uint32_t& err) {
  if (e.kind == GRB_EOS_IDEAL_GAS) {
    const double smin = id_entropy(e, e.ent_min, rho);
    const double smax = id_entropy(e, e.c2p_eps_max, rho);
    if (ent < smin) { ent = smin; setb(err, Q_ENT_TOO_LOW); }
    if (ent > smax) { ent = smax; setb(err, Q_ENT_TOO_HIGH); }
    eps = std::exp(e.g_m1 * (ent + std::log(rho)));
    const double p = e.g_m1 * eps * rho;
    h = 1.0 + e.g * eps;
    temp = eps * e.g_m1;
    cs2 = e.gg_m1 * eps / h;
    return p;
  }
  hy_check_rho(e, rho, err);
  {  // check_entropy_range on a copy of rho (hybrid_eos.hh:404-417, 195-205)
    double r = rho;
    uint32_t dummy_err = 0;
    hy_check_rho(e, r, dummy_err);
    err |= dummy_err;
    double ecr;
    pw_press_cold(e, ecr, r);
    const double smin = hy_entropy(e, e.entropy_min, r);
    const double smax = hy_entropy(e, e.c2p_eps_max - ecr, r);
    if (ent < smin) { setb(err, Q_ENT_TOO_LOW); ent = smin; }
    if (ent > smax) { setb(err, Q_ENT_TOO_HIGH); ent = smax; }
  }
  double ec;
  const double pc = pw_press_cold(e, ec, rho);
  const double eth = std::exp(e.gth_m1 * ent) * std::pow(rho, e.gth_m1);
  const double p = pc + eth * rho * e.gth_m1;
  temp = std::fmax(0.0, eth * e.gth_m1);
  eps = ec + eth;
  h = 1. + eps + p / rho;
  cs2 = hy_cs2(e, rho, eth, h);
  return p;
}
// eps range at (rho): hybrid_eos.hh:177-185, ideal_gas_eos.hh:194-200
inline void eps_range__rho(const Eos& e, double& lo, double& hi, double& rho, uint32_t& err) {
  if (e.kind == GRB_EOS_IDEAL_GAS) { lo = 0; hi = e.c2p_eps_max; return; }
  hy_check_rho(e, rho, err);
  double ec;
  pw_press_cold(e, ec, rho);
  lo = std::min(ec, e.c2p_eps_max);
  hi = e.c2p_eps_max;
}

// ---------------------------------------------------------------------------
// GRMHD algebra (standard formulas; reference: grmhd_subexpressions.hh)
// ---------------------------------------------------------------------------
// W = sqrt(1 + z^i z_i)                       (grmhd_subexpressions.hh:10-18)
inline double lorentz(const double g[6], const double z[3]) {
  return std::sqrt(1. + sq_sym(g, z));
}
// b^mu of the comoving field and b^2          (grmhd_subexpressions.hh:20-42)
//   b^0 = B^i z_i / alpha, b^i = (B^i + alpha b^0 u^i) / W,
//   b^2 = (B^i B_i + (B^i z_i)^2) / W^2,  with u^i = z^i - W beta^i / alpha.
inline void comoving_b(double alp, const double beta[3], const double g[6],
                       const double B[3], const double z[3], double W, double b[4],
                       double& b2) {
  double zl[3];
  mul_sym(g, z, zl);
  const double Bz = B[0] * zl[0] + B[1] * zl[1] + B[2] * zl[2];
  const double b0 = Bz / alp;
  b[0] = b0;
  for (int i = 0; i < 3; ++i) {
    const double ui = z[i] - W * beta[i] / alp;
    b[i + 1] = (B[i] + alp * b0 * ui) / W;
  }
  b2 = (sq_sym(g, B) + Bz * Bz) / (W * W);
}
// vtilde^i = alpha z^i / W - beta^i           (grmhd_subexpressions.hh:44-57)
inline void transport_velocity(double alp, const double beta[3], const double z[3],
                               double W, double vt[3]) {
  for (int i = 0; i < 3; ++i) vt[i] = alp * z[i] / W - beta[i];
}
// Fast-magnetosonic characteristic speeds along direction d
// (grmhd_subexpressions.hh:59-95).  Roots lambda of
//   (1-c2)(u^0 lambda - u^d)^2 = c2 (g^00 lambda^2 - 2 g^0d lambda + g^dd)
// with c2 = v_A^2 + c_s^2 (1 - v_A^2), v_A^2 = b^2 / (b^2 + rho h).
inline void char_speeds(double alp, const double beta[3], double rho, double press,
                        double eps, double cs2, double W, double b2, const double vt[3],
                        double guu_dd, int d, double& cm, double& cp) {
  const double va2 = b2 / (b2 + rho * (1. + eps) + press);
  const double c2 = va2 + cs2 * (1. - va2);
  const double ia2 = 1. / (alp * alp);
  const double u0 = W / alp;
  const double ud = W * vt[d] / alp;
  const double g00 = -ia2, g0d = beta[d] * ia2, gdd = guu_dd - beta[d] * beta[d] * ia2;
  const double A = (1. - c2) * u0 * u0 - c2 * g00;
  const double B = -2. * (1. - c2) * u0 * ud + 2. * c2 * g0d;
  const double C = (1. - c2) * ud * ud - c2 * gdd;
  const double disc = std::sqrt(std::fmax(0., B * B - 4. * A * C));
  const double l1 = (-B + disc) / (2. * A);
  const double l2 = (-B - disc) / (2. * A);
  cm = std::fmin(l1, l2);
  cp = std::fmax(l1, l2);
}
// Conserved (undensitized) and fluxes along d  (grmhd_subexpressions.hh:97-156,294-331)
//   D = rho W, tau = rho h* W^2 - P* - (alpha b^0)^2 - D,
//   S_j = rho h* W^2 v_j - alpha b^0 b_j,  s* = s D,
//   F_D = D vt^d, F_tau = alpha^2 T^{0d} - D vt^d, F_Sj = alpha T^d_j,
//   F_s* = s* vt^d;  rho h* = rho(1+eps) + P + b^2, P* = P + b^2/2.
inline void cons_and_flux(double alp, const double beta[3], const double g[6], double rho,
                          double press, double eps, const double z[3], double s, double W,
                          double b2, const double b[4], const double vt[3], int d,
                          double& D, double& tau, double S[3], double& ents, double& fD,
                          double& ftau, double fS[3], double& fent) {
  const double rhoh = rho * (1. + eps) + press + b2;
  const double pstar = press + 0.5 * b2;
  double bl[3], betal[3], zl[3];
  mul_sym(g, b + 1, bl);
  mul_sym(g, beta, betal);
  mul_sym(g, z, zl);
  for (int i = 0; i < 3; ++i) bl[i] += betal[i] * b[0];  // b_i = beta_i b^0 + g_ij b^j
  D = rho * W;
  tau = rhoh * W * W - pstar - alp * alp * b[0] * b[0] - D;
  for (int i = 0; i < 3; ++i) S[i] = rhoh * W * zl[i] - alp * b[0] * bl[i];
  ents = s * D;
  fD = D * vt[d];
  const double a2T0d = rhoh * W * W * vt[d] + pstar * beta[d] - alp * alp * b[0] * b[d + 1];
  ftau = a2T0d - fD;
  double vtl[3];
  mul_sym(g, vt, vtl);
  for (int j = 0; j < 3; ++j) {
    // u_j = (W/alpha)(beta_j + g_jk vt^k), u^d = W vt^d / alpha
    const double uu = W * W * vt[d] * (betal[j] + vtl[j]) / (alp * alp);
    fS[j] = alp * (rhoh * uu + (j == d ? pstar : 0.) - b[d + 1] * bl[j]);
  }
  fent = ents * vt[d];
}
// Geometric source terms (grmhd_subexpressions.hh:158-292), written as
//   S_tau = alpha [ (T^00 b^i b^j + 2 T^0i b^j + T^ij) K_ij - (T^00 b^i + T^0i) d_i alpha ]
//   S_Sj  = alpha [ 1/2 T^00 d_j g_00 + T^0i d_j g_0i + 1/2 T^ik d_j g_ik ]
// with T^{mu nu} = rho h* u^mu u^nu + P* g^{mu nu} - b^mu b^nu and
// d_j g_00 = -2 alpha d_j alpha + beta^i beta^k d_j g_ik + 2 beta_k d_j beta^k,
// d_j g_0i = beta^k d_j g_ik + g_ik d_j beta^k.  dgdd[6*j + a], dbeta[3*j + i].
inline void geom_sources(double alp, const double beta[3], const double g[6],
                         const double guu[6], const double K[6], const double dalp[3],
                         const double dgdd[18], const double dbeta[9], double rho,
                         double press, double eps, const double B[3], const double z[3],
                         double W, double& stau, double sS[3]) {
  double b[4], b2;
  comoving_b(alp, beta, g, B, z, W, b, b2);
  const double rhoh = rho * (1. + eps) + press + b2;
  const double pstar = press + 0.5 * b2;
  const double ia2 = 1. / (alp * alp);
  const double u0 = W / alp;
  double u[3];
  for (int i = 0; i < 3; ++i) u[i] = z[i] - W * beta[i] / alp;
  const double T00 = rhoh * u0 * u0 - pstar * ia2 - b[0] * b[0];
  double T0[3];
  for (int i = 0; i < 3; ++i) T0[i] = rhoh * u0 * u[i] + pstar * beta[i] * ia2 - b[0] * b[i + 1];
  static const int sym[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  double T[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      T[i][j] = rhoh * u[i] * u[j] + pstar * (guu[sym[i][j]] - beta[i] * beta[j] * ia2) -
                b[i + 1] * b[j + 1];
  stau = 0.;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      stau += (T00 * beta[i] * beta[j] + 2. * T0[i] * beta[j] + T[i][j]) * K[sym[i][j]];
  for (int i = 0; i < 3; ++i) stau -= (T00 * beta[i] + T0[i]) * dalp[i];
  stau *= alp;
  double betal[3];
  mul_sym(g, beta, betal);
  for (int jd = 0; jd < 3; ++jd) {
    const double* dg = dgdd + 6 * jd;
    const double* db = dbeta + 3 * jd;
    double dg00 = -2. * alp * dalp[jd];
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) dg00 += beta[i] * beta[k] * dg[sym[i][k]];
    for (int k = 0; k < 3; ++k) dg00 += 2. * betal[k] * db[k];
    double acc = 0.5 * T00 * dg00;
    for (int i = 0; i < 3; ++i) {
      double dg0i = 0.;
      for (int k = 0; k < 3; ++k) dg0i += beta[k] * dg[sym[i][k]] + g[sym[i][k]] * db[k];
      acc += T0[i] * dg0i;
    }
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) acc += 0.5 * T[i][k] * dg[sym[i][k]];
    sS[jd] = alp * acc;
  }
}

// HLL(E) flux (riemann_solvers.hh:60-70)
inline double hll(double fL, double fR, double uL, double uR, double cmin, double cmax) {
  return (cmax * fL + cmin * fR - cmax * cmin * (uR - uL)) / (cmax + cmin);
}

// ---------------------------------------------------------------------------
// Reconstruction at face i-1/2 from u[0..5] = cells i-3 .. i+2
// ---------------------------------------------------------------------------
// WENO-Z, 5th order, exponent 2, eps 1e-42 (weno_reconstruction.hh:174-278;
// Borges et al. 2008).  uL from cells i-3..i+1, uR from cells i-2..i+2.
inline void weno_z(const double u[6], double& uL, double& uR) {
  const double c13 = 13.0 / 12.0, c14 = 0.25, eps = 1.0e-42;
  const double um3 = u[0], um2 = u[1], um1 = u[2], u0 = u[3], up1 = u[4], up2 = u[5];
  auto sq = [](double x) { return x * x; };
  {
    const double b0 = c13 * sq(um2 + u0 - 2.0 * um1) + c14 * sq(um2 + 3.0 * u0 - 4.0 * um1);
    const double b1 = c13 * sq(um1 + up1 - 2.0 * u0) + c14 * sq(um1 - up1);
    const double b2 = c13 * sq(up2 + u0 - 2.0 * up1) + c14 * sq(up2 + 3.0 * u0 - 4.0 * up1);
    const double t5 = std::fabs(b0 - b2);
    const double i0 = sq(t5 / (b0 + eps)), i1 = sq(t5 / (b1 + eps)), i2 = sq(t5 / (b2 + eps));
    const double f0 = 2.0 * up2 - 7.0 * up1 + 11.0 * u0;
    const double f1 = -1.0 * up1 + 5.0 * u0 + 2.0 * um1;
    const double f2 = 2.0 * u0 + 5.0 * um1 - um2;
    const double a0 = 0.1 * (1.0 + i2), a1 = 0.6 * (1.0 + i1), a2 = 0.3 * (1.0 + i0);
    uR = (f0 * a0 + f1 * a1 + f2 * a2) / (6.0 * (a0 + a1 + a2));
  }
  {
    const double b0 = c13 * sq(um3 + um1 - 2.0 * um2) + c14 * sq(um3 + 3.0 * um1 - 4.0 * um2);
    const double b1 = c13 * sq(um2 + u0 - 2.0 * um1) + c14 * sq(um2 - u0);
    const double b2 = c13 * sq(up1 + um1 - 2.0 * u0) + c14 * sq(up1 + 3.0 * um1 - 4.0 * u0);
    const double t5 = std::fabs(b0 - b2);
    const double i0 = sq(t5 / (b0 + eps)), i1 = sq(t5 / (b1 + eps)), i2 = sq(t5 / (b2 + eps));
    const double f0 = 2.0 * um3 - 7.0 * um2 + 11.0 * um1;
    const double f1 = -1.0 * um2 + 5.0 * um1 + 2.0 * u0;
    const double f2 = 2.0 * um1 + 5.0 * u0 - up1;
    const double a0 = 0.1 * (1.0 + i0), a1 = 0.6 * (1.0 + i1), a2 = 0.3 * (1.0 + i2);
    uL = (f0 * a0 + f1 * a1 + f2 * a2) / (6.0 * (a0 + a1 + a2));
  }
}
// minmod / MC(beta=2) limiters (limiters.hh:42-80)
inline double lim_minmod(double sl, double sr) {
  return 0.5 * (std::copysign(1.0, sl) + std::copysign(1.0, sr)) *
         std::min(std::fabs(sl), std::fabs(sr));
}
inline double lim_mc2(double sl, double sr) {
  const double sc = 0.5 * (sr + sl);
  const double s = std::copysign(1.0, sr);
  return s * std::max(0., std::min(std::min(2. * std::fabs(sr), 2. * s * sl), s * sc));
}
// slope-limited / donor (reconstruction.hh:51-142)
inline void recon(int kind, const double u[6], double& uL, double& uR) {
  if (kind == GRB_RECON_WENOZ) { weno_z(u, uL, uR); return; }
  if (kind == GRB_RECON_DONOR) { uL = u[2]; uR = u[3]; return; }
  double (*lim)(double, double) = (kind == GRB_RECON_MC2) ? lim_mc2 : lim_minmod;
  uR = u[3] - 0.5 * lim(u[3] - u[2], u[4] - u[3]);
  uL = u[2] + 0.5 * lim(u[2] - u[1], u[3] - u[2]);
}

// 4-point face interpolation (grmhd_helpers.hh:360-380): inner pair, outer
// pair, then combine.  v[0..3] = cells i-2, i-1, i, i+1.
inline double face_interp4(double um2, double um1, double u0, double up1) {
  return 0.5625 * (um1 + u0) + (-0.0625) * (um2 + up1);
}
// 6th-order centred first derivative (fd_subexpressions.hh:44-50)
inline double fd6(double m3, double m2, double m1, double p1, double p2, double p3, double invh) {
  return (1.0 / 60.0) * invh * (45.0 * (p1 - m1) - 9.0 * (p2 - m2) + (p3 - m3));
}

// ---------------------------------------------------------------------------
// Root finders
// ---------------------------------------------------------------------------
// Brent's zero finder, Brent (1973) "Algorithms for Minimization without
// Derivatives", ch. 4, procedure zero; tol = 2 eps |b| + t
// (rootfinding.hh:73-231).  F is called as f(x) and may carry state.
template <class F>
inline double brent(F& f, double a, double b, double t, int* iters = nullptr) {
  double sa = a, sb = b;
  double fa = f(sa), fb = f(sb);
  double c = sa, fc = fa, e = sb - sa, d = e;
  const double macheps = std::numeric_limits<double>::epsilon();
  int it = 0;
  for (;;) {
    if (std::fabs(fc) < std::fabs(fb)) {
      sa = sb; sb = c; c = sa;
      fa = fb; fb = fc; fc = fa;
    }
    const double tol = 2.0 * macheps * std::fabs(sb) + t;
    const double m = 0.5 * (c - sb);
    if (std::fabs(m) <= tol || fb == 0.0) break;
    if (std::fabs(e) < tol || std::fabs(fa) <= std::fabs(fb)) {
      e = m; d = e;
    } else {
      double s = fb / fa, p, q;
      if (sa == c) {
        p = 2.0 * m * s;
        q = 1.0 - s;
      } else {
        q = fa / fc;
        const double r = fb / fc;
        p = s * (2.0 * m * q * (q - r) - (sb - sa) * (r - 1.0));
        q = (q - 1.0) * (r - 1.0) * (s - 1.0);
      }
      if (0.0 < p) q = -q; else p = -p;
      s = e; e = d;
      if (2.0 * p < 3.0 * m * q - std::fabs(tol * q) && p < std::fabs(0.5 * s * q)) {
        d = p / q;
      } else {
        e = m; d = e;
      }
    }
    sa = sb; fa = fb;
    if (tol < std::fabs(d)) sb = sb + d;
    else if (0.0 < m) sb = sb + tol;
    else sb = sb - tol;
    fb = f(sb);
    ++it;
    if ((0.0 < fb && 0.0 < fc) || (fb <= 0.0 && fc <= 0.0)) {
      c = sa; fc = fa; e = sb - sa; d = e;
    }
  }
  if (iters) *iters += it;
  return sb;
}
// Safeguarded Newton-Raphson on a bracket (rootfinding.hh:255-306).
// F is called as f(x, fx, dfx).
template <class F>
inline double newton_bracketed(double sa, double sb, const F& f, unsigned long maxiter,
                               double tol, int& err) {
  const double macheps = std::numeric_limits<double>::epsilon();
  double a = sa, b = sb, fa, fb, dum;
  f(a, fa, dum);
  f(b, fb, dum);
  if (fa == 0) { err = 0; return a; }
  if (fb == 0) { err = 0; return b; }
  if (fa * fb > 0) { err = 1; return 0; }
  double x = (fb * a - fa * b) / (fb - fa);
  unsigned long iter = 0;
  do {
    const double xold = x;
    double fx, dfx;
    f(x, fx, dfx);
    if (fx * fb > 0) { fb = fx; b = x; }
    else if (fx * fa > 0) { fa = fx; a = x; }
    x -= fx / dfx;
    const double tt = 2. * macheps * std::fabs(x) + tol;
    if (std::fabs(x - xold) < tt || fx == 0) { err = 0; return x; }
    if (x > b || x < a) x = 0.5 * (b + a);
    iter++;
  } while (iter < maxiter);
  err = 1;
  return 0;
}

}  // namespace orc
