// CPU oracle — test infrastructure only (see grmhd_numerics.hpp).
//
// Restatement of GRACE's conservative-to-primitive policy: Kastaun et al.
// (2021) root solve with the entropy-based backup, conserved/primitive
// limiting, atmosphere and temperature floors, and the signal/reset bit
// bookkeeping.  Follows src/physics/eos/c2p.cpp:40-455,
// include/grace/physics/eos/kastaun_c2p.hh:44-402,
// include/grace/physics/eos/ent_based_c2p.hh:44-260 and
// include/grace/physics/eos/c2p.hh:124-316.
#pragma once
#include "grmhd_numerics.hpp"

namespace orc {

struct C2PParams {
  double rho_fl, ye_fl, temp_fl, atmo_tol;       // atmo_params_t
  int excise_by_radius;
  double r_ex, alp_ex;                           // excision_params_t
  double tol, max_w, max_sigma, beta_fallback, alp_bh_thresh;
  int use_ent_backup;                            // c2p_params_t
};
inline C2PParams make_c2p_params(const grb_params& p) {
  C2PParams c;
  c.rho_fl = p.rho_fl; c.ye_fl = p.ye_fl; c.temp_fl = p.temp_fl; c.atmo_tol = p.atmo_tol;
  c.excise_by_radius = p.excise_by_radius; c.r_ex = p.r_ex; c.alp_ex = p.alp_ex;
  c.tol = p.c2p_tol; c.max_w = p.max_w; c.max_sigma = p.max_sigma;
  c.beta_fallback = p.beta_fallback; c.alp_bh_thresh = p.alp_bh_thresh;
  c.use_ent_backup = p.use_ent_backup;
  return c;
}


// Fatal-condition bits returned alongside (the reference aborts there).
enum { FATAL_C2P_RHO_HIGH = 1, FATAL_EOS_RHO_HIGH = 2, FATAL_EOS_EPS_HIGH = 4,
       FATAL_EOS_TEMP_HIGH = 8, FATAL_EOS_PRESS_HIGH = 16 };

struct C2PStats { int brent_iters = 0; int newton_fail = 0; double mu = 0; int guess_used = 0; };

// Learned-bracket hook: if set, called with the Kastaun scalars; returns
// true and a bracket [lo, hi] to try before the plain one.
struct BracketGuess {
  bool valid = false;
  double lo = 0, hi = 0;
};

// --- prims -> cons (c2p.cpp:416-455)
inline void prims_to_conservs(const double pr[13], double cons[10], const Metric& m) {
  const double W = lorentz(m.g, pr + PR_ZX);
  double b[4], b2;
  comoving_b(m.alp, m.beta, m.g, pr + PR_BX, pr + PR_ZX, W, b, b2);
  double vt[3] = {0, 0, 0};  // fluxes are not needed; direction irrelevant
  double D, tau, S[3], ents, fD, ft, fS[3], fe;
  cons_and_flux(m.alp, m.beta, m.g, pr[PR_RHO], pr[PR_PRESS], pr[PR_EPS], pr + PR_ZX,
                pr[PR_ENT], W, b2, b, vt, 0, D, tau, S, ents, fD, ft, fS, fe);
  cons[CONS_D] = m.sqrtg * D;
  cons[CONS_SX] = m.sqrtg * S[0];
  cons[CONS_SY] = m.sqrtg * S[1];
  cons[CONS_SZ] = m.sqrtg * S[2];
  cons[CONS_TAU] = m.sqrtg * tau;
  cons[CONS_ENTS] = m.sqrtg * ents;
  cons[CONS_YES] = cons[CONS_D] * pr[PR_YE];
}

inline void set_all_resets(uint32_t& e) {
  setb(e, E_RESET_DENS); setb(e, E_RESET_TAU); setb(e, E_RESET_STILDE);
  setb(e, E_RESET_ENTROPY); setb(e, E_RESET_YE);
}

// c2p_handle_signals (c2p.hh:152-222); has_ye is false for the ideal and
// hybrid-polytrope EOSes (eos_types.hh:46-50).
inline void handle_signals(uint32_t sig, bool lenient, uint32_t& err, int& fatal) {
  if (tstb(sig, S_RHO_TOO_HIGH)) {
    setb(err, E_SIG_RHO_TOO_HIGH);
    set_all_resets(err);                        // lenient branch; the strict
    if (!lenient) fatal |= FATAL_C2P_RHO_HIGH;  // one aborts in the reference
  }
  if (tstb(sig, S_RHO_TOO_LOW)) {
    setb(err, E_RESET_DENS); setb(err, E_RESET_TAU); setb(err, E_RESET_STILDE);
    setb(err, E_RESET_ENTROPY); setb(err, E_SIG_RHO_TOO_LOW);
  }
  if (tstb(sig, S_ENT_TOO_LOW)) { setb(err, E_RESET_ENTROPY); setb(err, E_SIG_ENT_TOO_LOW); }
  if (tstb(sig, S_ENT_TOO_HIGH)) { setb(err, E_RESET_ENTROPY); setb(err, E_SIG_ENT_TOO_HIGH); }
  if (tstb(sig, S_EPS_TOO_HIGH)) { setb(err, E_RESET_STILDE); setb(err, E_RESET_TAU); setb(err, E_SIG_EPS_TOO_HIGH); }
  if (tstb(sig, S_EPS_TOO_LOW)) { setb(err, E_RESET_STILDE); setb(err, E_RESET_TAU); setb(err, E_SIG_EPS_TOO_LOW); }
  if (tstb(sig, S_VEL_TOO_HIGH)) {
    setb(err, E_RESET_DENS); setb(err, E_RESET_TAU); setb(err, E_RESET_STILDE);
    setb(err, E_RESET_ENTROPY); setb(err, E_SIG_VEL_TOO_HIGH);
  }
  if (tstb(sig, S_SIGMA_TOO_HIGH)) {
    setb(err, E_RESET_DENS); setb(err, E_RESET_TAU); setb(err, E_RESET_STILDE);
    setb(err, E_RESET_ENTROPY); setb(err, E_SIG_SIGMA_TOO_HIGH);
  }
}
// c2p_handle_eos_signals (c2p.hh:236-316)
inline void handle_eos_signals(uint32_t q, bool lenient, uint32_t& err, int& fatal) {
  if (tstb(q, Q_RHO_TOO_HIGH)) { setb(err, E_SIG_RHO_TOO_HIGH); fatal |= FATAL_EOS_RHO_HIGH; }
  if (tstb(q, Q_RHO_TOO_LOW)) {
    setb(err, E_RESET_DENS); setb(err, E_RESET_TAU); setb(err, E_RESET_STILDE);
    setb(err, E_RESET_ENTROPY); setb(err, E_SIG_RHO_TOO_LOW);
  }
  if (tstb(q, Q_ENT_TOO_HIGH)) { setb(err, E_RESET_ENTROPY); setb(err, E_SIG_ENT_TOO_HIGH); }
  if (tstb(q, Q_ENT_TOO_LOW)) { setb(err, E_RESET_ENTROPY); setb(err, E_SIG_ENT_TOO_LOW); }
  if (tstb(q, Q_EPS_TOO_HIGH)) {
    setb(err, E_SIG_EPS_TOO_HIGH);
    if (!lenient) fatal |= FATAL_EOS_EPS_HIGH;
    setb(err, E_RESET_STILDE); setb(err, E_RESET_TAU);
  }
  if (tstb(q, Q_EPS_TOO_LOW)) { setb(err, E_RESET_STILDE); setb(err, E_RESET_TAU); setb(err, E_SIG_EPS_TOO_LOW); }
  if (tstb(q, Q_TEMP_TOO_HIGH)) {
    setb(err, E_SIG_TEMP_TOO_HIGH);
    if (!lenient) fatal |= FATAL_EOS_TEMP_HIGH;
    setb(err, E_RESET_STILDE); setb(err, E_RESET_TAU);
  }
  if (tstb(q, Q_TEMP_TOO_LOW)) { setb(err, E_RESET_STILDE); setb(err, E_RESET_TAU); setb(err, E_SIG_TEMP_TOO_LOW); }
  if (tstb(q, Q_PRESS_TOO_HIGH)) {
    setb(err, E_SIG_PRESS_TOO_HIGH);
    if (!lenient) fatal |= FATAL_EOS_PRESS_HIGH;
    setb(err, E_RESET_STILDE); setb(err, E_RESET_TAU);
  }
  if (tstb(q, Q_PRESS_TOO_LOW)) { setb(err, E_RESET_STILDE); setb(err, E_RESET_TAU); setb(err, E_SIG_PRESS_TOO_LOW); }
}

// Kastaun bracket helper f(mu) = mu sqrt(h0^2 + rbar_f^2(mu)) - 1
// (kastaun_c2p.hh:44-117)
struct KBracket {
  double rsqr, bsqr, rbsqr, h0sqr;
  double xmu(double mu) const { return 1. / (1. + mu * bsqr); }
  double rb2(double mu, double x) const { return x * (rsqr * x + mu * (x + 1.0) * rbsqr); }
  void operator()(double mu, double& f, double& df) const {
    const double x = xmu(mu), x2 = x * x;
    const double hw = std::sqrt(h0sqr + rb2(mu, x));
    const double b = x * (x2 * rsqr + mu * (1 + x + x2) * rbsqr);
    f = mu * hw - 1.;
    df = (h0sqr + b) / hw;
  }
  double operator()(double mu) const {
    const double x = xmu(mu);
    return mu * std::sqrt(h0sqr + rb2(mu, x)) - 1.;
  }
  void bracket(double& lo, double& hi) const {
    lo = 1. / (h0sqr + rsqr);
    const double mu0 = 1. / std::sqrt(h0sqr);
    hi = 1.0 / std::sqrt(h0sqr + rb2(mu0, xmu(mu0)));
    lo *= (1 - 1e-10);
    hi *= (1 + 1e-10);
    if (hi <= lo) { lo = 0; hi = mu0 * (1.0 + 1e-10); }
  }
};

// Kastaun master function f(mu) = mu - 1/(hbw + rbar_f^2 mu)
// (kastaun_c2p.hh:122-295)
struct KRoot {
  const Eos* eos;
  double d, qtot, ye, rsqr, bsqr, rbsqr, brosqr, vsqrmax, wmax;
  KRoot(const Eos& e, double d_, double q_, double rsqr_, double rbsqr_, double bsqr_,
        double ye_, double h0)
      : eos(&e), d(d_), qtot(q_), ye(ye_), rsqr(rsqr_), bsqr(bsqr_), rbsqr(rbsqr_),
        brosqr(rsqr_ * bsqr_ - rbsqr_) {
    const double zs = rsqr / (h0 * h0);
    const double ws = 1 + zs;
    wmax = std::sqrt(ws);
    vsqrmax = zs / ws;
  }
  double xmu(double mu) const { return 1. / (1. + mu * bsqr); }
  double rf2(double mu, double x) const { return x * (rsqr * x + mu * (x + 1.0) * rbsqr); }
  double qf(double mu, double x) const {
    const double mx = mu * x;
    return qtot - 0.5 * (bsqr + mx * mx * brosqr);
  }
  double eps_raw(double mu, double q, double rf, double w) const {
    return w * (q - mu * rf * (1.0 - mu * w / (1 + w)));
  }
  double operator()(double mu) {
    const double x = xmu(mu), rf = rf2(mu, x), q = qf(mu, x);
    double vsqr = rf * mu * mu, w;
    if (vsqr > vsqrmax) { vsqr = vsqrmax; w = wmax; }
    else w = 1 / std::sqrt(1 - vsqr);
    double rho = std::fmin(eos->rhomax, std::fmax(eos->rhomin, d / w));
    double eps = eps_raw(mu, q, rf, w);
    double lo, hi;
    uint32_t qe = 0;
    double rr = rho;
    eps_range__rho(*eos, lo, hi, rr, qe);
    eps = std::fmin(hi, std::fmax(lo, eps));
    const double press = press__eps_rho(*eos, eps, rho, qe);
    const double a = press / (rho * (1 + eps));
    const double h = (1 + eps) * (1 + a);
    const double hbw = std::fmax((1 + a) * (1 + q - mu * rf), h / w);
    return mu - 1. / (hbw + rf * mu);
  }
  double primitives(double mu, uint32_t& sig, double& x, double& w, double& rho,
                    double& press, double& eps, double& temp, double& ent) {
    x = xmu(mu);
    const double rf = rf2(mu, x), q = qf(mu, x);
    double vsqr = rf * mu * mu;
    if (vsqr > vsqrmax) { vsqr = vsqrmax; w = wmax; setb(sig, S_VEL_TOO_HIGH); }
    else w = 1 / std::sqrt(1 - vsqr);
    rho = d / w;
    if (rho >= eos->rhomax) { setb(sig, S_RHO_TOO_HIGH); rho = eos->rhomax; }
    else if (rho <= eos->rhomin) { setb(sig, S_RHO_TOO_LOW); rho = eos->rhomin; }
    eps = eps_raw(mu, q, rf, w);
    double lo, hi;
    uint32_t qe = 0;
    double rr = rho;
    eps_range__rho(*eos, lo, hi, rr, qe);
    hi = std::fmin(hi, eos->c2p_eps_max);
    if (eps >= hi) { setb(sig, S_EPS_TOO_HIGH); eps = hi * 0.999; }
    else if (eps < lo) { setb(sig, S_EPS_TOO_LOW); eps = lo; }
    double hh, cs2;
    press = press_h_csnd2_temp_entropy__eps_rho(*eos, hh, cs2, temp, ent, eps, rho, qe);
    const double a = press / (rho * (1 + eps));
    const double h = (1 + eps) * (1 + a);
    const double hbw = std::fmax((1 + a) * (1 + q - mu * rf), h / w);
    return mu - 1. / (hbw + rf * mu);
  }
};

// Entropy-based master function (ent_based_c2p.hh:44-170).  The entropy
// member is passed by reference into the EOS and stays clamped across
// evaluations, as in the reference.
struct ERoot {
  const Eos* eos;
  double d, s, ye, rsqr, bsqr, rbsqr, vsqrmax, wmax;
  ERoot(const Eos& e, double d_, double rsqr_, double rbsqr_, double bsqr_, double s_,
        double ye_, double h0)
      : eos(&e), d(d_), s(s_), ye(ye_), rsqr(rsqr_), bsqr(bsqr_), rbsqr(rbsqr_) {
    const double zs = rsqr / (h0 * h0);
    const double ws = 1 + zs;
    wmax = std::sqrt(ws);
    vsqrmax = zs / ws;
  }
  double xmu(double mu) const { return 1. / (1. + mu * bsqr); }
  double rf2(double mu, double x) const { return x * (rsqr * x + mu * (x + 1.0) * rbsqr); }
  double operator()(double mu) {
    const double x = xmu(mu), rf = rf2(mu, x);
    double vsqr = rf * mu * mu;
    double w = 1 / std::sqrt(1 - vsqr);
    if (vsqr > vsqrmax) { vsqr = vsqrmax; w = wmax; }
    double rho = std::fmin(eos->rhomax, std::fmax(eos->rhomin, d / w));
    double hh, cs2, temp, eps;
    uint32_t qe = 0;
    const double press = press_h_csnd2_temp_eps__entropy_rho(*eos, hh, cs2, temp, eps, s, rho, qe);
    const double a = press / (rho * (1 + eps));
    const double h = (1 + eps) * (1 + a);
    return mu - 1. / (h / w + rf * mu);
  }
  double primitives(double mu, uint32_t& sig, double& x, double& w, double& rho,
                    double& press, double& eps, double& temp, double& ent) {
    ent = s;
    x = xmu(mu);
    const double rf = rf2(mu, x);
    double vsqr = rf * mu * mu;
    w = 1 / std::sqrt(1 - vsqr);
    if (vsqr > vsqrmax) { vsqr = vsqrmax; w = wmax; setb(sig, S_VEL_TOO_HIGH); }
    rho = d / w;
    if (rho >= eos->rhomax) { setb(sig, S_RHO_TOO_HIGH); rho = eos->rhomax; }
    else if (rho <= eos->rhomin) { setb(sig, S_RHO_TOO_LOW); rho = eos->rhomin; }
    double hh, cs2;
    uint32_t qe = 0;
    press = press_h_csnd2_temp_eps__entropy_rho(*eos, hh, cs2, temp, eps, ent, rho, qe);
    if (tstb(qe, Q_ENT_TOO_LOW)) setb(sig, S_ENT_TOO_LOW);
    if (tstb(qe, Q_ENT_TOO_HIGH)) setb(sig, S_ENT_TOO_HIGH);
    const double a = press / (rho * (1 + eps));
    const double h = (1 + eps) * (1 + a);
    return mu - 1. / (h / w + rf * mu);
  }
};

// Shared set-up of the Kastaun scalars (kastaun_c2p.hh:306-337)
struct KScalars {
  double D, q, s, ye, r2, Bt2, rBt, rBt2, h0;
  double rup[3], Bt[3], B[3];
};
inline KScalars kastaun_setup(const Eos& e, const Metric& m, double cons[10]) {
  KScalars k;
  k.h0 = e.h_min;
  cons[CONS_D] = std::fmax(0, cons[CONS_D]);
  k.D = cons[CONS_D];
  k.q = cons[CONS_TAU] / k.D;
  k.s = cons[CONS_ENTS] / k.D;
  double r[3] = {cons[CONS_SX] / k.D, cons[CONS_SY] / k.D, cons[CONS_SZ] / k.D};
  const double sD = std::sqrt(k.D);
  for (int i = 0; i < 3; ++i) { k.Bt[i] = cons[CONS_BX + i] / sD; k.B[i] = cons[CONS_BX + i]; }
  k.r2 = sq_sym(m.ginv, r);
  k.Bt2 = sq_sym(m.g, k.Bt);
  k.rBt = r[0] * k.Bt[0] + r[1] * k.Bt[1] + r[2] * k.Bt[2];
  k.rBt2 = k.rBt * k.rBt;
  mul_sym(m.ginv, r, k.rup);
  k.ye = cons[CONS_YES] / k.D;
  return k;
}

// Upper end of the plain Kastaun bracket (kastaun_c2p.hh:355-369)
inline double kastaun_mu0(const KScalars& k) {
  double mu0 = 1 / k.h0;
  if (k.r2 >= k.h0 * k.h0) {
    KBracket g{k.r2, k.Bt2, k.rBt2, k.h0 * k.h0};
    double lo, hi;
    g.bracket(lo, hi);
    int err;
    mu0 = newton_bracketed(lo, hi, g, 30, 1e-10, err);
    if (err == 0) mu0 *= 1 + 1e-10;
    else mu0 = 1.0 / k.h0;
  }
  return mu0;
}

// kastaun_c2p_t::invert (kastaun_c2p.hh:352-395).  With a learned guess the
// Brent solve starts from [guess.lo, min(guess.hi, mu0)] when that bracket
// changes sign, and from the plain [0, mu0] otherwise.
inline double kastaun_invert(const Eos& e, const Metric& m, double cons[10], double pr[13],
                             uint32_t& sig, C2PStats* st, const BracketGuess* guess) {
  KScalars k = kastaun_setup(e, m, cons);
  KRoot f(e, k.D, k.q, k.r2, k.rBt2, k.Bt2, k.ye, k.h0);
  double mu;
  bool done = false;
  int* it = st ? &st->brent_iters : nullptr;
  const double mu0 = kastaun_mu0(k);
  if (guess && guess->valid) {
    const double lo = guess->lo, hi = std::fmin(guess->hi, mu0);
    if (hi > lo) {
      const double flo = f(lo), fhi = f(hi);
      if (flo * fhi < 0) {
        mu = brent(f, lo, hi, 1e-15, it);
        done = true;
        if (st) st->guess_used = 1;
      }
    }
  }
  if (!done) mu = brent(f, 0, mu0, 1e-15, it);
  double x, w, eps, rho, press, temp, ent;
  const double res = f.primitives(mu, sig, x, w, rho, press, eps, temp, ent);
  if (st) st->mu = mu;
  pr[PR_EPS] = eps; pr[PR_RHO] = rho; pr[PR_PRESS] = press; pr[PR_TEMP] = temp;
  pr[PR_ENT] = ent;
  for (int i = 0; i < 3; ++i) pr[PR_BX + i] = k.B[i];
  for (int i = 0; i < 3; ++i) pr[PR_ZX + i] = w * mu * x * (k.rup[i] + mu * k.rBt * k.Bt[i]);
  return std::fabs(res);
}

// entropy_fix_c2p_t::invert (ent_based_c2p.hh:210-245)
inline double entropy_invert(const Eos& e, const Metric& m, double cons[10], double pr[13],
                             uint32_t& sig) {
  KScalars k = kastaun_setup(e, m, cons);
  double mu0 = 1 / k.h0;
  if (k.r2 >= k.h0 * k.h0) {
    KBracket g{k.r2, k.Bt2, k.rBt2, k.h0 * k.h0};
    int rerr;
    mu0 = newton_bracketed(0, 1. / k.h0, g, 30, 1e-10, rerr);
    if (rerr == 0) mu0 *= 1 + 1e-10;
    else mu0 = brent(g, 0, 1. / k.h0, 1e-10) * (1 + 1e-10);
  }
  ERoot f(e, k.D, k.r2, k.rBt2, k.Bt2, k.s, k.ye, k.h0);
  const double mu = brent(f, 0, mu0, 1e-15);
  double x, w, eps, rho, press, temp, ent;
  const double res = f.primitives(mu, sig, x, w, rho, press, eps, temp, ent);
  pr[PR_EPS] = eps; pr[PR_RHO] = rho; pr[PR_PRESS] = press; pr[PR_TEMP] = temp;
  pr[PR_ENT] = ent;
  for (int i = 0; i < 3; ++i) pr[PR_BX + i] = k.B[i];
  for (int i = 0; i < 3; ++i) pr[PR_ZX + i] = w * mu * x * (k.rup[i] + mu * k.rBt * k.Bt[i]);
  return std::fabs(res);
}

// reset_to_atmosphere (c2p.cpp:159-186)
inline void reset_to_atmosphere(double cons[10], double pr[13], const Metric& m,
                                const C2PParams& c, const Eos& e, uint32_t& err) {
  pr[PR_RHO] = c.rho_fl;
  pr[PR_YE] = c.ye_fl;
  pr[PR_TEMP] = c.temp_fl;
  pr[PR_ZX] = pr[PR_ZY] = pr[PR_ZZ] = 0.;
  double cs2;
  uint32_t qe = 0;
  pr[PR_PRESS] = press_eps_csnd2_entropy__temp_rho(e, pr[PR_EPS], cs2, pr[PR_ENT], pr[PR_TEMP],
                                                   pr[PR_RHO], qe);
  prims_to_conservs(pr, cons, m);
  set_all_resets(err);
  setb(err, E_ATMO_RESET);
}

// limit_conservatives (c2p.cpp:117-157)
inline bool limit_conservatives(double cons[10], const Metric& m, const Eos& e, uint32_t& err) {
  bool any = false;
  double rhoL = cons[CONS_D];
  double lo, hi;
  uint32_t qe = 0;
  eps_range__rho(e, lo, hi, rhoL, qe);
  const double B2 = sq_sym(m.g, cons + CONS_BX);
  if (cons[CONS_TAU] / cons[CONS_D] - 0.5 * B2 / cons[CONS_D] < std::fmin(0.0, lo)) {
    cons[CONS_TAU] = lo * cons[CONS_D] + 0.5 * B2;
    setb(err, E_RESET_TAU);
    any = true;
  }
  const double qd = cons[CONS_TAU] / cons[CONS_D] + 1;
  const double st2max = qd * qd;
  const double st2 = sq_sym(m.ginv, cons + CONS_SX) / (cons[CONS_D] * cons[CONS_D]);
  if (st2 > st2max) {
    const double f = std::sqrt(st2max / st2);
    cons[CONS_SX] *= f; cons[CONS_SY] *= f; cons[CONS_SZ] *= f;
    setb(err, E_RESET_STILDE);
    any = true;
  }
  return any;
}

// limit_primitives (c2p.cpp:63-115)
inline void limit_primitives(double pr[13], const Metric& m, const Eos& e, double max_w,
                             double max_sigma, uint32_t& sig) {
  const double z2max = max_w * max_w - 1.;
  const double z2 = sq_sym(m.g, pr + PR_ZX);
  if (z2 >= z2max) {
    const double zn = 0.99 * std::sqrt(z2max / z2);
    pr[PR_ZX] *= zn; pr[PR_ZY] *= zn; pr[PR_ZZ] *= zn;
    setb(sig, S_VEL_TOO_HIGH);
  }
  const double W = lorentz(m.g, pr + PR_ZX);
  double b[4], b2;
  comoving_b(m.alp, m.beta, m.g, pr + PR_BX, pr + PR_ZX, W, b, b2);
  const double sigma = b2 / pr[PR_RHO];
  if (sigma >= max_sigma) {
    pr[PR_RHO] *= 1.001 * sigma / max_sigma;
    double cs2;
    uint32_t qe = 0;
    pr[PR_PRESS] = press_eps_csnd2_entropy__temp_rho(e, pr[PR_EPS], cs2, pr[PR_ENT],
                                                     pr[PR_TEMP], pr[PR_RHO], qe);
    setb(sig, S_SIGMA_TOO_HIGH);
  }
}

// conservs_to_prims (c2p.cpp:188-414).  cons in: densitized conserved with
// densitized cell-centred B; cons out: re-densitized conserved consistent
// with the returned primitives.  Returns the FOFC "floored" flag.
inline bool conservs_to_prims(double cons[10], double pr[13], const Metric& m, const Eos& e,
                              const C2PParams& c, double r_sph, uint32_t& err, bool dry_run,
                              int& fatal, C2PStats* st = nullptr,
                              const BracketGuess* guess = nullptr) {
  bool failed = false, floored = false;
  uint32_t ret = 0;
  err = 0;
  setb(err, E_RESET_ENTROPY);
  for (int v = 0; v < 10; ++v) cons[v] /= m.sqrtg;
  pr[PR_BX] = cons[CONS_BX]; pr[PR_BY] = cons[CONS_BY]; pr[PR_BZ] = cons[CONS_BZ];
  if (cons[CONS_D] < 0) {
    reset_to_atmosphere(cons, pr, m, c, e, err);
    return true;
  }
  pr[PR_YE] = cons[CONS_YES] / cons[CONS_D];
  if (pr[PR_YE] > e.yemax) { pr[PR_YE] = e.yemax; setb(err, E_RESET_YE); }
  if (pr[PR_YE] < e.yemin) { pr[PR_YE] = e.yemin; setb(err, E_RESET_YE); }
  const bool lenient = m.alp < c.alp_bh_thresh;
  floored |= limit_conservatives(cons, m, e, err);
  if (floored && dry_run) return floored;
  if (cons[CONS_D] >= c.rho_fl * (1 + c.atmo_tol)) {
    const double res = kastaun_invert(e, m, cons, pr, ret, st, guess);
    failed = (std::fabs(res) > c.tol) || tstb(ret, S_RHO_TOO_HIGH) ||
             tstb(ret, S_EPS_TOO_HIGH) || !std::isfinite(res);
    double beta;
    {
      const double W = lorentz(m.g, pr + PR_ZX);
      double b[4], b2;
      comoving_b(m.alp, m.beta, m.g, pr + PR_BX, pr + PR_ZX, W, b, b2);
      beta = 2.0 * pr[PR_PRESS] / std::fmax(b2, 1e-50);
    }
    const bool distrust = failed || tstb(ret, S_EPS_TOO_LOW) || (beta <= c.beta_fallback);
    if (distrust && c.use_ent_backup && !dry_run) {
      double save[13];
      for (int v = 0; v < 13; ++v) save[v] = pr[v];
      uint32_t bret = 0;
      const double rb = entropy_invert(e, m, cons, pr, bret);
      const bool ok = (std::fabs(rb) <= c.tol) && std::isfinite(rb) &&
                      (pr[PR_EPS] < e.c2p_eps_max);
      if (ok) {
        ret = bret;
        failed = false;
        setb(err, E_ENT_BACKUP_USED);
      } else if (!failed) {
        for (int v = 0; v < 13; ++v) pr[v] = save[v];
      }
    }
    if (tstb(ret, S_EPS_TOO_HIGH) || tstb(ret, S_RHO_TOO_LOW) || tstb(ret, S_RHO_TOO_HIGH) ||
        tstb(ret, S_VEL_TOO_HIGH))
      floored = true;
    if (e.kind == GRB_EOS_IDEAL_GAS && tstb(ret, S_EPS_TOO_LOW)) floored = true;
    handle_signals(ret, lenient, err, fatal);
  } else {
    failed = true;
  }
  const bool excise = c.excise_by_radius ? (r_sph <= c.r_ex) : (m.alp <= c.alp_ex);
  if (failed || excise || pr[PR_RHO] < (1. + c.atmo_tol) * c.rho_fl) {
    reset_to_atmosphere(cons, pr, m, c, e, err);
    floored = true;
  } else if (pr[PR_TEMP] < c.temp_fl) {
    pr[PR_TEMP] = c.temp_fl;
    double cs2;
    uint32_t qe = 0;
    pr[PR_PRESS] = press_eps_csnd2_entropy__temp_rho(e, pr[PR_EPS], cs2, pr[PR_ENT],
                                                     pr[PR_TEMP], pr[PR_RHO], qe);
    handle_eos_signals(qe, lenient, err, fatal);
    setb(err, E_RESET_TAU); setb(err, E_RESET_STILDE); setb(err, E_RESET_ENTROPY);
    setb(err, E_T_FLOORED);
    if (e.kind == GRB_EOS_IDEAL_GAS) floored = true;
  } else {
    uint32_t s2 = 0;
    limit_primitives(pr, m, e, c.max_w, c.max_sigma, s2);
    handle_signals(s2, lenient, err, fatal);
    if (tstb(s2, S_VEL_TOO_HIGH) || tstb(s2, S_SIGMA_TOO_HIGH)) floored = true;
  }
  prims_to_conservs(pr, cons, m);
  return floored;
}

}  // namespace orc
