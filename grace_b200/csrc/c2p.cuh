// Device conservative-to-primitive recovery (FP64), following
// src/physics/eos/c2p.cpp:40-455, include/grace/physics/eos/c2p.hh:124-316,
// include/grace/physics/eos/kastaun_c2p.hh:44-402 and
// include/grace/physics/eos/ent_based_c2p.hh:44-260.  Root solves are
// Brent's method (Brent 1973, "zero") and the safeguarded Newton of
// include/grace/utils/rootfinding.hh:73-306.  Every loop is bounded: Brent
// by an iteration cap far above its convergence bound for the 1e-15
// abscissa tolerance, Newton by its 30-step limit.
#pragma once
#include "physics.cuh"

namespace grb {

// fatal conditions (the reference calls Kokkos::abort there) -> status bits
enum : uint32_t {
  FAT_C2P_RHO_HIGH = GRB_FLAG_C2P_RHO_TOO_HIGH, FAT_EOS_RHO_HIGH = GRB_FLAG_EOS_RHO_TOO_HIGH,
  FAT_EOS_EPS_HIGH = GRB_FLAG_EOS_EPS_TOO_HIGH, FAT_EOS_TEMP_HIGH = GRB_FLAG_EOS_TEMP_TOO_HIGH,
  FAT_EOS_PRESS_HIGH = GRB_FLAG_EOS_PRESS_TOO_HIGH
};
constexpr int kBrentMaxIter = 200;

// Brent's zero finder on [a,b] with tol = 2 eps |b| + t, given f(a) and
// f(b) already evaluated (fa0, fb0).  F: double(double).
template <class F>
GRB_HD double brent_f(F& f, double a, double b, double fa0, double fb0, double t, int& iters) {
  double sa = a, sb = b;
  double fa = fa0, fb = fb0;
  double c = sa, fc = fa, e = sb - sa, d = e;
  const double macheps = 2.220446049250313e-16;
  for (int it = 0; it < kBrentMaxIter; ++it) {
    if (fabs(fc) < fabs(fb)) {
      sa = sb; sb = c; c = sa;
      fa = fb; fb = fc; fc = fa;
    }
    const double tol = 2.0 * macheps * fabs(sb) + t;
    const double m = 0.5 * (c - sb);
    if (fabs(m) <= tol || fb == 0.0) break;
    if (fabs(e) < tol || fabs(fa) <= fabs(fb)) {
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
      if (2.0 * p < 3.0 * m * q - fabs(tol * q) && p < fabs(0.5 * s * q)) d = p / q;
      else { e = m; d = e; }
    }
    sa = sb; fa = fb;
    if (tol < fabs(d)) sb = sb + d;
    else if (0.0 < m) sb = sb + tol;
    else sb = sb - tol;
    fb = f(sb);
    ++iters;
    if ((0.0 < fb && 0.0 < fc) || (fb <= 0.0 && fc <= 0.0)) {
      c = sa; fc = fa; e = sb - sa; d = e;
    }
  }
  return sb;
}
template <class F>
GRB_HD double brent(F& f, double a, double b, double t, int& iters) {
  const double fa = f(a);
  const double fb = f(b);
  return brent_f(f, a, b, fa, fb, t, iters);
}

// Kastaun auxiliary function mu sqrt(h0^2 + rbar^2(mu)) - 1 (kastaun_c2p.hh:44-117)
struct KBr {
  double rsqr, bsqr, rbsqr, h0sqr;
  GRB_HD double xmu(double mu) const { return 1. / (1. + mu * bsqr); }
  GRB_HD double rb2(double mu, double x) const { return x * (rsqr * x + mu * (x + 1.0) * rbsqr); }
  GRB_HD double operator()(double mu) const {
    const double x = xmu(mu);
    return mu * sqrt(h0sqr + rb2(mu, x)) - 1.;
  }
  GRB_HD void fdf(double mu, double& f, double& df) const {
    const double x = xmu(mu), x2 = x * x;
    const double hw = sqrt(h0sqr + rb2(mu, x));
    const double b = x * (x2 * rsqr + mu * (1 + x + x2) * rbsqr);
    f = mu * hw - 1.;
    df = (h0sqr + b) / hw;
  }
};
GRB_HD double newton_br(double sa, double sb, const KBr& g, int maxiter, double tol, int& err) {
  const double macheps = 2.220446049250313e-16;
  double a = sa, b = sb, fa, fb, dum;
  g.fdf(a, fa, dum);
  g.fdf(b, fb, dum);
  if (fa == 0) { err = 0; return a; }
  if (fb == 0) { err = 0; return b; }
  if (fa * fb > 0) { err = 1; return 0; }
  double x = (fb * a - fa * b) / (fb - fa);
  for (int it = 0; it < maxiter; ++it) {
    const double xold = x;
    double fx, dfx;
    g.fdf(x, fx, dfx);
    if (fx * fb > 0) { fb = fx; b = x; }
    else if (fx * fa > 0) { fa = fx; a = x; }
    x -= fx / dfx;
    const double tt = 2. * macheps * fabs(x) + tol;
    if (fabs(x - xold) < tt || fx == 0) { err = 0; return x; }
    if (x > b || x < a) x = 0.5 * (b + a);
  }
  err = 1;
  return 0;
}

// Kastaun scalars (kastaun_c2p.hh:306-337)
struct KSc {
  double D, iD, q, s, ye, r2, Bt2, rBt, rBt2, h0, ih0;
  double rup[3], Bt[3], B[3];
};
GRB_HD KSc kscalars(const DevEos& e, const Met& m, double c[10]) {
  KSc k;
  k.h0 = e.h_min;
  k.ih0 = e.ih0;  // 1/h_min, correctly rounded on the host as 1 / k.h0 is here
  c[0] = fmax(0., c[0]);
  k.D = c[0];
  const double iD = 1.0 / k.D;
  k.iD = iD;
  k.q = c[4] * iD;
  k.s = c[6] * iD;
  const double r[3] = {c[1] * iD, c[2] * iD, c[3] * iD};
  const double isD = 1.0 / sqrt(k.D);
#pragma unroll
  for (int i = 0; i < 3; ++i) { k.B[i] = c[7 + i]; k.Bt[i] = c[7 + i] * isD; }
  k.r2 = sqs(m.gi, r);
  k.Bt2 = sqs(m.g, k.Bt);
  k.rBt = r[0] * k.Bt[0] + r[1] * k.Bt[1] + r[2] * k.Bt[2];
  k.rBt2 = k.rBt * k.rBt;
  mvs(m.gi, r, k.rup);
  k.ye = c[5] * iD;
  return k;
}

// Kastaun master function (kastaun_c2p.hh:122-295).  FAST (tuned mode): the
// same function up to rounding with three divisions per evaluation instead
// of five: rho = D sqrt(1 - v^2) and h/W = h sqrt(1 - v^2); W and
// W/(1+W) = 1/(1 + 1/W) from one reciprocal of (1/W)(1 + 1/W);
// h = (1+eps)(1+a) with a = P/(rho(1+eps)) formed as 1 + eps + P/rho, with
// 1/rho = W/D; and nu = max(nu_A, nu_B), nu_A = (1+a)(1+q-mu r^2) =
// h (1+q-mu r^2)/(1+eps), nu_B = h/W, decided by comparing
// 1+q-mu r^2 with (1+eps)/W (h, 1+eps > 0), so that 1/(nu + mu r^2) takes
// one division either way.
template <bool FAST = false>
struct KRt {
  const DevEos* e;
  double d, qtot, rsqr, bsqr, rbsqr, brosqr, vsqrmax, wmax;
  double id, iwmax, w1max;  // FAST: 1/D, 1/wmax, wmax/(1+wmax)
  GRB_HD KRt(const DevEos& eos, const KSc& k) : e(&eos) {
    d = k.D; qtot = k.q; rsqr = k.r2; bsqr = k.Bt2; rbsqr = k.rBt2;
    brosqr = rsqr * bsqr - rbsqr;
    id = iwmax = w1max = 0.0;
    if (FAST) {
      // 1/ws, 1/wmax and 1/(1 + wmax) from one reciprocal (all >= 1)
      const double zs = rsqr * (k.ih0 * k.ih0);
      const double ws = 1 + zs;
      wmax = sqrt(ws);
      const double r = 1.0 / (ws * wmax * (1 + wmax));
      vsqrmax = zs * (wmax * (1 + wmax)) * r;
      iwmax = ws * (1 + wmax) * r;
      w1max = wmax * (ws * wmax) * r;
      id = k.iD;
    } else {
      const double zs = rsqr / (k.h0 * k.h0);
      const double ws = 1 + zs;
      wmax = sqrt(ws);
      vsqrmax = zs / ws;
    }
  }
  // FAST form of eval (same arguments and results).
  GRB_HD double eval_f(double mu, bool full, uint32_t& sig, double& x, double& w, double& rho,
                       double& press, double& eps, double& temp, double& ent) const {
    x = 1. / (1. + mu * bsqr);
    const double rf = x * (rsqr * x + mu * (x + 1.0) * rbsqr);
    const double mx = mu * x;
    const double qf = qtot - 0.5 * (bsqr + mx * mx * brosqr);
    const double vsqr = rf * mu * mu;
    double iw, w1;  // 1/W and W/(1+W)
    if (vsqr > vsqrmax) {
      w = wmax;
      iw = iwmax;
      w1 = w1max;
      if (full) sig |= SIG_VEL_HIGH;
    } else {
      iw = sqrt(1 - vsqr);
      const double r = 1.0 / (iw * (1.0 + iw));
      w = (1.0 + iw) * r;
      w1 = iw * r;
    }
    rho = d * iw;
    const double rho0 = rho;
    if (full) {
      if (rho >= e->rhomax) { sig |= SIG_RHO_HIGH; rho = e->rhomax; }
      else if (rho <= e->rhomin) { sig |= SIG_RHO_LOW; rho = e->rhomin; }
    } else {
      rho = fmin(e->rhomax, fmax(e->rhomin, rho));
    }
    const double irho = rho == rho0 ? w * id : 1.0 / rho;
    eps = w * (qf - mu * rf * (1.0 - mu * w1));
    double lo, hi;
    eos_eps_range(*e, lo, hi, rho);
    uint32_t qe = 0;
    if (full) {
      hi = fmin(hi, e->eps_max);
      if (eps >= hi) { sig |= SIG_EPS_HIGH; eps = hi * 0.999; }
      else if (eps < lo) { sig |= SIG_EPS_LOW; eps = lo; }
      press = eos_Peps_full(*e, temp, ent, eps, rho, qe);
    } else {
      eps = fmin(hi, fmax(lo, eps));
      press = eos_Peps(*e, eps, rho, qe);
    }
    const double h = 1 + eps + press * irho;
    const double qa = 1 + qf - mu * rf;
    const double rmu = rf * mu;
    if (qa >= iw * (1 + eps)) return mu - (1 + eps) / (h * qa + rmu * (1 + eps));
    return mu - 1. / (h * iw + rmu);
  }
  GRB_HD double eval(double mu, bool full, uint32_t& sig, double& x, double& w, double& rho,
                     double& press, double& eps, double& temp, double& ent) const {
    if (FAST) return eval_f(mu, full, sig, x, w, rho, press, eps, temp, ent);
    x = 1. / (1. + mu * bsqr);
    const double rf = x * (rsqr * x + mu * (x + 1.0) * rbsqr);
    const double mx = mu * x;
    const double qf = qtot - 0.5 * (bsqr + mx * mx * brosqr);
    const double vsqr = rf * mu * mu;
    if (vsqr > vsqrmax) {
      w = wmax;
      if (full) sig |= SIG_VEL_HIGH;
    } else {
      w = 1 / sqrt(1 - vsqr);
    }
    rho = d / w;
    if (full) {
      if (rho >= e->rhomax) { sig |= SIG_RHO_HIGH; rho = e->rhomax; }
      else if (rho <= e->rhomin) { sig |= SIG_RHO_LOW; rho = e->rhomin; }
    } else {
      rho = fmin(e->rhomax, fmax(e->rhomin, rho));
    }
    eps = w * (qf - mu * rf * (1.0 - mu * w / (1 + w)));
    double lo, hi;
    eos_eps_range(*e, lo, hi, rho);
    uint32_t qe = 0;
    if (full) {
      hi = fmin(hi, e->eps_max);
      if (eps >= hi) { sig |= SIG_EPS_HIGH; eps = hi * 0.999; }
      else if (eps < lo) { sig |= SIG_EPS_LOW; eps = lo; }
      press = eos_Peps_full(*e, temp, ent, eps, rho, qe);
    } else {
      eps = fmin(hi, fmax(lo, eps));
      press = eos_Peps(*e, eps, rho, qe);
    }
    const double a = press / (rho * (1 + eps));
    const double h = (1 + eps) * (1 + a);
    const double hbw = fmax((1 + a) * (1 + qf - mu * rf), h / w);
    return mu - 1. / (hbw + rf * mu);
  }
  GRB_HD double operator()(double mu) const {
    uint32_t s = 0;
    double x, w, rho, p, eps, t, en;
    return eval(mu, false, s, x, w, rho, p, eps, t, en);
  }
};

// Entropy master function (ent_based_c2p.hh:44-170); s persists clamped.
struct ERt {
  const DevEos* e;
  double d, s, rsqr, bsqr, rbsqr, vsqrmax, wmax;
  GRB_HD ERt(const DevEos& eos, const KSc& k) : e(&eos) {
    d = k.D; s = k.s; rsqr = k.r2; bsqr = k.Bt2; rbsqr = k.rBt2;
    const double zs = rsqr / (k.h0 * k.h0);
    const double ws = 1 + zs;
    wmax = sqrt(ws);
    vsqrmax = zs / ws;
  }
  GRB_HD double eval(double mu, double& ent, bool full, uint32_t& sig, double& x, double& w,
                     double& rho, double& press, double& eps, double& temp) {
    x = 1. / (1. + mu * bsqr);
    const double rf = x * (rsqr * x + mu * (x + 1.0) * rbsqr);
    const double vsqr = rf * mu * mu;
    w = 1 / sqrt(1 - vsqr);
    if (vsqr > vsqrmax) { w = wmax; if (full) sig |= SIG_VEL_HIGH; }
    rho = d / w;
    if (full) {
      if (rho >= e->rhomax) { sig |= SIG_RHO_HIGH; rho = e->rhomax; }
      else if (rho <= e->rhomin) { sig |= SIG_RHO_LOW; rho = e->rhomin; }
    } else {
      rho = fmin(e->rhomax, fmax(e->rhomin, rho));
    }
    uint32_t qe = 0;
    press = eos_Pent(*e, temp, eps, ent, rho, qe);
    if (full) {
      if (qe & EOS_ENT_LOW) sig |= SIG_ENT_LOW;
      if (qe & EOS_ENT_HIGH) sig |= SIG_ENT_HIGH;
    }
    const double a = press / (rho * (1 + eps));
    const double h = (1 + eps) * (1 + a);
    return mu - 1. / (h / w + rf * mu);
  }
  GRB_HD double operator()(double mu) {
    uint32_t sg = 0;
    double x, w, rho, p, eps, t;
    return eval(mu, s, false, sg, x, w, rho, p, eps, t);
  }
};

GRB_HD double kastaun_mu0(const KSc& k) {
  double mu0 = k.ih0;  // = 1 / k.h0
  if (k.r2 >= k.h0 * k.h0) {
    KBr g{k.r2, k.Bt2, k.rBt2, k.h0 * k.h0};
    double lo = 1. / (g.h0sqr + g.rsqr);
    const double m0 = 1. / sqrt(g.h0sqr);
    double hi = 1.0 / sqrt(g.h0sqr + g.rb2(m0, g.xmu(m0)));
    lo *= (1 - 1e-10);
    hi *= (1 + 1e-10);
    if (hi <= lo) { lo = 0; hi = m0 * (1.0 + 1e-10); }
    int err;
    mu0 = newton_br(lo, hi, g, 30, 1e-10, err);
    if (err == 0) mu0 *= 1 + 1e-10;
    else mu0 = k.ih0;
  }
  return mu0;
}

// Optional learned bracket for the Kastaun solve.  mu0 (has_mu0): the plain
// bracket top already computed from the unchanged state.
struct Guess {
  bool valid;
  double lo, hi;
  double mu0;
  bool has_mu0;
};
GRB_HD Guess no_guess() { return Guess{false, 0., 0., 0., false}; }

// kastaun_c2p_t::invert (kastaun_c2p.hh:352-395).  With a learned bracket
// the unchanged Brent iteration starts from [gs.lo, gs.hi] when f changes
// sign there (the two end values are the iteration's own first two
// evaluations), and from the plain [0, mu0] otherwise.
template <bool FAST = false>
GRB_HD double kastaun_invert(const DevEos& e, const Met& m, double c[10], double pr[13],
                             uint32_t& sig, int& iters, const Guess& gs, bool& guess_used,
                             double& mu_out) {
  const KSc k = kscalars(e, m, c);
  const KRt<FAST> f(e, k);
  double mu;
  guess_used = false;
  const double mu0 = gs.has_mu0 ? gs.mu0 : kastaun_mu0(k);
  if (gs.valid) {
    const double lo = gs.lo, hi = fmin(gs.hi, mu0);
    if (hi > lo) {
      const double flo = f(lo), fhi = f(hi);
      if (flo * fhi < 0) {
        mu = brent_f(f, lo, hi, flo, fhi, 1e-15, iters);
        guess_used = true;
      }
    }
  }
  if (!guess_used) mu = brent(f, 0, mu0, 1e-15, iters);
  double x, w, rho, press, eps, temp, ent;
  const double res = f.eval(mu, true, sig, x, w, rho, press, eps, temp, ent);
  mu_out = mu;
  pr[GRB_P_EPS] = eps; pr[GRB_P_RHO] = rho; pr[GRB_P_PRESS] = press;
  pr[GRB_P_TEMP] = temp; pr[GRB_P_ENT] = ent;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    pr[GRB_P_BX + i] = k.B[i];
    pr[GRB_P_ZX + i] = w * mu * x * (k.rup[i] + mu * k.rBt * k.Bt[i]);
  }
  return fabs(res);
}

GRB_HD double entropy_invert(const DevEos& e, const Met& m, double c[10], double pr[13],
                             uint32_t& sig) {
  const KSc k = kscalars(e, m, c);
  double mu0 = 1 / k.h0;
  int it = 0;
  if (k.r2 >= k.h0 * k.h0) {
    KBr g{k.r2, k.Bt2, k.rBt2, k.h0 * k.h0};
    int rerr;
    mu0 = newton_br(0, 1. / k.h0, g, 30, 1e-10, rerr);
    if (rerr == 0) mu0 *= 1 + 1e-10;
    else mu0 = brent(g, 0, 1. / k.h0, 1e-10, it) * (1 + 1e-10);
  }
  ERt f(e, k);
  const double mu = brent(f, 0, mu0, 1e-15, it);
  double x, w, rho, press, eps, temp;
  double ent = f.s;
  const double res = f.eval(mu, ent, true, sig, x, w, rho, press, eps, temp);
  pr[GRB_P_EPS] = eps; pr[GRB_P_RHO] = rho; pr[GRB_P_PRESS] = press;
  pr[GRB_P_TEMP] = temp; pr[GRB_P_ENT] = ent;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    pr[GRB_P_BX + i] = k.B[i];
    pr[GRB_P_ZX + i] = w * mu * x * (k.rup[i] + mu * k.rBt * k.Bt[i]);
  }
  return fabs(res);
}

// prims -> densitized cons (c2p.cpp:416-455)
GRB_HD void prims_to_cons(const double pr[13], double c[10], const Met& m) {
  const double W = lorentz(m.g, pr + GRB_P_ZX);
  double b[4], b2;
  comoving_b(m.alp, m.beta, m.g, pr + GRB_P_BX, pr + GRB_P_ZX, W, b, b2);
  const double rhoh = pr[GRB_P_RHO] * (1. + pr[GRB_P_EPS]) + pr[GRB_P_PRESS] + b2;
  const double pstar = pr[GRB_P_PRESS] + 0.5 * b2;
  double bl[3], betal[3], zl[3];
  mvs(m.g, b + 1, bl);
  mvs(m.g, m.beta, betal);
  mvs(m.g, pr + GRB_P_ZX, zl);
  const double D = pr[GRB_P_RHO] * W;
  const double tau = rhoh * W * W - pstar - m.alp * m.alp * b[0] * b[0] - D;
  c[0] = m.sqrtg * D;
#pragma unroll
  for (int i = 0; i < 3; ++i) c[1 + i] = m.sqrtg * (rhoh * W * zl[i] - m.alp * b[0] * (bl[i] + betal[i] * b[0]));
  c[4] = m.sqrtg * tau;
  c[6] = m.sqrtg * (pr[GRB_P_ENT] * D);
  c[5] = c[0] * pr[GRB_P_YE];
}

// Lorentz factor and comoving-field scalars of one set of primitives (tuned
// mode), kept while z and B stay unchanged: z2 = z_i z^i, W = sqrt(1 + z2),
// Bz = B^i z_i, b^2 = (B_i B^i + Bz^2) / W^2 (comoving_b's b^2).
struct WB {
  double z2, W, iW, Bz, b2;
};
GRB_HD WB wb_of(const Met& m, const double pr[13]) {
  WB o;
  double zl[3];
  mvs(m.g, pr + GRB_P_ZX, zl);
  const double* z = pr + GRB_P_ZX;
  const double* B = pr + GRB_P_BX;
  o.z2 = z[0] * zl[0] + z[1] * zl[1] + z[2] * zl[2];
  o.iW = rsqrt(1. + o.z2);  // 1/W; W = (1 + z^2) / W without a square root
  o.W = (1. + o.z2) * o.iW;
  o.Bz = B[0] * zl[0] + B[1] * zl[1] + B[2] * zl[2];
  o.b2 = (sqs(m.g, B) + o.Bz * o.Bz) * o.iW * o.iW;
  return o;
}
// prims_to_cons from a cached WB; with `need` holding no ERR_RESET_STILDE
// or ERR_RESET_TAU bit the momenta and tau (and b^mu) are not formed (D,
// Ye* and the entropy density always are).
GRB_HD void prims_to_cons_wb(const double pr[13], double c[10], const Met& m, const WB& q, double ialp,
                             uint32_t need) {
  const double D = pr[GRB_P_RHO] * q.W;
  c[0] = m.sqrtg * D;
  c[6] = m.sqrtg * (pr[GRB_P_ENT] * D);
  c[5] = c[0] * pr[GRB_P_YE];
  if (need & (ERR_RESET_STILDE | ERR_RESET_TAU)) {
    const double b0 = q.Bz * ialp;
    double b[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
      b[i] = (pr[GRB_P_BX + i] + m.alp * b0 * (pr[GRB_P_ZX + i] - q.W * m.beta[i] * ialp)) * q.iW;
    const double rhoh = pr[GRB_P_RHO] * (1. + pr[GRB_P_EPS]) + pr[GRB_P_PRESS] + q.b2;
    const double pstar = pr[GRB_P_PRESS] + 0.5 * q.b2;
    double bl[3], betal[3], zl[3];
    mvs(m.g, b, bl);
    mvs(m.g, m.beta, betal);
    mvs(m.g, pr + GRB_P_ZX, zl);
    const double tau = rhoh * q.W * q.W - pstar - m.alp * m.alp * b0 * b0 - D;
#pragma unroll
    for (int i = 0; i < 3; ++i) c[1 + i] = m.sqrtg * (rhoh * q.W * zl[i] - m.alp * b0 * (bl[i] + betal[i] * b0));
    c[4] = m.sqrtg * tau;
  }
}

GRB_HD void handle_sig(uint32_t sig, bool lenient, uint32_t& err, uint32_t& fatal) {
  if (sig & SIG_RHO_HIGH) {
    err |= ERR_SIG_RHO_HIGH | ERR_ALL_RESETS;
    if (!lenient) fatal |= FAT_C2P_RHO_HIGH;
  }
  if (sig & SIG_RHO_LOW)
    err |= ERR_RESET_DENS | ERR_RESET_TAU | ERR_RESET_STILDE | ERR_RESET_ENTROPY | ERR_SIG_RHO_LOW;
  if (sig & SIG_ENT_LOW) err |= ERR_RESET_ENTROPY | ERR_SIG_ENT_LOW;
  if (sig & SIG_ENT_HIGH) err |= ERR_RESET_ENTROPY | ERR_SIG_ENT_HIGH;
  if (sig & SIG_EPS_HIGH) err |= ERR_RESET_STILDE | ERR_RESET_TAU | ERR_SIG_EPS_HIGH;
  if (sig & SIG_EPS_LOW) err |= ERR_RESET_STILDE | ERR_RESET_TAU | ERR_SIG_EPS_LOW;
  if (sig & SIG_VEL_HIGH)
    err |= ERR_RESET_DENS | ERR_RESET_TAU | ERR_RESET_STILDE | ERR_RESET_ENTROPY | ERR_SIG_VEL_HIGH;
  if (sig & SIG_SIGMA_HIGH)
    err |= ERR_RESET_DENS | ERR_RESET_TAU | ERR_RESET_STILDE | ERR_RESET_ENTROPY | ERR_SIG_SIGMA_HIGH;
}
GRB_HD void handle_eos_sig(uint32_t q, bool lenient, uint32_t& err, uint32_t& fatal) {
  if (q & EOS_RHO_HIGH) { err |= ERR_SIG_RHO_HIGH; fatal |= FAT_EOS_RHO_HIGH; }
  if (q & EOS_RHO_LOW)
    err |= ERR_RESET_DENS | ERR_RESET_TAU | ERR_RESET_STILDE | ERR_RESET_ENTROPY | ERR_SIG_RHO_LOW;
  if (q & EOS_ENT_HIGH) err |= ERR_RESET_ENTROPY | ERR_SIG_ENT_HIGH;
  if (q & EOS_ENT_LOW) err |= ERR_RESET_ENTROPY | ERR_SIG_ENT_LOW;
  if (q & EOS_EPS_HIGH) { err |= ERR_SIG_EPS_HIGH | ERR_RESET_STILDE | ERR_RESET_TAU; if (!lenient) fatal |= FAT_EOS_EPS_HIGH; }
  if (q & EOS_EPS_LOW) err |= ERR_RESET_STILDE | ERR_RESET_TAU | ERR_SIG_EPS_LOW;
  if (q & EOS_TEMP_HIGH) { err |= ERR_SIG_TEMP_HIGH | ERR_RESET_STILDE | ERR_RESET_TAU; if (!lenient) fatal |= FAT_EOS_TEMP_HIGH; }
  if (q & EOS_TEMP_LOW) err |= ERR_RESET_STILDE | ERR_RESET_TAU | ERR_SIG_TEMP_LOW;
  if (q & EOS_PRESS_HIGH) { err |= ERR_SIG_PRESS_HIGH | ERR_RESET_STILDE | ERR_RESET_TAU; if (!lenient) fatal |= FAT_EOS_PRESS_HIGH; }
  if (q & EOS_PRESS_LOW) err |= ERR_RESET_STILDE | ERR_RESET_TAU | ERR_SIG_PRESS_LOW;
}

GRB_HD void reset_atmo(double c[10], double pr[13], const Met& m, const DevParams& P,
                       uint32_t& err) {
  pr[GRB_P_RHO] = P.rho_fl;
  pr[GRB_P_YE] = P.ye_fl;
  pr[GRB_P_TEMP] = P.temp_fl;
  pr[GRB_P_ZX] = pr[GRB_P_ZY] = pr[GRB_P_ZZ] = 0.;
  double cs2;
  uint32_t q = 0;
  pr[GRB_P_PRESS] = eos_PT(P.eos, pr[GRB_P_EPS], cs2, &pr[GRB_P_ENT], pr[GRB_P_TEMP], pr[GRB_P_RHO], q);
  prims_to_cons(pr, c, m);
  err |= ERR_ALL_RESETS | ERR_ATMO;
}

struct C2POut {
  uint32_t err;
  uint32_t fatal;
  int iters;
  bool floored;
  bool guess_used;
  double mu;  // Kastaun root, 0 where the Kastaun solve did not run
  double W, iW;  // Lorentz factor of the final primitives (tuned mode)
};

// conservs_to_prims (c2p.cpp:188-414), in three parts so that a batch can
// defer the entropy backup of the states that need it to a second pass
// (c2p_front: up to the decision to distrust the Kastaun result;
// c2p_backup: the entropy-based solve; c2p_back: signals, atmosphere,
// temperature floor, limit_primitives, prims_to_cons).  c2p() runs the three
// in sequence: the reference's order of operations.  c: densitized cons
// with densitized cell-centred B (in), re-densitized consistent cons (out).
// FAST (tuned mode): multiplications by 1/sqrt(gamma) and 1/D where the
// reference divides repeatedly by the same value, the FAST master function,
// and W, b^mu, b^2 formed once per set of primitives (WB) instead of in
// each of the beta test, limit_primitives and prims_to_cons; equal to the
// reference's operations up to rounding.  kAllCons false (tuned mode):
// the returned cons hold only what the reset flags in o.err ask for.
struct C2PState {
  C2POut o;
  uint32_t ret;
  bool failed, lenient, ran, backup, done;
  WB wb;
  bool wb_ok;  // wb belongs to the current z and B
};

template <bool FAST = false>
GRB_HD C2PState c2p_front(double c[10], double pr[13], const Met& m, const DevParams& P, bool dry_run,
                          double alp_bh_thresh, const Guess& gs) {
  C2PState F{};
  F.o = C2POut{0u, 0u, 0, false, false, 0.0, 0.0, 0.0};
  F.wb_ok = false;
  F.failed = false;
  F.ret = 0;
  const DevEos& e = P.eos;
  C2POut& o = F.o;
  o.err = ERR_RESET_ENTROPY;
  const double isg = FAST ? 1.0 / m.sqrtg : 0.0;
#pragma unroll
  for (int v = 0; v < 10; ++v) c[v] = FAST ? c[v] * isg : c[v] / m.sqrtg;
  pr[GRB_P_BX] = c[7]; pr[GRB_P_BY] = c[8]; pr[GRB_P_BZ] = c[9];
  if (c[0] < 0) {
    reset_atmo(c, pr, m, P, o.err);
    o.floored = true;
    F.done = true;
    return F;
  }
  const double iD0 = FAST ? 1.0 / c[0] : 0.0;
  pr[GRB_P_YE] = FAST ? c[5] * iD0 : c[5] / c[0];
  if (pr[GRB_P_YE] > e.yemax) { pr[GRB_P_YE] = e.yemax; o.err |= ERR_RESET_YE; }
  if (pr[GRB_P_YE] < 0.0) { pr[GRB_P_YE] = 0.0; o.err |= ERR_RESET_YE; }
  F.lenient = m.alp < alp_bh_thresh;
  {  // limit_conservatives (c2p.cpp:117-157)
    double lo, hi;
    eos_eps_range(e, lo, hi, c[0]);
    const double B2 = sqs(m.g, c + 7);
    if ((FAST ? c[4] * iD0 - 0.5 * B2 * iD0 : c[4] / c[0] - 0.5 * B2 / c[0]) < fmin(0.0, lo)) {
      c[4] = lo * c[0] + 0.5 * B2;
      o.err |= ERR_RESET_TAU;
      o.floored = true;
    }
    const double qd = (FAST ? c[4] * iD0 : c[4] / c[0]) + 1;
    const double st2 = FAST ? sqs(m.gi, c + 1) * (iD0 * iD0) : sqs(m.gi, c + 1) / (c[0] * c[0]);
    if (st2 > qd * qd) {
      const double f = sqrt(qd * qd / st2);
      c[1] *= f; c[2] *= f; c[3] *= f;
      o.err |= ERR_RESET_STILDE;
      o.floored = true;
    }
  }
  if (o.floored && dry_run) {
    F.done = true;
    return F;
  }
  if (c[0] >= P.rho_fl * (1 + P.atmo_tol)) {
    F.ran = true;
    Guess g2 = gs;
    if (o.floored) g2.has_mu0 = false;  // limit_conservatives changed the state
    const double res = kastaun_invert<FAST>(e, m, c, pr, F.ret, o.iters, g2, o.guess_used, o.mu);
    F.failed = (fabs(res) > P.tol) || (F.ret & SIG_RHO_HIGH) || (F.ret & SIG_EPS_HIGH) || !isfinite(res);
    if (dry_run) return F;  // no backup in a dry run: beta is not needed
    double beta;
    if (FAST) {
      F.wb = wb_of(m, pr);
      F.wb_ok = true;
      beta = 2.0 * pr[GRB_P_PRESS] / fmax(F.wb.b2, 1e-50);
    } else {
      const double W = lorentz(m.g, pr + GRB_P_ZX);
      double b[4], b2;
      comoving_b(m.alp, m.beta, m.g, pr + GRB_P_BX, pr + GRB_P_ZX, W, b, b2);
      beta = 2.0 * pr[GRB_P_PRESS] / fmax(b2, 1e-50);
    }
    const bool distrust = F.failed || (F.ret & SIG_EPS_LOW) || (beta <= P.beta_fallback);
    F.backup = distrust && P.use_ent_backup && !dry_run;
  } else {
    F.failed = true;
  }
  return F;
}

// The entropy-based backup of a distrusted Kastaun result (c2p.cpp:262-290).
GRB_HD void c2p_backup(C2PState& F, double c[10], double pr[13], const Met& m, const DevParams& P) {
  double save[13];
#pragma unroll
  for (int v = 0; v < 13; ++v) save[v] = pr[v];
  uint32_t bret = 0;
  const double rb = entropy_invert(P.eos, m, c, pr, bret);
  const bool ok = (fabs(rb) <= P.tol) && isfinite(rb) && (pr[GRB_P_EPS] < P.eos.eps_max);
  if (ok) {
    F.ret = bret;
    F.failed = false;
    F.o.err |= ERR_ENT_BACKUP;
    F.wb_ok = false;
  } else if (!F.failed) {
#pragma unroll
    for (int v = 0; v < 13; ++v) pr[v] = save[v];
  } else {
    F.wb_ok = false;
  }
}

// kDry: a dry run (the FOFC flag's), which needs only o.floored: the final
// prims_to_cons is skipped.
template <bool FAST = false, bool kAllCons = true, bool kDry = false>
GRB_HD void c2p_back(C2PState& F, double c[10], double pr[13], const Met& m, const DevParams& P, double r_sph) {
  const DevEos& e = P.eos;
  C2POut& o = F.o;
  WB& wb = F.wb;
  const double ialp = FAST ? 1.0 / m.alp : 0.0;
  if (F.ran) {
    const uint32_t ret = F.ret;
    if (ret & (SIG_EPS_HIGH | SIG_RHO_LOW | SIG_RHO_HIGH | SIG_VEL_HIGH)) o.floored = true;
    if (e.kind == GRB_EOS_IDEAL_GAS && (ret & SIG_EPS_LOW)) o.floored = true;
    handle_sig(ret, F.lenient, o.err, o.fatal);
  }
  const bool excise = P.excise_by_radius ? (r_sph <= P.r_ex) : (m.alp <= P.alp_ex);
  if (F.failed || excise || pr[GRB_P_RHO] < (1. + P.atmo_tol) * P.rho_fl) {
    reset_atmo(c, pr, m, P, o.err);
    o.floored = true;
    F.wb_ok = false;
  } else if (pr[GRB_P_TEMP] < P.temp_fl) {
    pr[GRB_P_TEMP] = P.temp_fl;
    double cs2;
    uint32_t q = 0;
    pr[GRB_P_PRESS] = eos_PT(e, pr[GRB_P_EPS], cs2, &pr[GRB_P_ENT], pr[GRB_P_TEMP], pr[GRB_P_RHO], q);
    handle_eos_sig(q, F.lenient, o.err, o.fatal);
    o.err |= ERR_RESET_TAU | ERR_RESET_STILDE | ERR_RESET_ENTROPY | ERR_T_FLOORED;
    if (e.kind == GRB_EOS_IDEAL_GAS) o.floored = true;
  } else {  // limit_primitives (c2p.cpp:63-115)
    uint32_t s2 = 0;
    const double z2max = P.max_w * P.max_w - 1.;
    if (FAST && !F.wb_ok) { wb = wb_of(m, pr); F.wb_ok = true; }
    const double z2 = FAST ? wb.z2 : sqs(m.g, pr + GRB_P_ZX);
    if (z2 >= z2max) {
      const double zn = 0.99 * sqrt(z2max / z2);
      pr[GRB_P_ZX] *= zn; pr[GRB_P_ZY] *= zn; pr[GRB_P_ZZ] *= zn;
      s2 |= SIG_VEL_HIGH;
      if (FAST) wb = wb_of(m, pr);
    }
    double b2;
    if (FAST) {
      b2 = wb.b2;
    } else {
      const double W = lorentz(m.g, pr + GRB_P_ZX);
      double b[4];
      comoving_b(m.alp, m.beta, m.g, pr + GRB_P_BX, pr + GRB_P_ZX, W, b, b2);
    }
    const double sigma = b2 / pr[GRB_P_RHO];
    if (sigma >= P.max_sigma) {
      pr[GRB_P_RHO] *= 1.001 * sigma / P.max_sigma;
      double cs2;
      uint32_t q = 0;
      pr[GRB_P_PRESS] = eos_PT(e, pr[GRB_P_EPS], cs2, &pr[GRB_P_ENT], pr[GRB_P_TEMP], pr[GRB_P_RHO], q);
      s2 |= SIG_SIGMA_HIGH;
    }
    handle_sig(s2, F.lenient, o.err, o.fatal);
    if (s2 & (SIG_VEL_HIGH | SIG_SIGMA_HIGH)) o.floored = true;
  }
  if (kDry) return;
  if (FAST) {
    if (!F.wb_ok) wb = wb_of(m, pr);
    prims_to_cons_wb(pr, c, m, wb, ialp, kAllCons ? ~0u : o.err);
    o.W = wb.W;
    o.iW = wb.iW;
  } else {
    prims_to_cons(pr, c, m);
  }
}

template <bool FAST = false, bool kAllCons = true>
GRB_HD C2POut c2p(double c[10], double pr[13], const Met& m, const DevParams& P, double r_sph,
                  bool dry_run, double alp_bh_thresh, const Guess& gs) {
  C2PState F = c2p_front<FAST>(c, pr, m, P, dry_run, alp_bh_thresh, gs);
  if (F.done) return F.o;
  if (F.backup) c2p_backup(F, c, pr, m, P);
  c2p_back<FAST, kAllCons>(F, c, pr, m, P, r_sph);
  return F.o;
}
// The FOFC flag's dry run (c2p.cpp:188-414 with the dry-run flag): whether
// the state would be floored; no entropy backup, no final prims_to_cons.
template <bool FAST = false>
GRB_HD bool c2p_floored(double c[10], double pr[13], const Met& m, const DevParams& P, double r_sph) {
  C2PState F = c2p_front<FAST>(c, pr, m, P, true, 1e30, no_guess());
  if (F.done) return F.o.floored;
  c2p_back<FAST, true, true>(F, c, pr, m, P, r_sph);
  return F.o.floored;
}

}  // namespace grb
