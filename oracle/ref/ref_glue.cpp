// Pinning build — test infrastructure only.  Compiled (with the shim headers
// in oracle/ref/shim) against the GRACE sources where they lie, together
// with GRACE's src/physics/eos/c2p.cpp, into oracle/_ref/libgrace_ref.so.
// It binds the reference's OWN per-cell numerics (SymPy kernels, WENO-Z /
// slope-limited reconstruction, HLLE, EOS classes, conservs_to_prims,
// Gardiner-Stone edge EMF, 4-point face interpolation, 6th-order
// derivatives) to the shared loop drivers of stage_driver.hpp and exports
// them with the ref_ prefix.  Tests compare the oracle (orc_) against it.
#include <grace_config.h>

#include <grace/physics/grmhd_subexpressions.hh>
#include <grace/physics/fd_subexpressions.hh>
#include <grace/physics/eos/c2p.hh>
#include <grace/physics/grmhd_helpers.hh>
#include <grace/utils/reconstruction.hh>
#include <grace/utils/weno_reconstruction.hh>
#include <grace/utils/riemann_solvers.hh>

#include "stage_driver.hpp"

namespace refglue {

using hyb_t = grace::hybrid_eos_t<grace::piecewise_polytropic_eos_t>;
using ideal_t = grace::ideal_gas_eos_t;

struct Eos {
  int kind = 0;
  ideal_t ideal;
  hyb_t hyb;
};

// 1-D stencil adapter: u(i,j,k) over a short array, with the stencil along i.
struct Line {
  const double* v;
  int base;
  double operator()(int i, int, int) const { return v[i - base]; }
};
// 5-index adapter for face_interp_4: view(i,j,k,ivar,q)
struct Line5 {
  const double* v;
  int base;
  double operator()(int i, int, int, int, int) const { return v[i - base]; }
};

template <class St>
struct EfaceV {
  St* s;
  double operator()(int i, int j, int k, int c, int dir, int q) const { return s->EF(i, j, k, c, dir, q); }
};
template <class St>
struct EcV {
  St* s;
  double operator()(int i, int j, int k, int c, int q) const { return s->EC(i, j, k, c, q); }
};
template <class St>
struct FluxV {
  St* s;
  double operator()(int i, int j, int k, int v, int dir, int q) const { return s->F(i, j, k, v, dir, q); }
};

struct RefNumerics {
  using Eos = refglue::Eos;
  static Eos make_eos(const grb_eos_params& p) {
    Eos e;
    e.kind = p.kind;
    if (p.kind == GRB_EOS_IDEAL_GAS) {
      grace::shim_param_table()["eos.ideal_gas_eos.gamma"] = p.gamma;
      grace::shim_param_table()["eos.ideal_gas_eos.kappa_id"] = 0.0;
      e.ideal = ideal_t(p.temp_atm, p.eps_max);
    } else {
      using V = Kokkos::View<double[grace::piecewise_polytropic_eos_t::max_n_pieces], grace::default_space>;
      V k, g, r, ep, pr;
      for (int i = 0; i < GRB_MAX_PIECES; ++i) {
        k(i) = p.pw_kappa[i]; g(i) = p.pw_gamma[i]; r(i) = p.pw_rho[i];
        ep(i) = p.pw_eps[i]; pr(i) = p.pw_press[i];
      }
      grace::piecewise_polytropic_eos_t cold(k, g, r, ep, pr, p.n_pieces, 1e+10, 1e-100);
      e.hyb = hyb_t(cold, p.gamma_th - 1., p.entropy_min, 1. + 1e-10, 1, p.eps_max, p.temp_atm);
    }
    return e;
  }
  static grace::metric_array_t gm(const double g[6], const double b[3], double alp) {
    return grace::metric_array_t({g[0], g[1], g[2], g[3], g[4], g[5]}, {b[0], b[1], b[2]}, alp);
  }
  static orc::Metric metric(const double g[6], const double b[3], double alp) {
    const auto m = gm(g, b, alp);
    orc::Metric o;
    for (int a = 0; a < 6; ++a) { o.g[a] = m._g[a]; o.ginv[a] = m._ginv[a]; }
    for (int a = 0; a < 3; ++a) o.beta[a] = m._beta[a];
    o.alp = m._alp;
    o.sqrtg = m._sqrtg;
    return o;
  }
  static void recon(int kind, const double u[6], double& L, double& R) {
    Line v{u, 0};
    if (kind == GRB_RECON_WENOZ) { grace::weno_reconstructor_t<5> r; r(v, 3, 0, 0, L, R, 0); }
    else if (kind == GRB_RECON_MC2) { grace::slope_limited_reconstructor_t<grace::MCbeta> r; r(v, 3, 0, 0, L, R, 0); }
    else if (kind == GRB_RECON_MINMOD) { grace::slope_limited_reconstructor_t<grace::minmod> r; r(v, 3, 0, 0, L, R, 0); }
    else { grace::donor_cell_reconstructor_t r; r(v, 3, 0, 0, L, R, 0); }
  }
  static double face_interp4(double a, double b, double c, double d) {
    const double v[4] = {a, b, c, d};
    Line5 w{v, 0};
    return grace::face_interp_4(w, 2, 0, 0, 0, 0, 0);
  }
  static double fd6(double m3, double m2, double m1, double p1, double p2, double p3, double h) {
    const double v[7] = {m3, m2, m1, 0.0, p1, p2, p3};
    Line w{v, 0};
    double du;
    fd_der_x<6>(w, 3, 0, 0, h, &du);
    return du;
  }
  static double press_eps_csnd2__temp_rho(const Eos& e, double& eps, double& cs2, double& t, double& r) {
    grace::eos_err_t err;
    double ye = 0.0;
    if (e.kind == GRB_EOS_IDEAL_GAS) return e.ideal.press_eps_csnd2__temp_rho_ye(eps, cs2, t, r, ye, err);
    return e.hyb.press_eps_csnd2__temp_rho_ye(eps, cs2, t, r, ye, err);
  }
  static double press_h_csnd2__temp_rho(const Eos& e, double& h, double& cs2, double& t, double& r) {
    grace::eos_err_t err;
    double ye = 0.0;
    if (e.kind == GRB_EOS_IDEAL_GAS) return e.ideal.press_h_csnd2__temp_rho_ye(h, cs2, t, r, ye, err);
    return e.hyb.press_h_csnd2__temp_rho_ye(h, cs2, t, r, ye, err);
  }
  static double lorentz(const double g[6], const double z[3]) {
    double W;
    grmhd_get_W(g, z, &W);
    return W;
  }
  static void comoving_b(double alp, const double* beta, const double* g, const double* B,
                         const double* z, double W, double b[4], double& b2) {
    double bb[4];
    grmhd_get_smallbu_smallb2(alp, beta, g, B, z, W, &bb, &b2);
    for (int i = 0; i < 4; ++i) b[i] = bb[i];
  }
  static void vtilde(double alp, const double* beta, const double* z, double W, double vt[3]) {
    double v[3];
    grmhd_get_vtildeu(alp, beta, z, W, &v);
    for (int i = 0; i < 3; ++i) vt[i] = v[i];
  }
  static void char_speeds(double alp, const double* beta, double rho, double p, double eps,
                          double cs2, double W, double b2, const double* vt, double guu, int d,
                          double& cm, double& cp) {
    grmhd_get_cm_cp(alp, beta, rho, p, eps, cs2, W, b2, vt, guu, d, &cm, &cp);
  }
  static void cons_and_flux(double alp, const double* beta, const double* g, double rho, double p,
                            double eps, const double* z, double s, double W, double b2,
                            const double* b, const double* vt, int d, double& D, double& tau,
                            double S[3], double& ents, double& fD, double& ft, double fS[3],
                            double& fe) {
    double st[3], fst[3];
    grmhd_get_fluxes(alp, beta, g, rho, p, eps, z, s, W, b2, b, vt, d, &D, &tau, &st, &ents, &fD,
                     &ft, &fst, &fe);
    for (int i = 0; i < 3; ++i) { S[i] = st[i]; fS[i] = fst[i]; }
  }
  static void geom_sources(double alp, const double* beta, const double* g, const double* guu,
                           const double* K, const double* dalp, const double* dg, const double* db,
                           double rho, double p, double eps, const double* B, const double* z,
                           double W, double& st, double sS[3]) {
    double s3[3];
    grmhd_get_geom_sources(alp, beta, g, guu, K, dalp, dg, db, rho, p, eps, B, z, W, &st, &s3);
    for (int i = 0; i < 3; ++i) sS[i] = s3[i];
  }
  static double hll(double fL, double fR, double uL, double uR, double cmin, double cmax) {
    grace::hll_riemann_solver_t s;
    return s(fL, fR, uL, uR, cmin, cmax);
  }
  static void prims_to_conservs(const double pr[13], double c[10], const orc::Metric& m) {
    grace::grmhd_prims_array_t p;
    grace::grmhd_cons_array_t cc{};
    for (int v = 0; v < 13; ++v) p[v] = pr[v];
    grace::prims_to_conservs(p, cc, gm(m.g, m.beta, m.alp));
    for (int v = 0; v < 10; ++v) c[v] = cc[v];
  }
  static bool c2p_counted(double cons[10], double pr[13], const orc::Metric& m, const Eos& e,
                          const grb_params& P, double r, uint32_t& err, bool dry, int& fatal,
                          double alp_bh_override, int* iters) {
    atmo_params_t atmo{P.ye_fl, P.rho_fl, P.temp_fl, 0.0, 0.0, P.atmo_tol};
    excision_params_t ex{P.rho_ex, P.temp_ex, P.ye_ex, P.r_ex, P.alp_ex, P.excise_by_radius != 0};
    c2p_params_t cp{P.c2p_tol, P.max_w, P.max_sigma, P.beta_fallback, P.use_ent_backup != 0,
                    alp_bh_override > 0 ? alp_bh_override : P.alp_bh_thresh};
    grace::grmhd_cons_array_t c;
    grace::grmhd_prims_array_t p{};
    for (int v = 0; v < 10; ++v) c[v] = cons[v];
    grace::c2p_err_t ce;
    double rtp[3] = {r, 0.0, 0.0};
    bool fl = false;
    try {
      if (e.kind == GRB_EOS_IDEAL_GAS)
        fl = grace::conservs_to_prims<ideal_t>(c, p, gm(m.g, m.beta, m.alp), e.ideal, atmo, ex, cp, rtp, ce, dry);
      else
        fl = grace::conservs_to_prims<hyb_t>(c, p, gm(m.g, m.beta, m.alp), e.hyb, atmo, ex, cp, rtp, ce, dry);
    } catch (...) {
      fatal |= 1 << 30;  // the reference aborted here
    }
    for (int v = 0; v < 10; ++v) cons[v] = c[v];
    for (int v = 0; v < 13; ++v) pr[v] = p[v];
    err = (uint32_t)ce.words[0];
    if (iters) *iters = 0;
    return fl;
  }
  static bool c2p(double cons[10], double pr[13], const orc::Metric& m, const Eos& e,
                  const grb_params& P, double r, uint32_t& err, bool dry, int& fatal,
                  double alp_bh_override) {
    return c2p_counted(cons, pr, m, e, P, r, err, dry, fatal, alp_bh_override, nullptr);
  }
  template <class St>
  static double gs_edge(St& s, int dir, int i, int j, int k, int64_t q) {
    EfaceV<St> ef{&s};
    EcV<St> ec{&s};
    FluxV<St> fl{&s};
    if (dir == 0) return grace::gs_edge_emf_x(ef, ec, fl, i, j, k, (int)q);
    if (dir == 1) return grace::gs_edge_emf_y(ef, ec, fl, i, j, k, (int)q);
    return grace::gs_edge_emf_z(ef, ec, fl, i, j, k, (int)q);
  }
};

}  // namespace refglue

#define NUMERICS refglue::RefNumerics
#define API(name) ref_##name
#include "api_impl.hpp"

// FMR restriction: the reference's own per-point operators
// (include/grace/amr/ghostzone_kernels/pr_helpers.hh:187-322, with the
// coefficient table of pr_ho_coeffs.hh), driven by the restated loops of
// amr_oracle.hpp.
#include <grace/amr/ghostzone_kernels/pr_helpers.hh>
#include <grace/amr/ghostzone_kernels/pr_ho_coeffs.hh>
#include "amr_oracle.hpp"
namespace {
struct RefOps {
  std::vector<double> coeffs;
  int n, ngz;
  RefOps(int n_, int g_) : n(n_), ngz(g_) { grace::detail::fill_fifth_order_restriction_coefficients(coeffs); }
  double lo(const orc_amr::Acc& u, int i, int j, int k) const { return grace::second_order_restrict_op{}(u, i, j, k); }
  double hi(const orc_amr::Acc& u, int, int, int i, int j, int k, int hx, int hy, int hz) const {
    Kokkos::View<double*, grace::default_space> cv(const_cast<double*>(coeffs.data()));
    grace::lagrange_restrict_op<4> op(cv, n, n, n, ngz);
    return op(u, i, j, k, hx, hy, hz);
  }
};
}  // namespace
extern "C" void ref_restrict_cells(int n, int ngz, int nvars, const double* src, double* dst, int64_t nquads,
                                   const int64_t* src_q, const int64_t* dst_q, const uint8_t* child,
                                   const int* vlo, int nlo, const int* vhi, int nhi) {
  orc_amr::restrict_cells(RefOps(n, ngz), n, ngz, nvars, src, dst, nquads, src_q, dst_q, child, vlo, nlo, vhi,
                          nhi);
}

// FMR prolongation into ghost zones: the reference's own functors
// (prolong_op and div_free_prolong_op of
// include/grace/amr/ghostzone_kernels/prolongation_kernels.hh, with their
// index_transformer_t and the operators slope_limited_prolong_op<minmod>,
// lagrange_prolong_op<4> of pr_helpers.hh), each called over the iteration
// range its task factory gives it (prolongation_task_factories.hh:150-230),
// serially.
#include <grace/amr/ghostzone_kernels/prolongation_kernels.hh>
namespace {
// LayoutLeft (N0, N1, N2, nv, nq) array of doubles, in the view shape the
// functors index.
struct Acc3 {
  double* a;
  size_t N0, N1;
  double& operator()(size_t i, size_t j, size_t k) const { return a[(k * N1 + j) * N0 + i]; }
};
struct Acc4 {
  double* a;
  size_t N0, N1, N2, nv;
  double& operator()(size_t i, size_t j, size_t k, size_t v) const { return a[((v * N2 + k) * N1 + j) * N0 + i]; }
  size_t extent(int) const { return nv; }
};
struct Arr5 {
  double* a;
  size_t N0, N1, N2, nv;
  double& operator()(size_t i, size_t j, size_t k, size_t v, size_t q) const {
    return a[(((q * nv + v) * N2 + k) * N1 + j) * N0 + i];
  }
  Acc3 sub(int iv, int q) const { return Acc3{a + ((size_t)q * nv + iv) * N0 * N1 * N2, N0, N1}; }
  Acc4 sub4(size_t q) const { return Acc4{a + q * nv * N0 * N1 * N2, N0, N1, N2, nv}; }
};
template <grace::amr::element_kind_t K>
void ref_prolong_cells_k(int n, int ngz, int nvars, double* fine, const double* cbuf, int64_t nelems,
                         const int64_t* fine_q, const int64_t* cbuf_q, const uint8_t* elem, const int* vlo, int nlo,
                         const int* vhi, int nhi) {
  const size_t N = n + 2 * ngz;
  std::vector<size_t> q(fine_q, fine_q + nelems), c(cbuf_q, cbuf_q + nelems);
  std::vector<uint8_t> e(elem, elem + nelems);
  std::vector<size_t> lo(vlo, vlo + nlo), hi(vhi, vhi + nhi);
  std::vector<double> co;
  grace::detail::fill_fifth_order_prolongation_coefficients(co);
  Arr5 F{fine, N, N, N, (size_t)nvars}, C{const_cast<double*>(cbuf), N, N, N, (size_t)nvars};
  Kokkos::View<size_t*> Q(q.data()), Cq(c.data()), L(lo.data()), H(hi.data());
  Kokkos::View<uint8_t*> E(e.data());
  grace::amr::prolong_op<grace::slope_limited_prolong_op<grace::minmod>, K, Arr5> f_lo(F, C, Q, Cq, E, L, {}, n, ngz);
  grace::lagrange_prolong_op<4> ho{Kokkos::View<double*, grace::default_space>(co.data())};
  grace::amr::prolong_op<grace::lagrange_prolong_op<4>, K, Arr5> f_hi(F, C, Q, Cq, E, H, ho, n, ngz);
  for (int pass = 0; pass < 2; ++pass) {
    const auto r = grace::amr::get_iter_range<K>(ngz, n, pass == 0 ? nlo : nhi, nelems);
    for (int64_t iq = 0; iq < r[4]; ++iq)
      for (int64_t v = 0; v < r[3]; ++v)
        for (int64_t k = 0; k < r[2]; ++k)
          for (int64_t j = 0; j < r[1]; ++j)
            for (int64_t i = 0; i < r[0]; ++i) {
              if (pass == 0) f_lo(i, j, k, v, iq);
              else f_hi(i, j, k, v, iq);
            }
  }
}
template <grace::amr::element_kind_t K>
void ref_prolong_faces_k(int n, int ngz, double* fx, double* fy, double* fz, const double* cx, const double* cy,
                         const double* cz, int64_t nelems, const int64_t* fine_q, const int64_t* cbuf_q,
                         const uint8_t* elem, const int8_t* have_fine) {
  const size_t N = n + 2 * ngz;
  std::vector<size_t> q(fine_q, fine_q + nelems), c(cbuf_q, cbuf_q + nelems);
  std::vector<uint8_t> e(elem, elem + nelems);
  // have_fine_data(axis, side, element) from have_fine[element][axis][side]
  std::vector<int8_t> hf(6 * nelems);
  for (int64_t i = 0; i < nelems; ++i)
    for (int a = 0; a < 3; ++a)
      for (int sd = 0; sd < 2; ++sd) hf[a + 3 * (sd + 2 * i)] = have_fine[6 * i + 2 * a + sd];
  Arr5 X{fx, N + 1, N, N, 1}, Y{fy, N, N + 1, N, 1}, Z{fz, N, N, N + 1, 1};
  Arr5 CX{const_cast<double*>(cx), N + 1, N, N, 1}, CY{const_cast<double*>(cy), N, N + 1, N, 1},
      CZ{const_cast<double*>(cz), N, N, N + 1, 1};
  Kokkos::View<size_t*> Q(q.data()), Cq(c.data());
  Kokkos::View<uint8_t*> E(e.data());
  Kokkos::View<int8_t***> HF(hf.data(), 3, 2);
  grace::amr::div_free_prolong_op<K, Arr5> op(X, Y, Z, CX, CY, CZ, Q, Cq, E, HF, n, ngz);
  for (int64_t iq = 0; iq < nelems; ++iq) op(Kokkos::SerialTeam{(int)iq});
}
}  // namespace
extern "C" void ref_prolong_cells(int kind, int n, int ngz, int nvars, double* fine, const double* cbuf,
                                  int64_t nelems, const int64_t* fine_q, const int64_t* cbuf_q, const uint8_t* elem,
                                  const int* vlo, int nlo, const int* vhi, int nhi) {
  using namespace grace::amr;
  if (kind == 0) ref_prolong_cells_k<FACE>(n, ngz, nvars, fine, cbuf, nelems, fine_q, cbuf_q, elem, vlo, nlo, vhi, nhi);
  if (kind == 1) ref_prolong_cells_k<EDGE>(n, ngz, nvars, fine, cbuf, nelems, fine_q, cbuf_q, elem, vlo, nlo, vhi, nhi);
  if (kind == 2)
    ref_prolong_cells_k<CORNER>(n, ngz, nvars, fine, cbuf, nelems, fine_q, cbuf_q, elem, vlo, nlo, vhi, nhi);
}
extern "C" void ref_prolong_faces(int kind, int n, int ngz, double* fx, double* fy, double* fz, const double* cx,
                                  const double* cy, const double* cz, int64_t nelems, const int64_t* fine_q,
                                  const int64_t* cbuf_q, const uint8_t* elem, const int8_t* have_fine) {
  using namespace grace::amr;
  if (kind == 0) ref_prolong_faces_k<FACE>(n, ngz, fx, fy, fz, cx, cy, cz, nelems, fine_q, cbuf_q, elem, have_fine);
  if (kind == 1) ref_prolong_faces_k<EDGE>(n, ngz, fx, fy, fz, cx, cy, cz, nelems, fine_q, cbuf_q, elem, have_fine);
  if (kind == 2)
    ref_prolong_faces_k<CORNER>(n, ngz, fx, fy, fz, cx, cy, cz, nelems, fine_q, cbuf_q, elem, have_fine);
}
