// CPU oracle — test infrastructure only.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load liboracle.so; the CUDA library never
// does.  This translation unit binds the restated numerics
// (grmhd_numerics.hpp, c2p_oracle.hpp) to the shared loop drivers
// (stage_driver.hpp) and exports them with the orc_ prefix.
#include "c2p_oracle.hpp"
#include "stage_driver.hpp"

namespace orc {
struct OracleNumerics {
  using Eos = orc::Eos;
  static Eos make_eos(const grb_eos_params& p) { return orc::make_eos(p); }
  static Metric metric(const double g[6], const double b[3], double alp) { return make_metric(g, b, alp); }
  static void recon(int kind, const double u[6], double& L, double& R) { orc::recon(kind, u, L, R); }
  static double face_interp4(double a, double b, double c, double d) { return orc::face_interp4(a, b, c, d); }
  static double fd6(double m3, double m2, double m1, double p1, double p2, double p3, double h) {
    return orc::fd6(m3, m2, m1, p1, p2, p3, h);
  }
  static double press_eps_csnd2__temp_rho(const Eos& e, double& eps, double& cs2, double& t, double& r) {
    uint32_t err = 0;
    return orc::press_eps_csnd2__temp_rho(e, eps, cs2, t, r, err);
  }
  static double press_h_csnd2__temp_rho(const Eos& e, double& h, double& cs2, double& t, double& r) {
    uint32_t err = 0;
    return orc::press_h_csnd2__temp_rho(e, h, cs2, t, r, err);
  }
  static double lorentz(const double g[6], const double z[3]) { return orc::lorentz(g, z); }
  static void comoving_b(double alp, const double* beta, const double* g, const double* B,
                         const double* z, double W, double b[4], double& b2) {
    orc::comoving_b(alp, beta, g, B, z, W, b, b2);
  }
  static void vtilde(double alp, const double* beta, const double* z, double W, double vt[3]) {
    orc::transport_velocity(alp, beta, z, W, vt);
  }
  static void char_speeds(double alp, const double* beta, double rho, double p, double eps,
                          double cs2, double W, double b2, const double* vt, double guu,
                          int d, double& cm, double& cp) {
    orc::char_speeds(alp, beta, rho, p, eps, cs2, W, b2, vt, guu, d, cm, cp);
  }
  static void cons_and_flux(double alp, const double* beta, const double* g, double rho,
                            double p, double eps, const double* z, double s, double W,
                            double b2, const double* b, const double* vt, int d, double& D,
                            double& tau, double S[3], double& ents, double& fD, double& ft,
                            double fS[3], double& fe) {
    orc::cons_and_flux(alp, beta, g, rho, p, eps, z, s, W, b2, b, vt, d, D, tau, S, ents, fD,
                       ft, fS, fe);
  }
  static void geom_sources(double alp, const double* beta, const double* g, const double* guu,
                           const double* K, const double* dalp, const double* dg,
                           const double* db, double rho, double p, double eps, const double* B,
                           const double* z, double W, double& st, double sS[3]) {
    orc::geom_sources(alp, beta, g, guu, K, dalp, dg, db, rho, p, eps, B, z, W, st, sS);
  }
  static double hll(double fL, double fR, double uL, double uR, double cmin, double cmax) {
    return orc::hll(fL, fR, uL, uR, cmin, cmax);
  }
  static void prims_to_conservs(const double pr[13], double c[10], const Metric& m) {
    orc::prims_to_conservs(pr, c, m);
  }
  static bool c2p_counted(double cons[10], double pr[13], const Metric& m, const Eos& e,
                          const grb_params& P, double r, uint32_t& err, bool dry, int& fatal,
                          double alp_bh_override, int* iters) {
    C2PParams c = make_c2p_params(P);
    if (alp_bh_override > 0) c.alp_bh_thresh = alp_bh_override;
    C2PStats st;
    const bool fl = conservs_to_prims(cons, pr, m, e, c, r, err, dry, fatal, &st);
    if (iters) *iters = st.brent_iters;
    return fl;
  }
  static bool c2p(double cons[10], double pr[13], const Metric& m, const Eos& e,
                  const grb_params& P, double r, uint32_t& err, bool dry, int& fatal,
                  double alp_bh_override) {
    return c2p_counted(cons, pr, m, e, P, r, err, dry, fatal, alp_bh_override, nullptr);
  }
  // Gardiner-Stone edge EMF (grmhd_helpers.hh:492-627): average of the four
  // face EMFs plus upwinded (by the sign of the mass flux) corrections
  // towards the cell-centred E.
  template <class St>
  static double gs_edge(St& s, int dir, int i, int j, int k, int64_t q) {
    auto sg = [](double x) { return std::copysign(1., x); };
    if (dir == 0) {
      const double Ezf = s.EF(i, j, k, 0, 2, q), Ezfm = s.EF(i, j - 1, k, 0, 2, q);
      const double Eyf = s.EF(i, j, k, 0, 1, q), Eyfm = s.EF(i, j, k - 1, 0, 1, q);
      const double NE = s.EC(i, j, k, 0, q), NW = s.EC(i, j - 1, k, 0, q);
      const double SE = s.EC(i, j, k - 1, 0, q), SW = s.EC(i, j - 1, k - 1, 0, q);
      const double avg = 0.25 * (Ezf + Ezfm + Eyf + Eyfm);
      const double a = sg(s.F(i, j, k, GRB_DENS, 1, q)), am = sg(s.F(i, j, k - 1, GRB_DENS, 1, q));
      const double dN = (1. - a) * (NE - Ezf) + (1. + a) * (NW - Ezfm);
      const double dS = (1. - am) * (Ezf - SE) + (1. + am) * (Ezfm - SW);
      const double b = sg(s.F(i, j, k, GRB_DENS, 2, q)), bm = sg(s.F(i, j - 1, k, GRB_DENS, 2, q));
      const double dE = (1. - b) * (NE - Eyf) + (1. + b) * (SE - Eyfm);
      const double dW = (1. - bm) * (Eyf - NW) + (1. + bm) * (Eyfm - SW);
      return avg + (1. / 8.) * (dS - dN) + (1. / 8.) * (dW - dE);
    } else if (dir == 1) {
      const double Ezf = s.EF(i, j, k, 1, 2, q), Ezfm = s.EF(i - 1, j, k, 1, 2, q);
      const double Exf = s.EF(i, j, k, 0, 0, q), Exfm = s.EF(i, j, k - 1, 0, 0, q);
      const double NE = s.EC(i, j, k, 1, q), NW = s.EC(i - 1, j, k, 1, q);
      const double SE = s.EC(i, j, k - 1, 1, q), SW = s.EC(i - 1, j, k - 1, 1, q);
      const double avg = 0.25 * (Ezf + Ezfm + Exf + Exfm);
      const double a = sg(s.F(i, j, k, GRB_DENS, 0, q)), am = sg(s.F(i, j, k - 1, GRB_DENS, 0, q));
      const double dN = (1. - a) * (NE - Ezf) + (1. + a) * (NW - Ezfm);
      const double dS = (1. - am) * (Ezf - SE) + (1. + am) * (Ezfm - SW);
      const double b = sg(s.F(i, j, k, GRB_DENS, 2, q)), bm = sg(s.F(i - 1, j, k, GRB_DENS, 2, q));
      const double dE = (1. - b) * (NE - Exf) + (1. + b) * (SE - Exfm);
      const double dW = (1. - bm) * (Exf - NW) + (1. + bm) * (Exfm - SW);
      return avg + (1. / 8.) * (dS - dN) + (1. / 8.) * (dW - dE);
    } else {
      const double Eyf = s.EF(i, j, k, 1, 1, q), Eyfm = s.EF(i - 1, j, k, 1, 1, q);
      const double Exf = s.EF(i, j, k, 1, 0, q), Exfm = s.EF(i, j - 1, k, 1, 0, q);
      const double NE = s.EC(i, j, k, 2, q), NW = s.EC(i - 1, j, k, 2, q);
      const double SE = s.EC(i, j - 1, k, 2, q), SW = s.EC(i - 1, j - 1, k, 2, q);
      const double avg = 0.25 * (Eyf + Eyfm + Exf + Exfm);
      const double a = sg(s.F(i, j, k, GRB_DENS, 0, q)), am = sg(s.F(i, j - 1, k, GRB_DENS, 0, q));
      const double dN = (1. - a) * (NE - Eyf) + (1. + a) * (NW - Eyfm);
      const double dS = (1. - am) * (Eyf - SE) + (1. + am) * (Eyfm - SW);
      const double b = sg(s.F(i, j, k, GRB_DENS, 1, q)), bm = sg(s.F(i - 1, j, k, GRB_DENS, 1, q));
      const double dE = (1. - b) * (NE - Exf) + (1. + b) * (SE - Exfm);
      const double dW = (1. - bm) * (Exf - NW) + (1. + bm) * (Exfm - SW);
      return avg + (1. / 8.) * (dS - dN) + (1. / 8.) * (dW - dE);
    }
  }
};
}  // namespace orc

#define NUMERICS orc::OracleNumerics
#define API(name) orc_##name
#include "api_impl.hpp"
#include "mlp_oracle.hpp"

// FMR restriction into coarse buffers (amr_oracle.hpp).
#include "amr_oracle.hpp"
extern "C" void orc_restrict_cells(int n, int ngz, int nvars, const double* src, double* dst, int64_t nquads,
                                   const int64_t* src_q, const int64_t* dst_q, const uint8_t* child,
                                   const int* vlo, int nlo, const int* vhi, int nhi) {
  orc_amr::restrict_cells(orc_amr::OrcOps{}, n, ngz, nvars, src, dst, nquads, src_q, dst_q, child, vlo, nlo, vhi,
                          nhi);
}
extern "C" void orc_restrict_faces(int dir, int n, int ngz, const double* src, double* dst, int64_t nquads,
                                   const int64_t* src_q, const int64_t* dst_q) {
  orc_amr::restrict_faces(dir, n, ngz, src, dst, nquads, src_q, dst_q);
}
extern "C" void orc_prolong_cells(int kind, int n, int ngz, int nvars, double* fine, const double* cbuf,
                                  int64_t nelems, const int64_t* fine_q, const int64_t* cbuf_q, const uint8_t* elem,
                                  const int* vlo, int nlo, const int* vhi, int nhi) {
  orc_amr::prolong_cells(kind, n, ngz, nvars, fine, cbuf, nelems, fine_q, cbuf_q, elem, vlo, nlo, vhi, nhi);
}
extern "C" void orc_prolong_faces(int kind, int n, int ngz, double* fx, double* fy, double* fz, const double* cx,
                                  const double* cy, const double* cz, int64_t nelems, const int64_t* fine_q,
                                  const int64_t* cbuf_q, const uint8_t* elem, const int8_t* have_fine) {
  orc_amr::prolong_faces(kind, n, ngz, fx, fy, fz, cx, cy, cz, nelems, fine_q, cbuf_q, elem, have_fine);
}
