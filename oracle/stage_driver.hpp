// CPU oracle — test infrastructure only (see grmhd_numerics.hpp).
//
// Restatement of the loop drivers of GRACE's Cowling GRMHD stage on host
// arrays with GRACE's LayoutLeft layout.  Loop ranges, evaluation order and
// the scratch-array conventions follow:
//   src/evolution/evolve.cpp:456-811   flag_fofc_cells / apply_fofc_correction
//   src/evolution/evolve.cpp:813-1340  compute_fluxes / compute_emfs (GS, UCT)
//   src/evolution/evolve.cpp:1342-1479 add_fluxes_and_source_terms / update_CT
//   src/evolution/evolve.cpp:1671-1717 advance_substep
//   src/evolution/auxiliaries.cpp:81-162 compute_auxiliary_quantities
//   include/grace/physics/grmhd.hh:190-434, 551-970 (per-face / per-cell work)
//   include/grace/utils/tstep_utils.hh:54-229 linop_apply
// The per-cell numerics come from the policy N, so the same loops run with
// this repository's restated numerics (the oracle) and with the reference's
// own functions compiled in place (the pinning build under oracle/ref/).
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>

#include "grace_b200.h"
#include "grmhd_numerics.hpp"

namespace orc {

struct Dims {
  int nx, ny, nz, g;
  int64_t nq;
  int NX, NY, NZ;  // with ghosts
  int FX, FY, FZ;  // face grid (NX+1, ...)
  Dims() = default;
  Dims(int nx_, int ny_, int nz_, int g_, int64_t nq_)
      : nx(nx_), ny(ny_), nz(nz_), g(g_), nq(nq_), NX(nx_ + 2 * g_), NY(ny_ + 2 * g_),
        NZ(nz_ + 2 * g_), FX(NX + 1), FY(NY + 1), FZ(NZ + 1) {}
  size_t cells() const { return (size_t)NX * NY * NZ; }
  size_t fcells() const { return (size_t)FX * FY * FZ; }
};

// Host views over the caller's arrays (GRACE LayoutLeft).
struct Fields {
  double* state;
  double* bx;
  double* by;
  double* bz;
};

template <class N>
struct Stage {
  using Eos = typename N::Eos;
  grb_params P;
  Eos eos;
  Dims d;
  const double* idx = nullptr;     // (3, nq)
  const double* coords = nullptr;  // (3, nq) or null
  // library-owned scratch (persisting between stages, like the singleton
  // arrays of variables.hh:147-206)
  std::vector<double> flux, eface, vbar, ecenter, emf;
  std::vector<int8_t> ftag, etag;
  int fatal = 0;
  int64_t n_fofc_faces = 0, n_fofc_edges = 0;
  // reflux descriptors (grb_reflux, host copies); empty: no refluxing
  struct Reflux {
    std::vector<int64_t> face_cq, face_fq, same_q, edge_q, sedge_q;
    std::vector<uint8_t> face_cid, same_id, edge_ns, edge_id, edge_fine, edge_off, sedge_ns, sedge_id;
    bool flux_same = false;
  } rf;

  Stage(const grb_params& p, const Dims& dd) : P(p), eos(N::make_eos(p.eos)), d(dd) {
    flux.assign(d.fcells() * 7 * 3 * d.nq, 0.0);
    if (P.emf == GRB_EMF_GS) eface.assign(d.fcells() * 2 * 3 * d.nq, 0.0);
    else vbar.assign(d.fcells() * 4 * 3 * d.nq, 0.0);
    ecenter.assign(d.cells() * 3 * d.nq, 0.0);
    emf.assign(d.fcells() * 3 * d.nq, 0.0);
    ftag.assign(d.fcells() * 3 * d.nq, 0);
    etag.assign(d.fcells() * 3 * d.nq, 0);
  }

  // ---- indexing ----------------------------------------------------------
  size_t ci(int i, int j, int k) const { return (size_t)i + d.NX * ((size_t)j + d.NY * (size_t)k); }
  size_t cv(int i, int j, int k, int v, int nv, int64_t q) const {
    return ci(i, j, k) + d.cells() * ((size_t)v + (size_t)nv * q);
  }
  double& S(double* s, int i, int j, int k, int v, int64_t q) const { return s[cv(i, j, k, v, GRB_N_EVOL_VARS, q)]; }
  double& A(double* a, int i, int j, int k, int v, int64_t q) const { return a[cv(i, j, k, v, GRB_N_AUX_VARS, q)]; }
  double& BX(double* b, int i, int j, int k, int64_t q) const {
    return b[(size_t)i + (size_t)(d.NX + 1) * ((size_t)j + d.NY * ((size_t)k + (size_t)d.NZ * q))];
  }
  double& BY(double* b, int i, int j, int k, int64_t q) const {
    return b[(size_t)i + (size_t)d.NX * ((size_t)j + (d.NY + 1) * ((size_t)k + (size_t)d.NZ * q))];
  }
  double& BZ(double* b, int i, int j, int k, int64_t q) const {
    return b[(size_t)i + (size_t)d.NX * ((size_t)j + d.NY * ((size_t)k + (size_t)(d.NZ + 1) * q))];
  }
  double& Bf(const Fields& f, int dir, int i, int j, int k, int64_t q) const {
    return dir == 0 ? BX(f.bx, i, j, k, q) : dir == 1 ? BY(f.by, i, j, k, q) : BZ(f.bz, i, j, k, q);
  }
  size_t fi(int i, int j, int k) const { return (size_t)i + d.FX * ((size_t)j + d.FY * (size_t)k); }
  // fluxes(i,j,k,v,dir,q), v in [0,7)
  double& F(int i, int j, int k, int v, int dir, int64_t q) {
    return flux[fi(i, j, k) + d.fcells() * ((size_t)v + 7 * ((size_t)dir + 3 * q))];
  }
  double& EF(int i, int j, int k, int c, int dir, int64_t q) {
    return eface[fi(i, j, k) + d.fcells() * ((size_t)c + 2 * ((size_t)dir + 3 * q))];
  }
  double& VB(int i, int j, int k, int c, int dir, int64_t q) {
    return vbar[fi(i, j, k) + d.fcells() * ((size_t)c + 4 * ((size_t)dir + 3 * q))];
  }
  double& EC(int i, int j, int k, int c, int64_t q) { return ecenter[ci(i, j, k) + d.cells() * ((size_t)c + 3 * q)]; }
  double& EM(int i, int j, int k, int c, int64_t q) { return emf[fi(i, j, k) + d.fcells() * ((size_t)c + 3 * q)]; }
  int8_t& FT(int i, int j, int k, int dir, int64_t q) { return ftag[fi(i, j, k) + d.fcells() * ((size_t)dir + 3 * q)]; }
  int8_t& ET(int i, int j, int k, int dir, int64_t q) { return etag[fi(i, j, k) + d.fcells() * ((size_t)dir + 3 * q)]; }
  double ix(int dd, int64_t q) const { return idx[dd + 3 * q]; }

  Metric cell_metric(double* s, int i, int j, int k, int64_t q) const {
    double g[6], b[3];
    for (int a = 0; a < 6; ++a) g[a] = S(s, i, j, k, GRB_GXX + a, q);
    for (int a = 0; a < 3; ++a) b[a] = S(s, i, j, k, GRB_BETAX + a, q);
    return N::metric(g, b, S(s, i, j, k, GRB_ALP, q));
  }
  double cell_radius(int i, int j, int k, int64_t q) const {
    if (!coords) return 0.0;
    const double x = coords[3 * q] + i / ix(0, q);
    const double y = coords[3 * q + 1] + j / ix(1, q);
    const double z = coords[3 * q + 2] + k / ix(2, q);
    return std::sqrt(x * x + y * y + z * z);
  }

  // ---- per-face Riemann problem (grmhd.hh:774-970) -----------------------
  void mhd_fluxes(int dir, bool rusanov, double* pl, double* pr, const Metric& m, double f[7],
                  double vb[4]) {
    const double* g = m.g;
    const double* beta = m.beta;
    const double alp = m.alp, sqrtg = m.sqrtg;
    const double wl = N::lorentz(g, pl + PR_ZX), wr = N::lorentz(g, pr + PR_ZX);
    double bl[4], br[4], b2l, b2r;
    N::comoving_b(alp, beta, g, pl + PR_BX, pl + PR_ZX, wl, bl, b2l);
    N::comoving_b(alp, beta, g, pr + PR_BX, pr + PR_ZX, wr, br, b2r);
    double vtl[3], vtr[3];
    N::vtilde(alp, beta, pl + PR_ZX, wl, vtl);
    N::vtilde(alp, beta, pr + PR_ZX, wr, vtr);
    static const int diag[3] = {0, 3, 5};
    double cml, cpl, cmr, cpr, cmin, cmax;
    N::char_speeds(alp, beta, pl[PR_RHO], pl[PR_PRESS], pl[PR_EPS], pl[PR_CS2], wl, b2l, vtl,
                   m.ginv[diag[dir]], dir, cml, cpl);
    N::char_speeds(alp, beta, pr[PR_RHO], pr[PR_PRESS], pr[PR_EPS], pr[PR_CS2], wr, b2r, vtr,
                   m.ginv[diag[dir]], dir, cmr, cpr);
    if (rusanov) {
      cmax = std::max(std::max(std::fabs(cml), std::fabs(cmr)), std::max(std::fabs(cpl), std::fabs(cpr)));
      if (std::min(pl[PR_RHO], pr[PR_RHO]) < P.rusanov_use_c_limit) {
        const double cg = alp * std::sqrt(m.ginv[diag[dir]]) + std::fabs(beta[dir]);
        cmax = std::max(cmax, cg);
      }
      cmin = cmax;
    } else {
      cmin = -std::min(0., std::min(cml, cmr));
      cmax = std::max(0., std::max(cpl, cpr));
    }
    if (cmin < 1e-12 && cmax < 1e-12) { cmin = 1; cmax = 1; }
    if (P.emf == GRB_EMF_UCT) {
      static const int jk[3][2] = {{1, 2}, {0, 2}, {0, 1}};
      vb[0] = N::hll(vtl[jk[dir][0]], vtr[jk[dir][0]], 0, 0, cmin, cmax);
      vb[1] = N::hll(vtl[jk[dir][1]], vtr[jk[dir][1]], 0, 0, cmin, cmax);
      vb[2] = cmin;
      vb[3] = cmax;
    }
    double Dl, tl, Sl[3], el, fdl, ftl, fsl[3], fel;
    double Dr, tr, Sr[3], er, fdr, ftr, fsr[3], fer;
    N::cons_and_flux(alp, beta, g, pl[PR_RHO], pl[PR_PRESS], pl[PR_EPS], pl + PR_ZX, pl[PR_ENT],
                     wl, b2l, bl, vtl, dir, Dl, tl, Sl, el, fdl, ftl, fsl, fel);
    N::cons_and_flux(alp, beta, g, pr[PR_RHO], pr[PR_PRESS], pr[PR_EPS], pr + PR_ZX, pr[PR_ENT],
                     wr, b2r, br, vtr, dir, Dr, tr, Sr, er, fdr, ftr, fsr, fer);
    f[GRB_DENS] = sqrtg * N::hll(fdl, fdr, Dl, Dr, cmin, cmax);
    f[GRB_ENTROPYSTAR] = sqrtg * N::hll(fel, fer, el, er, cmin, cmax);
    f[GRB_TAU] = sqrtg * N::hll(ftl, ftr, tl, tr, cmin, cmax);
    for (int c = 0; c < 3; ++c) f[GRB_SX + c] = sqrtg * N::hll(fsl[c], fsr[c], Sl[c], Sr[c], cmin, cmax);
    const double yl = pl[PR_YE], yr = pr[PR_YE];
    f[GRB_YESTAR] = sqrtg * N::hll(yl * fdl, yr * fdr, yl * Dl, yr * Dr, cmin, cmax);
    if (P.emf == GRB_EMF_GS) {
      const double* Bl = pl + PR_BX;
      const double* Br = pr + PR_BX;
      if (dir == 0) {
        const double Fzl = -Bl[0] * vtl[2] + Bl[2] * vtl[0], Fzr = -Br[0] * vtr[2] + Br[2] * vtr[0];
        vb[0] = sqrtg * N::hll(Fzl, Fzr, Bl[2], Br[2], cmin, cmax);
        const double Fyl = -Bl[0] * vtl[1] + Bl[1] * vtl[0], Fyr = -Br[0] * vtr[1] + Br[1] * vtr[0];
        vb[1] = -sqrtg * N::hll(Fyl, Fyr, Bl[1], Br[1], cmin, cmax);
      } else if (dir == 1) {
        const double Fzl = -Bl[1] * vtl[2] + Bl[2] * vtl[1], Fzr = -Br[1] * vtr[2] + Br[2] * vtr[1];
        vb[0] = -sqrtg * N::hll(Fzl, Fzr, Bl[2], Br[2], cmin, cmax);
        const double Fxl = Bl[0] * vtl[1] - Bl[1] * vtl[0], Fxr = Br[0] * vtr[1] - Br[1] * vtr[0];
        vb[1] = sqrtg * N::hll(Fxl, Fxr, Bl[0], Br[0], cmin, cmax);
      } else {
        const double Fyl = Bl[1] * vtl[2] - Bl[2] * vtl[1], Fyr = Br[1] * vtr[2] - Br[2] * vtr[1];
        vb[0] = sqrtg * N::hll(Fyl, Fyr, Bl[1], Br[1], cmin, cmax);
        const double Fxl = Bl[0] * vtl[2] - Bl[2] * vtl[0], Fxr = Br[0] * vtr[2] - Br[2] * vtr[0];
        vb[1] = -sqrtg * N::hll(Fxl, Fxr, Bl[0], Br[0], cmin, cmax);
      }
    }
  }

  // ---- getflux<idir> (grmhd.hh:551-773) ----------------------------------
  void getflux(int dir, int i, int j, int k, int64_t q, int recon, bool rusanov,
               const Fields& old, const double* aux) {
    const int di = dir == 0, dj = dir == 1, dk = dir == 2;
    double* s = old.state;
    const double alpl = S(s, i - di, j - dj, k - dk, GRB_ALP, q);
    const double alpr = S(s, i, j, k, GRB_ALP, q);
    double gm[10];
    for (int a = 0; a < 10; ++a) {
      const int v = GRB_GXX + a;  // GXX..GZZ, ALP, BETAX..BETAZ
      gm[a] = N::face_interp4(S(s, i - 2 * di, j - 2 * dj, k - 2 * dk, v, q),
                              S(s, i - di, j - dj, k - dk, v, q), S(s, i, j, k, v, q),
                              S(s, i + di, j + dj, k + dk, v, q));
    }
    // gm[6] = ALP, gm[7..9] = BETA
    const Metric m = N::metric(gm, gm + 7, gm[6]);
    static const int av[10] = {GRB_RHO, GRB_ZVECX, GRB_ZVECY, GRB_ZVECZ, GRB_YE,
                               GRB_TEMP, GRB_ENTROPY, GRB_BX, GRB_BY, GRB_BZ};
    static const int pv[10] = {PR_RHO, PR_ZX, PR_ZY, PR_ZZ, PR_YE, PR_TEMP, PR_ENT, PR_BX, PR_BY, PR_BZ};
    double pl[13] = {0}, pr[13] = {0};
    double* a = const_cast<double*>(aux);
    for (int r = 0; r < 10; ++r) {
      double u[6];
      for (int o = -3; o <= 2; ++o) u[o + 3] = A(a, i + o * di, j + o * dj, k + o * dk, av[r], q);
      N::recon(recon, u, pl[pv[r]], pr[pv[r]]);
    }
    if (alpl <= P.alp_ex || alpr <= P.alp_ex) {
      for (int r = 0; r < 10; ++r) {
        pl[pv[r]] = A(a, i - di, j - dj, k - dk, av[r], q);
        pr[pv[r]] = A(a, i, j, k, av[r], q);
      }
    }
    const double bn = Bf(old, dir, i, j, k, q) / m.sqrtg;
    pl[PR_BX + dir] = pr[PR_BX + dir] = bn;
    pl[PR_PRESS] = N::press_eps_csnd2__temp_rho(eos, pl[PR_EPS], pl[PR_CS2], pl[PR_TEMP], pl[PR_RHO]);
    pr[PR_PRESS] = N::press_eps_csnd2__temp_rho(eos, pr[PR_EPS], pr[PR_CS2], pr[PR_TEMP], pr[PR_RHO]);
    double f[7], vb[4];
    mhd_fluxes(dir, rusanov, pl, pr, m, f, vb);
    for (int v = 0; v < 7; ++v) F(i, j, k, v, dir, q) = f[v];
    if (P.emf == GRB_EMF_GS) {
      EF(i, j, k, 0, dir, q) = vb[0];
      EF(i, j, k, 1, dir, q) = vb[1];
    } else {
      for (int c = 0; c < 4; ++c) VB(i, j, k, c, dir, q) = vb[c];
    }
  }

  // compute_fluxes (evolve.cpp:908-998): the full transverse ghost range.
  void compute_fluxes(const Fields& old, const double* aux) {
    const bool rus = P.riemann == GRB_RIEMANN_LLF;
    const int g = d.g;
    for (int dir = 0; dir < 3; ++dir) {
      int lo[3] = {0, 0, 0}, hi[3] = {d.NX, d.NY, d.NZ};
      lo[dir] = g - 1;
      hi[dir] = (dir == 0 ? d.nx : dir == 1 ? d.ny : d.nz) + g + 2;
#pragma omp parallel for collapse(2) schedule(static)
      for (int64_t q = 0; q < d.nq; ++q)
        for (int k = lo[2]; k < hi[2]; ++k)
          for (int j = lo[1]; j < hi[1]; ++j)
            for (int i = lo[0]; i < hi[0]; ++i) getflux(dir, i, j, k, q, P.recon, rus, old, aux);
    }
  }

  // ---- EMFs --------------------------------------------------------------
  // Gardiner-Stone edge EMF (grmhd_helpers.hh:492-627) via the policy.
  void compute_emfs_gs() {
    const int g = d.g;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = g; k < d.nz + g + 1; ++k)
        for (int j = g; j < d.ny + g + 1; ++j)
          for (int i = g; i < d.nx + g + 1; ++i) {
            if (i < d.nx + g) EM(i, j, k, 0, q) = N::gs_edge(*this, 0, i, j, k, q);
            if (j < d.ny + g) EM(i, j, k, 1, q) = N::gs_edge(*this, 1, i, j, k, q);
            if (k < d.nz + g) EM(i, j, k, 2, q) = N::gs_edge(*this, 2, i, j, k, q);
          }
  }
  // UCT (evolve.cpp:1131-1340)
  void recon_face(int recon, const Fields& f, int fdir, int rdir, int i, int j, int k, int64_t q,
                  double& L, double& R) {
    const int di = rdir == 0, dj = rdir == 1, dk = rdir == 2;
    double u[6];
    for (int o = -3; o <= 2; ++o) u[o + 3] = Bf(f, fdir, i + o * di, j + o * dj, k + o * dk, q);
    N::recon(recon, u, L, R);
  }
  void recon_vbar(int recon, int fdir, int comp, int rdir, int i, int j, int k, int64_t q,
                  double& L, double& R) {
    const int di = rdir == 0, dj = rdir == 1, dk = rdir == 2;
    double u[6];
    for (int o = -3; o <= 2; ++o) u[o + 3] = VB(i + o * di, j + o * dj, k + o * dk, comp, fdir, q);
    N::recon(recon, u, L, R);
  }
  void compute_emfs_uct(const Fields& old) {
    const int g = d.g, rk = P.recon;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = g; k < d.nz + g + 1; ++k)
        for (int j = g; j < d.ny + g + 1; ++j)
          for (int i = g; i < d.nx + g + 1; ++i) {
            if (i < d.nx + g) {  // E^x at (i, j-1/2, k-1/2)
              double ByL, ByR, vzL, vzR, BzL, BzR, vyL, vyR;
              recon_face(rk, old, 1, 2, i, j, k, q, ByL, ByR);
              recon_vbar(rk, 1, 1, 2, i, j, k, q, vzL, vzR);
              recon_face(rk, old, 2, 1, i, j, k, q, BzL, BzR);
              recon_vbar(rk, 2, 1, 1, i, j, k, q, vyL, vyR);
              const double cmin_y = std::max(VB(i, j, k, 2, 1, q), VB(i, j, k - 1, 2, 1, q));
              const double cmax_y = std::max(VB(i, j, k, 3, 1, q), VB(i, j, k - 1, 3, 1, q));
              const double cmin_z = std::max(VB(i, j, k, 2, 2, q), VB(i, j - 1, k, 2, 2, q));
              const double cmax_z = std::max(VB(i, j, k, 3, 2, q), VB(i, j - 1, k, 3, 2, q));
              EM(i, j, k, 0, q) = N::hll(vzL * ByL, vzR * ByR, ByL, ByR, cmin_z, cmax_z) -
                                  N::hll(vyL * BzL, vyR * BzR, BzL, BzR, cmin_y, cmax_y);
            }
            if (j < d.ny + g) {  // E^y at (i-1/2, j, k-1/2)
              double BzL, BzR, vxL, vxR, BxL, BxR, vzL, vzR;
              recon_face(rk, old, 2, 0, i, j, k, q, BzL, BzR);
              recon_vbar(rk, 2, 0, 0, i, j, k, q, vxL, vxR);
              recon_face(rk, old, 0, 2, i, j, k, q, BxL, BxR);
              recon_vbar(rk, 0, 1, 2, i, j, k, q, vzL, vzR);
              const double cmin_z = std::max(VB(i, j, k, 2, 2, q), VB(i - 1, j, k, 2, 2, q));
              const double cmax_z = std::max(VB(i, j, k, 3, 2, q), VB(i - 1, j, k, 3, 2, q));
              const double cmin_x = std::max(VB(i, j, k, 2, 0, q), VB(i, j, k - 1, 2, 0, q));
              const double cmax_x = std::max(VB(i, j, k, 3, 0, q), VB(i, j, k - 1, 3, 0, q));
              EM(i, j, k, 1, q) = N::hll(vxL * BzL, vxR * BzR, BzL, BzR, cmin_x, cmax_x) -
                                  N::hll(vzL * BxL, vzR * BxR, BxL, BxR, cmin_z, cmax_z);
            }
            if (k < d.nz + g) {  // E^z at (i-1/2, j-1/2, k)
              double BxL, BxR, vyL, vyR, ByL, ByR, vxL, vxR;
              recon_face(rk, old, 0, 1, i, j, k, q, BxL, BxR);
              recon_vbar(rk, 0, 0, 1, i, j, k, q, vyL, vyR);
              recon_face(rk, old, 1, 0, i, j, k, q, ByL, ByR);
              recon_vbar(rk, 1, 0, 0, i, j, k, q, vxL, vxR);
              const double cmin_x = std::max(VB(i, j, k, 2, 0, q), VB(i, j - 1, k, 2, 0, q));
              const double cmax_x = std::max(VB(i, j, k, 3, 0, q), VB(i, j - 1, k, 3, 0, q));
              const double cmin_y = std::max(VB(i, j, k, 2, 1, q), VB(i - 1, j, k, 2, 1, q));
              const double cmax_y = std::max(VB(i, j, k, 3, 1, q), VB(i - 1, j, k, 3, 1, q));
              EM(i, j, k, 2, q) = N::hll(vyL * BxL, vyR * BxR, BxL, BxR, cmin_y, cmax_y) -
                                  N::hll(vxL * ByL, vxR * ByR, ByL, ByR, cmin_x, cmax_x);
            }
          }
  }

  // CT face update helpers (grmhd_helpers.hh:441-475)
  double ct_bx(const Fields& f, int i, int j, int k, int64_t q, double dte) {
    return BX(f.bx, i, j, k, q) + dte * ((EM(i, j, k + 1, 1, q) - EM(i, j, k, 1, q)) * ix(2, q) +
                                         (EM(i, j, k, 2, q) - EM(i, j + 1, k, 2, q)) * ix(1, q));
  }
  double ct_by(const Fields& f, int i, int j, int k, int64_t q, double dte) {
    return BY(f.by, i, j, k, q) + dte * ((EM(i + 1, j, k, 2, q) - EM(i, j, k, 2, q)) * ix(0, q) +
                                         (EM(i, j, k, 0, q) - EM(i, j, k + 1, 0, q)) * ix(2, q));
  }
  double ct_bz(const Fields& f, int i, int j, int k, int64_t q, double dte) {
    return BZ(f.bz, i, j, k, q) + dte * ((EM(i, j + 1, k, 0, q) - EM(i, j, k, 0, q)) * ix(1, q) +
                                         (EM(i, j, k, 1, q) - EM(i + 1, j, k, 1, q)) * ix(0, q));
  }

  // ---- FOFC (evolve.cpp:456-811) -----------------------------------------
  void flag_fofc(double dt, double dtfact, const Fields& nw, const Fields& old) {
    std::fill(ftag.begin(), ftag.end(), 0);
    std::fill(etag.begin(), etag.end(), 0);
    const int g = d.g;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = g - 1; k < d.nz + g + 1; ++k)
        for (int j = g - 1; j < d.ny + g + 1; ++j)
          for (int i = g - 1; i < d.nx + g + 1; ++i) {
            double cons[10];
            for (int v = 0; v <= GRB_ENTROPYSTAR; ++v)
              cons[v] = S(nw.state, i, j, k, v, q) +
                        dt * dtfact *
                            ((F(i, j, k, v, 0, q) - F(i + 1, j, k, v, 0, q)) * ix(0, q) +
                             (F(i, j, k, v, 1, q) - F(i, j + 1, k, v, 1, q)) * ix(1, q) +
                             (F(i, j, k, v, 2, q) - F(i, j, k + 1, v, 2, q)) * ix(2, q));
            const double dte = dt * dtfact;
            cons[CONS_BX] = 0.5 * (ct_bx(old, i, j, k, q, dte) + ct_bx(old, i + 1, j, k, q, dte));
            cons[CONS_BY] = 0.5 * (ct_by(old, i, j, k, q, dte) + ct_by(old, i, j + 1, k, q, dte));
            cons[CONS_BZ] = 0.5 * (ct_bz(old, i, j, k, q, dte) + ct_bz(old, i, j, k + 1, q, dte));
            bool dmp = false;
            if (P.dmp_enable) {
              const double invM = 1.0 / P.dmp_M;
              const int lv[2] = {GRB_DENS, GRB_TAU};
              for (int n = 0; n < 2 && !dmp; ++n) {
                double vmax = -std::numeric_limits<double>::max();
                double vmin = std::numeric_limits<double>::max();
                for (int kt = -1; kt <= 1; ++kt)
                  for (int jt = -1; jt <= 1; ++jt)
                    for (int it = -1; it <= 1; ++it) {
                      const double v = S(nw.state, i + it, j + jt, k + kt, lv[n], q);
                      vmax = std::fmax(vmax, v);
                      vmin = std::fmin(vmin, v);
                    }
                const double t = cons[lv[n]];
                if (t > P.dmp_M * vmax || t < vmin * invM) dmp = true;
              }
            }
            const Metric m = cell_metric(old.state, i, j, k, q);
            double pr[13] = {0};
            uint32_t err = 0;
            int fat = 0;
            const bool floored = N::c2p(cons, pr, m, eos, P, cell_radius(i, j, k, q), err, true, fat, 1e30);
            if (floored || dmp) {
              FT(i, j, k, 0, q) = 1; FT(i + 1, j, k, 0, q) = 1;
              FT(i, j, k, 1, q) = 1; FT(i, j + 1, k, 1, q) = 1;
              FT(i, j, k, 2, q) = 1; FT(i, j, k + 1, 2, q) = 1;
              ET(i, j, k, 0, q) = 1; ET(i, j + 1, k, 0, q) = 1; ET(i, j, k + 1, 0, q) = 1; ET(i, j + 1, k + 1, 0, q) = 1;
              ET(i, j, k, 1, q) = 1; ET(i + 1, j, k, 1, q) = 1; ET(i, j, k + 1, 1, q) = 1; ET(i + 1, j, k + 1, 1, q) = 1;
              ET(i, j, k, 2, q) = 1; ET(i + 1, j, k, 2, q) = 1; ET(i, j + 1, k, 2, q) = 1; ET(i + 1, j + 1, k, 2, q) = 1;
            }
          }
  }
  void apply_fofc(const Fields& old, const double* aux) {
    const int g = d.g;
    int64_t nf = 0, ne = 0;
    // faces first (correct_{x,y,z}_fluxes_fofc), compaction ranges of evolve.cpp:650-678
#pragma omp parallel for collapse(2) schedule(dynamic) reduction(+ : nf)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = g - 1; k < d.nz + g + 1; ++k)
        for (int j = g - 1; j < d.ny + g + 1; ++j)
          for (int i = g - 1; i < d.nx + g + 1; ++i) {
            if (i >= g && FT(i, j, k, 0, q)) { getflux(0, i, j, k, q, GRB_RECON_DONOR, true, old, aux); ++nf; }
            if (j >= g && FT(i, j, k, 1, q)) { getflux(1, i, j, k, q, GRB_RECON_DONOR, true, old, aux); ++nf; }
            if (k >= g && FT(i, j, k, 2, q)) { getflux(2, i, j, k, q, GRB_RECON_DONOR, true, old, aux); ++nf; }
          }
#pragma omp parallel for collapse(2) schedule(dynamic) reduction(+ : ne)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = g - 1; k < d.nz + g + 1; ++k)
        for (int j = g - 1; j < d.ny + g + 1; ++j)
          for (int i = g - 1; i < d.nx + g + 1; ++i) {
            const bool in3 = i >= g && j >= g && k >= g;
            if (in3 && i < d.nx + g && ET(i, j, k, 0, q)) { EM(i, j, k, 0, q) = N::gs_edge(*this, 0, i, j, k, q); ++ne; }
            if (in3 && j < d.ny + g && ET(i, j, k, 1, q)) { EM(i, j, k, 1, q) = N::gs_edge(*this, 1, i, j, k, q); ++ne; }
            if (in3 && k < d.nz + g && ET(i, j, k, 2, q)) { EM(i, j, k, 2, q) = N::gs_edge(*this, 2, i, j, k, q); ++ne; }
          }
    n_fofc_faces = nf;
    n_fofc_edges = ne;
  }

  // ---- flux divergence + geometric sources (evolve.cpp:1342-1404, grmhd.hh:190-297)
  void add_fluxes_and_sources(double dt, double dtfact, const Fields& nw, const Fields& old,
                              const double* aux) {
    const int g = d.g;
    double* a = const_cast<double*>(aux);
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = g; k < d.nz + g; ++k)
        for (int j = g; j < d.ny + g; ++j)
          for (int i = g; i < d.nx + g; ++i) {
            double* s = old.state;
            const Metric m = cell_metric(s, i, j, k, q);
            const double z[3] = {A(a, i, j, k, GRB_ZVECX, q), A(a, i, j, k, GRB_ZVECY, q), A(a, i, j, k, GRB_ZVECZ, q)};
            const double B[3] = {A(a, i, j, k, GRB_BX, q), A(a, i, j, k, GRB_BY, q), A(a, i, j, k, GRB_BZ, q)};
            const double W = N::lorentz(m.g, z);
            const double h = ix(0, q);  // the reference uses idx(0,q) for all three axes
            auto der = [&](int v, double out[3]) {
              out[0] = N::fd6(S(s, i - 3, j, k, v, q), S(s, i - 2, j, k, v, q), S(s, i - 1, j, k, v, q),
                              S(s, i + 1, j, k, v, q), S(s, i + 2, j, k, v, q), S(s, i + 3, j, k, v, q), h);
              out[1] = N::fd6(S(s, i, j - 3, k, v, q), S(s, i, j - 2, k, v, q), S(s, i, j - 1, k, v, q),
                              S(s, i, j + 1, k, v, q), S(s, i, j + 2, k, v, q), S(s, i, j + 3, k, v, q), h);
              out[2] = N::fd6(S(s, i, j, k - 3, v, q), S(s, i, j, k - 2, v, q), S(s, i, j, k - 1, v, q),
                              S(s, i, j, k + 1, v, q), S(s, i, j, k + 2, v, q), S(s, i, j, k + 3, v, q), h);
            };
            double dalp[3], dbeta[9], dg[18], t3[3];
            der(GRB_ALP, dalp);
            for (int c = 0; c < 3; ++c) {
              der(GRB_BETAX + c, t3);
              for (int dd = 0; dd < 3; ++dd) dbeta[3 * dd + c] = t3[dd];
            }
            for (int c = 0; c < 6; ++c) {
              der(GRB_GXX + c, t3);
              for (int dd = 0; dd < 3; ++dd) dg[6 * dd + c] = t3[dd];
            }
            double K[6];
            for (int c = 0; c < 6; ++c) K[c] = S(s, i, j, k, GRB_KXX + c, q);
            double stau, sS[3];
            N::geom_sources(m.alp, m.beta, m.g, m.ginv, K, dalp, dg, dbeta, A(a, i, j, k, GRB_RHO, q),
                            A(a, i, j, k, GRB_PRESS, q), A(a, i, j, k, GRB_EPS, q), B, z, W, stau, sS);
            double* ns = nw.state;
            S(ns, i, j, k, GRB_TAU, q) += m.sqrtg * dt * dtfact * stau;
            S(ns, i, j, k, GRB_SX, q) += m.sqrtg * dt * dtfact * sS[0];
            S(ns, i, j, k, GRB_SY, q) += m.sqrtg * dt * dtfact * sS[1];
            S(ns, i, j, k, GRB_SZ, q) += m.sqrtg * dt * dtfact * sS[2];
            for (int v = 0; v < GRB_N_HRSC; ++v) {
              const double dFx = (F(i, j, k, v, 0, q) - F(i + 1, j, k, v, 0, q)) * ix(0, q);
              const double dFy = (F(i, j, k, v, 1, q) - F(i, j + 1, k, v, 1, q)) * ix(1, q);
              const double dFz = (F(i, j, k, v, 2, q) - F(i, j, k + 1, v, 2, q)) * ix(2, q);
              S(ns, i, j, k, v, q) += dt * dtfact * ((dFx + dFy) + dFz);
            }
          }
  }

  // update_CT (evolve.cpp:1406-1479)
  void update_ct(double dt, double dtfact, const Fields& nw) {
    const int g = d.g;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = g; k < d.nz + g + 1; ++k)
        for (int j = g; j < d.ny + g + 1; ++j)
          for (int i = g; i < d.nx + g + 1; ++i) {
            if (j < d.ny + g && k < d.nz + g)
              BX(nw.bx, i, j, k, q) += dt * dtfact * ((EM(i, j, k + 1, 1, q) - EM(i, j, k, 1, q)) * ix(2, q) +
                                                      (EM(i, j, k, 2, q) - EM(i, j + 1, k, 2, q)) * ix(1, q));
            if (i < d.nx + g && k < d.nz + g)
              BY(nw.by, i, j, k, q) += dt * dtfact * ((EM(i + 1, j, k, 2, q) - EM(i, j, k, 2, q)) * ix(0, q) +
                                                      (EM(i, j, k, 0, q) - EM(i, j, k + 1, 0, q)) * ix(2, q));
            if (i < d.nx + g && j < d.ny + g)
              BZ(nw.bz, i, j, k, q) += dt * dtfact * ((EM(i, j + 1, k, 0, q) - EM(i, j, k, 0, q)) * ix(1, q) +
                                                      (EM(i, j, k, 1, q) - EM(i + 1, j, k, 1, q)) * ix(0, q));
          }
  }

  // ---- refluxing (refluxing.cpp:528-1170, local branches) --------------
  static int odir(int axis, int which) { return which == 0 ? (axis == 0 ? 1 : 0) : (axis == 2 ? 1 : 2); }
  // reflux_correct_fluxes: the coarse flux on a hanging face := 0.25 x the
  // sum of the 4 fine fluxes (loop order x, y, z); same-level faces (the
  // GRACE_SAME_LEVEL_FACE_AVERAGE option): the mean of the two sides.
  void reflux_fluxes() {
    const int n = d.nx, g = d.g;
    const int64_t nf = (int64_t)rf.face_cq.size();
    for (int64_t iq = 0; iq < nf; ++iq)
      for (int v = 0; v < 7; ++v)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            const int face = rf.face_cid[iq], dir = face / 2;
            int c[3], f[3];
            c[dir] = (face & 1) ? g + n : g;
            c[odir(dir, 0)] = g + i;
            c[odir(dir, 1)] = g + j;
            const int child = (2 * i >= n) + 2 * (2 * j >= n);
            const int64_t qf = rf.face_fq[4 * iq + child];
            f[dir] = (face & 1) ? g : g + n;
            f[odir(dir, 0)] = g + (2 * i) % n;
            f[odir(dir, 1)] = g + (2 * j) % n;
            double s = 0.0;
            for (int ii = 0; ii <= (dir != 0); ++ii)
              for (int jj = 0; jj <= (dir != 1); ++jj)
                for (int kk = 0; kk <= (dir != 2); ++kk) s += F(f[0] + ii, f[1] + jj, f[2] + kk, v, dir, qf);
            s *= 0.25;
            F(c[0], c[1], c[2], v, dir, rf.face_cq[iq]) = s;
          }
    if (!rf.flux_same) return;
    const int64_t ns = (int64_t)rf.same_q.size() / 2;
    for (int64_t iq = 0; iq < ns; ++iq)
      for (int v = 0; v < 7; ++v)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            double* at[2];
            double s = 0.0;
            for (int is = 0; is < 2; ++is) {
              const int fid = rf.same_id[2 * iq + is], fdir = fid / 2;
              int c[3];
              c[fdir] = (fid & 1) ? n + g : g;
              c[odir(fdir, 0)] = g + i;
              c[odir(fdir, 1)] = g + j;
              at[is] = &F(c[0], c[1], c[2], v, fdir, rf.same_q[2 * iq + is]);
              s += *at[is];
            }
            s *= 0.5;
            *at[0] = s;
            *at[1] = s;
          }
  }
  double& edge_em(int eid, int i, bool off_i, bool off_j, int64_t q) {
    const int n = d.nx, g = d.g, edir = eid / 4;
    int c[3];
    c[edir] = g + i;
    c[odir(edir, 0)] = off_i ? n / 2 + g : ((eid & 1) ? n + g : g);
    c[odir(edir, 1)] = off_j ? n / 2 + g : (((eid >> 1) & 1) ? n + g : g);
    return EM(c[0], c[1], c[2], edir, q);
  }
  // reflux_correct_emfs: hanging faces' inner lines, same-level faces'
  // inner lines, hanging edges, same-level edges, in that order
  void reflux_emfs() {
    const int n = d.nx, g = d.g, h = n / 2;
    const int64_t nf = (int64_t)rf.face_cq.size();
    for (int64_t iq = 0; iq < nf; ++iq)
      for (int j = 0; j < h; ++j)
        for (int i = 0; i < h; ++i) {
          const int face = rf.face_cid[iq];
          const int fdir = face / 2, idir = odir(fdir, 0), jdir = odir(fdir, 1), side = face & 1;
          for (int ch = 0; ch < 4; ++ch) {
            const int64_t qf = rf.face_fq[4 * iq + ch];
            int f[3], c[3];
            f[fdir] = side ? g : n + g;
            f[idir] = 2 * i + g;
            f[jdir] = 2 * j + g;
            const double ei = 0.5 * (EM(f[0], f[1], f[2], idir, qf) +
                                     EM(f[0] + (idir == 0), f[1] + (idir == 1), f[2] + (idir == 2), idir, qf));
            const double ej = 0.5 * (EM(f[0], f[1], f[2], jdir, qf) +
                                     EM(f[0] + (jdir == 0), f[1] + (jdir == 1), f[2] + (jdir == 2), jdir, qf));
            c[fdir] = side ? n + g : g;
            c[idir] = i + ((ch & 1) ? h : 0) + g;
            c[jdir] = j + ((ch & 2) ? h : 0) + g;
            if (c[jdir] != h + g && c[jdir] != g) EM(c[0], c[1], c[2], idir, rf.face_cq[iq]) = ei;
            if (c[idir] != h + g && c[idir] != g) EM(c[0], c[1], c[2], jdir, rf.face_cq[iq]) = ej;
          }
        }
    const int64_t ns = (int64_t)rf.same_q.size() / 2;
    for (int64_t iq = 0; iq < ns; ++iq)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double s0 = 0.0, s1 = 0.0;
          double *a0[2], *a1[2];
          bool w0[2], w1[2];
          for (int is = 0; is < 2; ++is) {
            const int fid = rf.same_id[2 * iq + is], fdir = fid / 2, idir = odir(fdir, 0), jdir = odir(fdir, 1);
            const int64_t q = rf.same_q[2 * iq + is];
            int c[3];
            c[fdir] = (fid & 1) ? n + g : g;
            c[idir] = g + i;
            c[jdir] = g + j;
            a0[is] = &EM(c[0], c[1], c[2], idir, q);
            a1[is] = &EM(c[0], c[1], c[2], jdir, q);
            w0[is] = c[jdir] > g;
            w1[is] = c[idir] > g;
            s0 += *a0[is];
            s1 += *a1[is];
          }
          s0 *= 0.5;
          s1 *= 0.5;
          for (int is = 0; is < 2; ++is) {
            if (w0[is]) *a0[is] = s0;
            if (w1[is]) *a1[is] = s1;
          }
        }
    // hanging edges: the fine side of smallest edge id gives every side's value
    const int64_t ne = (int64_t)rf.edge_ns.size();
    std::vector<double> acc((size_t)ne * 2 * n);
    for (int64_t iq = 0; iq < ne; ++iq)
      for (int i = 0; i < n; ++i) {
        int best = 256;
        double v0 = 0.0, v1 = 0.0;
        for (int s = 0; s < rf.edge_ns[iq]; ++s) {
          if (!rf.edge_fine[4 * iq + s]) continue;
          const int eid = rf.edge_id[4 * iq + s];
          if (eid >= best) continue;
          best = eid;
          v0 = edge_em(eid, i, false, false, rf.edge_q[8 * iq + 2 * s]);
          v1 = edge_em(eid, i, false, false, rf.edge_q[8 * iq + 2 * s + 1]);
        }
        acc[(2 * iq) * n + i] = v0;
        acc[(2 * iq + 1) * n + i] = v1;
      }
    for (int64_t iq = 0; iq < ne; ++iq)
      for (int i = 0; i < n; ++i)
        for (int s = 0; s < rf.edge_ns[iq]; ++s) {
          const int eid = rf.edge_id[4 * iq + s];
          const double* a = acc.data() + 2 * iq * n;
          if (!rf.edge_fine[4 * iq + s]) {
            const int ch = (2 * i) >= n, k = (2 * i) % n;
            edge_em(eid, i, rf.edge_off[8 * iq + 2 * s] != 0, rf.edge_off[8 * iq + 2 * s + 1] != 0,
                    rf.edge_q[8 * iq + 2 * s]) = 0.5 * (a[ch * n + k] + a[ch * n + k + 1]);
          } else {
            for (int ch = 0; ch < 2; ++ch) edge_em(eid, i, false, false, rf.edge_q[8 * iq + 2 * s + ch]) = a[ch * n + i];
          }
        }
    // same-level edges: the side of smallest edge id
    const int64_t nse = (int64_t)rf.sedge_ns.size();
    std::vector<double> sacc((size_t)nse * n);
    for (int64_t iq = 0; iq < nse; ++iq)
      for (int i = 0; i < n; ++i) {
        int best = 256;
        double v = 0.0;
        for (int s = 0; s < rf.sedge_ns[iq]; ++s) {
          const int eid = rf.sedge_id[4 * iq + s];
          if (eid >= best) continue;
          best = eid;
          v = edge_em(eid, i, false, false, rf.sedge_q[4 * iq + s]);
        }
        sacc[iq * n + i] = v;
      }
    for (int64_t iq = 0; iq < nse; ++iq)
      for (int i = 0; i < n; ++i)
        for (int s = 0; s < rf.sedge_ns[iq]; ++s)
          edge_em(rf.sedge_id[4 * iq + s], i, false, false, rf.sedge_q[4 * iq + s]) = sacc[iq * n + i];
  }

  // advance_substep (evolve.cpp:1671-1717), with refluxing when descriptor
  // lists are set
  void advance_substep(double dt, double dtfact, const Fields& nw, const Fields& old,
                       const double* aux) {
    compute_fluxes(old, aux);
    if (P.emf == GRB_EMF_GS) compute_emfs_gs(); else compute_emfs_uct(old);
    if (P.fofc_enable && P.emf == GRB_EMF_GS) {
      flag_fofc(dt, dtfact, nw, old);
      apply_fofc(old, aux);
    }
    reflux_fluxes();
    add_fluxes_and_sources(dt, dtfact, nw, old, aux);
    reflux_emfs();
    update_ct(dt, dtfact, nw);
  }

  // compute_auxiliary_quantities (auxiliaries.cpp:81-162, grmhd.hh:306-434)
  void compute_aux(const Fields& st, double* aux) {
    double* s = st.state;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = 0; k < d.NZ; ++k)
        for (int j = 0; j < d.NY; ++j)
          for (int i = 0; i < d.NX; ++i) {
            double cons[10];
            for (int v = 0; v < 7; ++v) cons[v] = S(s, i, j, k, v, q);
            cons[CONS_BX] = 0.5 * (BX(st.bx, i, j, k, q) + BX(st.bx, i + 1, j, k, q));
            cons[CONS_BY] = 0.5 * (BY(st.by, i, j, k, q) + BY(st.by, i, j + 1, k, q));
            cons[CONS_BZ] = 0.5 * (BZ(st.bz, i, j, k, q) + BZ(st.bz, i, j, k + 1, q));
            const Metric m = cell_metric(s, i, j, k, q);
            A(aux, i, j, k, GRB_BX, q) = cons[CONS_BX] / m.sqrtg;
            A(aux, i, j, k, GRB_BY, q) = cons[CONS_BY] / m.sqrtg;
            A(aux, i, j, k, GRB_BZ, q) = cons[CONS_BZ] / m.sqrtg;
            double pr[13] = {0};
            uint32_t err = 0;
            int fat = 0;
            N::c2p(cons, pr, m, eos, P, cell_radius(i, j, k, q), err, false, fat, -1.0);
            if (fat) {
#pragma omp atomic
              fatal |= fat;
            }
            A(aux, i, j, k, GRB_RHO, q) = pr[PR_RHO];
            A(aux, i, j, k, GRB_EPS, q) = pr[PR_EPS];
            A(aux, i, j, k, GRB_PRESS, q) = pr[PR_PRESS];
            A(aux, i, j, k, GRB_TEMP, q) = pr[PR_TEMP];
            A(aux, i, j, k, GRB_ENTROPY, q) = pr[PR_ENT];
            A(aux, i, j, k, GRB_YE, q) = pr[PR_YE];
            A(aux, i, j, k, GRB_ZVECX, q) = pr[PR_ZX];
            A(aux, i, j, k, GRB_ZVECY, q) = pr[PR_ZY];
            A(aux, i, j, k, GRB_ZVECZ, q) = pr[PR_ZZ];
            if (tstb(err, E_RESET_DENS)) {
              A(aux, i, j, k, GRB_C2P_DENS_ERR, q) += S(s, i, j, k, GRB_DENS, q) - cons[CONS_D];
              S(s, i, j, k, GRB_DENS, q) = cons[CONS_D];
            }
            if (tstb(err, E_RESET_STILDE))
              for (int c = 0; c < 3; ++c) S(s, i, j, k, GRB_SX + c, q) = cons[CONS_SX + c];
            if (tstb(err, E_RESET_TAU)) S(s, i, j, k, GRB_TAU, q) = cons[CONS_TAU];
            if (tstb(err, E_RESET_ENTROPY)) S(s, i, j, k, GRB_ENTROPYSTAR, q) = cons[CONS_ENTS];
            if (tstb(err, E_RESET_YE)) S(s, i, j, k, GRB_YESTAR, q) = cons[CONS_YES];
            {
              const uint64_t prev = (uint64_t)A(aux, i, j, k, GRB_C2P_ERR, q);
              A(aux, i, j, k, GRB_C2P_ERR, q) = (double)(prev | (uint64_t)err);
            }
            A(aux, i, j, k, GRB_BDIV, q) =
                ((BX(st.bx, i + 1, j, k, q) - BX(st.bx, i, j, k, q)) * ix(0, q) +
                 (BY(st.by, i, j + 1, k, q) - BY(st.by, i, j, k, q)) * ix(1, q) +
                 (BZ(st.bz, i, j, k + 1, q) - BZ(st.bz, i, j, k, q)) * ix(2, q)) /
                m.sqrtg;
          }
    if (P.emf == GRB_EMF_GS) {
#pragma omp parallel for collapse(2) schedule(static)
      for (int64_t q = 0; q < d.nq; ++q)
        for (int k = 0; k < d.NZ; ++k)
          for (int j = 0; j < d.NY; ++j)
            for (int i = 0; i < d.NX; ++i) {
              const Metric m = cell_metric(s, i, j, k, q);
              const double bx = 0.5 * (BX(st.bx, i, j, k, q) + BX(st.bx, i + 1, j, k, q));
              const double by = 0.5 * (BY(st.by, i, j, k, q) + BY(st.by, i, j + 1, k, q));
              const double bz = 0.5 * (BZ(st.bz, i, j, k, q) + BZ(st.bz, i, j, k + 1, q));
              const double z[3] = {A(aux, i, j, k, GRB_ZVECX, q), A(aux, i, j, k, GRB_ZVECY, q),
                                   A(aux, i, j, k, GRB_ZVECZ, q)};
              const double W = std::sqrt(1. + sq_sym(m.g, z));
              double vt[3];
              for (int c = 0; c < 3; ++c) vt[c] = m.alp * z[c] / W - m.beta[c];
              EC(i, j, k, 0, q) = by * vt[2] - bz * vt[1];
              EC(i, j, k, 1, q) = -bx * vt[2] + bz * vt[0];
              EC(i, j, k, 2, q) = bx * vt[1] - by * vt[0];
            }
    }
  }

  // compute_max_eigenspeed (grmhd.hh:444-519) of one cell from its primitives
  // in aux and the metric in the state
  double max_eigenspeed(double* s, const double* aux, int i, int j, int k, int64_t q) const {
    double* a = const_cast<double*>(aux);
    const double z[3] = {A(a, i, j, k, GRB_ZVECX, q), A(a, i, j, k, GRB_ZVECY, q), A(a, i, j, k, GRB_ZVECZ, q)};
    const double B[3] = {A(a, i, j, k, GRB_BX, q), A(a, i, j, k, GRB_BY, q), A(a, i, j, k, GRB_BZ, q)};
    double rho = A(a, i, j, k, GRB_RHO, q), T = A(a, i, j, k, GRB_TEMP, q);
    const double eps = A(a, i, j, k, GRB_EPS, q), press = A(a, i, j, k, GRB_PRESS, q);
    const Metric m = cell_metric(s, i, j, k, q);
    double h, cs2;
    N::press_h_csnd2__temp_rho(eos, h, cs2, T, rho);
    const double W = N::lorentz(m.g, z);
    double b[4], b2;
    N::comoving_b(m.alp, m.beta, m.g, B, z, W, b, b2);
    double vt[3];
    N::vtilde(m.alp, m.beta, z, W, vt);
    const int diag[3] = {0, 3, 5};
    double cmax = 0.0;
    for (int dir = 0; dir < 3; ++dir) {
      double cm, cp;
      N::char_speeds(m.alp, m.beta, rho, press, eps, cs2, W, b2, vt, m.ginv[diag[dir]], dir, cm, cp);
      cmax = std::fmax(cmax, std::fmax(std::fabs(cp), std::fabs(cm)));
    }
    return cmax;
  }

  // find_stable_timestep_impl (find_stable_timestep.cpp:73-125) on this
  // rank's blocks: min over interior cells of CFL / cmax * dx(0, q)
  double find_stable_timestep(const Fields& st, const double* aux, const double* dx, double cfl) const {
    double dt = std::numeric_limits<double>::max();
#pragma omp parallel for collapse(2) schedule(static) reduction(min : dt)
    for (int64_t q = 0; q < d.nq; ++q)
      for (int k = d.g; k < d.nz + d.g; ++k)
        for (int j = d.g; j < d.ny + d.g; ++j)
          for (int i = d.g; i < d.nx + d.g; ++i) {
            const double cmax = max_eigenspeed(st.state, aux, i, j, k, q);
            const double L = dx[3 * q];
            const double c = cfl / cmax * L;
            dt = dt > c ? c : dt;
          }
    return dt;
  }

  // reset_c2p_diagnostics (evolve.cpp:154-161)
  void reset_diag(double* aux) {
    for (int64_t q = 0; q < d.nq; ++q) {
      std::memset(&A(aux, 0, 0, 0, GRB_C2P_DENS_ERR, q), 0, sizeof(double) * d.cells());
      std::memset(&A(aux, 0, 0, 0, GRB_C2P_ERR, q), 0, sizeof(double) * d.cells());
    }
  }

  // linop_apply (tstep_utils.hh:54-229): A = b B (+ c C)
  void linop(const Fields& Ao, const Fields& Bi, const Fields* Ci, double b, double c) {
    const size_t nc = d.cells() * GRB_N_EVOL_VARS * d.nq;
    const size_t nx = (size_t)(d.NX + 1) * d.NY * d.NZ * d.nq;
    const size_t ny = (size_t)d.NX * (d.NY + 1) * d.NZ * d.nq;
    const size_t nz = (size_t)d.NX * d.NY * (d.NZ + 1) * d.nq;
    auto run = [&](double* a, const double* bb, const double* cc, size_t n) {
#pragma omp parallel for schedule(static)
      for (size_t t = 0; t < n; ++t) a[t] = cc ? b * bb[t] + c * cc[t] : b * bb[t];
    };
    run(Ao.state, Bi.state, Ci ? Ci->state : nullptr, nc);
    run(Ao.bx, Bi.bx, Ci ? Ci->bx : nullptr, nx);
    run(Ao.by, Bi.by, Ci ? Ci->by : nullptr, ny);
    run(Ao.bz, Bi.bz, Ci ? Ci->bz : nullptr, nz);
  }
};

}  // namespace orc
