// CPU oracle — test infrastructure only (see grmhd_numerics.hpp).
//
// extern "C" entry points over Stage<N>, shared by the oracle build (prefix
// orc_) and the reference-numerics pinning build (prefix ref_).  Before
// including, define NUMERICS (the policy type) and API(name) (the prefixed
// symbol name).
#include <cstdint>
#include <cstring>
#include <vector>

#include "stage_driver.hpp"

using StageT = orc::Stage<NUMERICS>;

namespace {
struct Handle {
  StageT st;
  Handle(const grb_params& p, const orc::Dims& d) : st(p, d) {}
};
orc::Fields mk(double* s, double* bx, double* by, double* bz) { return orc::Fields{s, bx, by, bz}; }
}  // namespace

extern "C" {

void* API(create)(const grb_params* p, int nx, int ny, int nz, int g, int64_t nq) {
  return new Handle(*p, orc::Dims(nx, ny, nz, g, nq));
}
void API(destroy)(void* h) { delete static_cast<Handle*>(h); }

int API(advance_substep)(void* hh, const double* idx, const double* coords, double dt,
                         double dtfact, double* ns, double* nbx, double* nby, double* nbz,
                         double* os, double* obx, double* oby, double* obz, const double* aux) {
  auto& st = static_cast<Handle*>(hh)->st;
  st.idx = idx;
  st.coords = coords;
  st.advance_substep(dt, dtfact, mk(ns, nbx, nby, nbz), mk(os, obx, oby, obz), aux);
  return 0;
}
int API(compute_aux)(void* hh, const double* idx, const double* coords, double* s, double* bx,
                     double* by, double* bz, double* aux) {
  auto& st = static_cast<Handle*>(hh)->st;
  st.idx = idx;
  st.coords = coords;
  st.compute_aux(mk(s, bx, by, bz), aux);
  return st.fatal;
}
// Reflux descriptor lists (the layout of grb_reflux, host arrays, copied).
void API(set_reflux)(void* hh, int64_t nfaces, const int64_t* fcq, const uint8_t* fcid, const int64_t* ffq,
                     int64_t nsame, const int64_t* sq, const uint8_t* sid, int32_t flux_same, int64_t nedges,
                     const uint8_t* ens, const uint8_t* eid, const uint8_t* efine, const int64_t* eq,
                     const uint8_t* eoff, int64_t nsedges, const uint8_t* sens, const uint8_t* seid,
                     const int64_t* seq) {
  auto& r = static_cast<Handle*>(hh)->st.rf;
  auto cp = [](auto& v, const auto* p, int64_t n) { v.assign(p, p + (p ? n : 0)); };
  cp(r.face_cq, fcq, nfaces); cp(r.face_cid, fcid, nfaces); cp(r.face_fq, ffq, 4 * nfaces);
  cp(r.same_q, sq, 2 * nsame); cp(r.same_id, sid, 2 * nsame);
  r.flux_same = flux_same != 0;
  cp(r.edge_ns, ens, nedges); cp(r.edge_id, eid, 4 * nedges); cp(r.edge_fine, efine, 4 * nedges);
  cp(r.edge_q, eq, 8 * nedges); cp(r.edge_off, eoff, 8 * nedges);
  cp(r.sedge_ns, sens, nsedges); cp(r.sedge_id, seid, 4 * nsedges); cp(r.sedge_q, seq, 4 * nsedges);
}
void API(reset_diag)(void* hh, double* aux) { static_cast<Handle*>(hh)->st.reset_diag(aux); }
double API(find_stable_timestep)(void* hh, double* s, const double* aux, const double* dx, double cfl) {
  return static_cast<Handle*>(hh)->st.find_stable_timestep(mk(s, nullptr, nullptr, nullptr), aux, dx, cfl);
}
void API(linop)(void* hh, double* as, double* abx, double* aby, double* abz, double* bs,
                double* bbx, double* bby, double* bbz, double* cs, double* cbx, double* cby,
                double* cbz, double b, double c) {
  auto& st = static_cast<Handle*>(hh)->st;
  orc::Fields C = mk(cs, cbx, cby, cbz);
  st.linop(mk(as, abx, aby, abz), mk(bs, bbx, bby, bbz), cs ? &C : nullptr, b, c);
}
// copy out a scratch array: 0 fluxes, 1 Eface, 2 vbar, 3 Ecenter, 4 emf;
// returns the element count (call with out == NULL to size).
int64_t API(scratch)(void* hh, int which, double* out) {
  auto& st = static_cast<Handle*>(hh)->st;
  std::vector<double>* v = which == 0 ? &st.flux : which == 1 ? &st.eface : which == 2 ? &st.vbar
                         : which == 3 ? &st.ecenter : &st.emf;
  if (out) std::memcpy(out, v->data(), v->size() * sizeof(double));
  return (int64_t)v->size();
}
// Mass outflux of the last substep through the listed outer-boundary faces
// (boundary_outflow_t::accumulate, include/grace/evolution/
// boundary_outflow.hh:79-180): per face (quad[f], face[f] = 2 axis + side)
// the DENS face flux of the boundary plane summed over the face's interior
// cells in the reference's order (first tangential index fastest), times
// the outward sign, dt * dtfact and the face area from dx[3 q + d]; the
// faces' contributions summed in list order.
double API(boundary_outflow)(void* hh, int64_t nfaces, const int64_t* quad, const uint8_t* face,
                             const double* dx, double dt, double dtfact) {
  auto& st = static_cast<Handle*>(hh)->st;
  const auto& d = st.d;
  const int n[3] = {d.nx, d.ny, d.nz};
  double total = 0.0;
  for (int64_t f = 0; f < nfaces; ++f) {
    const int64_t q = quad[f];
    const int axis = face[f] / 2;
    const double sgn = (face[f] & 1) ? 1.0 : -1.0;
    const double* h = dx + 3 * q;
    const double dA = axis == 0 ? h[1] * h[2] : axis == 1 ? h[0] * h[2] : h[0] * h[1];
    const int plane = (face[f] & 1) ? n[axis] + d.g : d.g;
    const int na = axis == 0 ? d.ny : d.nx, nb = axis == 2 ? d.ny : d.nz;
    double sum = 0.0;
    for (int lin = 0; lin < na * nb; ++lin) {
      const int a = d.g + lin % na, b = d.g + lin / na;
      const int i = axis == 0 ? plane : a;
      const int j = axis == 1 ? plane : (axis == 0 ? a : b);
      const int k = axis == 2 ? plane : b;
      sum += st.F(i, j, k, 0, axis, q);
    }
    total += sgn * (dt * dtfact) * dA * sum;
  }
  return total;
}
void API(fofc_counts)(void* hh, int64_t* faces, int64_t* edges) {
  auto& st = static_cast<Handle*>(hh)->st;
  *faces = st.n_fofc_faces;
  *edges = st.n_fofc_edges;
}

// Batched c2p on SoA arrays: cons[10][n], metric[10][n] (g6, beta3, alp)
// or NULL (flat), prims[13][n], cons_out[10][n] or NULL, err[n], floored[n]
// or NULL, iters[n] or NULL (Brent iterations of the Kastaun solve).
int API(c2p_batch)(const grb_params* p, int64_t n, const double* cons, const double* metric,
                   double* prims, double* cons_out, uint32_t* err, int32_t* floored,
                   int32_t dry_run, int32_t* iters) {
  const auto eos = NUMERICS::make_eos(p->eos);
  int fatal_all = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : fatal_all)
  for (int64_t t = 0; t < n; ++t) {
    double g[6] = {1, 0, 0, 1, 0, 1}, b[3] = {0, 0, 0}, alp = 1.0;
    if (metric) {
      for (int a = 0; a < 6; ++a) g[a] = metric[a * n + t];
      for (int a = 0; a < 3; ++a) b[a] = metric[(6 + a) * n + t];
      alp = metric[9 * n + t];
    }
    const orc::Metric m = NUMERICS::metric(g, b, alp);
    double c[10], pr[13] = {0};
    for (int v = 0; v < 10; ++v) c[v] = cons[v * n + t];
    uint32_t e = 0;
    int fat = 0;
    int it = 0;
    const bool fl = NUMERICS::c2p_counted(c, pr, m, eos, *p, 0.0, e, dry_run != 0, fat,
                                          dry_run ? 1e30 : -1.0, &it);
    fatal_all |= fat;
    for (int v = 0; v < 13; ++v) prims[v * n + t] = pr[v];
    if (cons_out)
      for (int v = 0; v < 10; ++v) cons_out[v * n + t] = c[v];
    if (err) err[t] = e;
    if (floored) floored[t] = fl ? 1 : 0;
    if (iters) iters[t] = it;
  }
  return fatal_all;
}

int API(prims_to_conservs)(const grb_params* p, int64_t n, const double* prims,
                           const double* metric, double* cons) {
  (void)p;
  for (int64_t t = 0; t < n; ++t) {
    double g[6] = {1, 0, 0, 1, 0, 1}, b[3] = {0, 0, 0}, alp = 1.0;
    if (metric) {
      for (int a = 0; a < 6; ++a) g[a] = metric[a * n + t];
      for (int a = 0; a < 3; ++a) b[a] = metric[(6 + a) * n + t];
      alp = metric[9 * n + t];
    }
    const orc::Metric m = NUMERICS::metric(g, b, alp);
    double pr[13], c[10] = {0};
    for (int v = 0; v < 13; ++v) pr[v] = prims[v * n + t];
    NUMERICS::prims_to_conservs(pr, c, m);
    for (int v = 0; v < 10; ++v) cons[v * n + t] = c[v];
  }
  return 0;
}

// EOS: P, eps, cs2 from (T, rho) on n samples (in-place clamps written back)
int API(eos_press_eps_csnd2_temp_rho)(const grb_params* p, int64_t n, double* temp, double* rho,
                                      double* press, double* eps, double* cs2) {
  const auto eos = NUMERICS::make_eos(p->eos);
  for (int64_t t = 0; t < n; ++t)
    press[t] = NUMERICS::press_eps_csnd2__temp_rho(eos, eps[t], cs2[t], temp[t], rho[t]);
  return 0;
}

void API(recon)(int kind, int64_t n, const double* u6, double* uL, double* uR) {
  for (int64_t t = 0; t < n; ++t) NUMERICS::recon(kind, u6 + 6 * t, uL[t], uR[t]);
}

// Per-state physics kernels for pinning (all arrays AoS per sample):
// in[24*t]: alp, beta3, g6, rho, press, eps, cs2, z3, B3, s (21 used of 24);
// out[32*t]: W, b^mu, b2, vtilde3, cm, cp, D, tau, S3, s*, fD, ftau, fS3, fs*,
// sqrtg, ginv6.
void API(kernels)(int64_t n, const double* in, int dir, double* out) {
  for (int64_t t = 0; t < n; ++t) {
    const double* a = in + 24 * t;
    const double alp = a[0];
    const double* beta = a + 1;
    const double* g = a + 4;
    const double rho = a[10], press = a[11], eps = a[12], cs2 = a[13];
    const double* z = a + 14;
    const double* B = a + 17;
    const double s = a[20];
    const orc::Metric m = NUMERICS::metric(g, beta, alp);
    double* o = out + 32 * t;
    const double W = NUMERICS::lorentz(g, z);
    double b[4], b2, vt[3];
    NUMERICS::comoving_b(alp, beta, g, B, z, W, b, b2);
    NUMERICS::vtilde(alp, beta, z, W, vt);
    static const int diag[3] = {0, 3, 5};
    double cm, cp;
    NUMERICS::char_speeds(alp, beta, rho, press, eps, cs2, W, b2, vt, m.ginv[diag[dir]], dir, cm, cp);
    double D, tau, S[3], ents, fD, ft, fS[3], fe;
    NUMERICS::cons_and_flux(alp, beta, g, rho, press, eps, z, s, W, b2, b, vt, dir, D, tau, S,
                            ents, fD, ft, fS, fe);
    o[0] = W; o[1] = b[0]; o[2] = b[1]; o[3] = b[2]; o[4] = b[3]; o[5] = b2;
    o[6] = vt[0]; o[7] = vt[1]; o[8] = vt[2]; o[9] = cm; o[10] = cp;
    o[11] = D; o[12] = tau; o[13] = S[0]; o[14] = S[1]; o[15] = S[2]; o[16] = ents;
    o[17] = fD; o[18] = ft; o[19] = fS[0]; o[20] = fS[1]; o[21] = fS[2]; o[22] = fe;
    o[23] = m.sqrtg;
    for (int c = 0; c < 6; ++c) o[24 + c] = m.ginv[c];
  }
}

// geometric sources: per sample (alp, beta3, g6, guu6, K6, dalp3, dg18,
// dbeta9, rho, press, eps, B3, z3, W) = 62 doubles; out (stau, sS3).
void API(geom_sources)(int64_t n, const double* in, double* out) {
  for (int64_t t = 0; t < n; ++t) {
    const double* a = in + 62 * t;
    double stau, sS[3];
    NUMERICS::geom_sources(a[0], a + 1, a + 4, a + 10, a + 16, a + 22, a + 25, a + 43, a[52],
                           a[53], a[54], a + 55, a + 58, a[61], stau, sS);
    out[4 * t] = stau;
    for (int c = 0; c < 3; ++c) out[4 * t + 1 + c] = sS[c];
  }
}


// Brick ghost fill (same sweeps as the library's harness helper): periodic
// axes copy from the neighbouring block, the others copy the nearest
// interior cell / face.  HRSC variables and face B only.
void API(fill_ghosts_brick)(int nx, int ny, int nz, int g, int nbx, int nby, int nbz,
                            const int32_t* periodic, double* st, double* bx, double* by, double* bz) {
  const int nin[3] = {nx, ny, nz};
  const int N[3] = {nx + 2 * g, ny + 2 * g, nz + 2 * g};
  const int nb[3] = {nbx, nby, nbz};
  const int64_t nq = (int64_t)nbx * nby * nbz;
  auto qof = [&](const int* c) { return c[0] + (int64_t)nbx * (c[1] + (int64_t)nby * c[2]); };
  for (int ax = 0; ax < 3; ++ax) {
    const int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
    // fd = -1: cell vars; 0..2: face arrays staggered along fd
    for (int fd = -1; fd < 3; ++fd) {
      int n[3] = {N[0], N[1], N[2]};
      if (fd >= 0) n[fd] += 1;
      const bool stag = fd == ax;
      const int nv = fd < 0 ? GRB_N_HRSC : 1;
      double* arr = fd < 0 ? st : fd == 0 ? bx : fd == 1 ? by : bz;
      const int64_t cellsq = (int64_t)n[0] * n[1] * n[2];
      const int64_t vstride = cellsq;
      const int64_t qstride = cellsq * (fd < 0 ? GRB_N_EVOL_VARS : 1);
      for (int64_t q = 0; q < nq; ++q) {
        const int qc[3] = {(int)(q % nbx), (int)((q / nbx) % nby), (int)(q / ((int64_t)nbx * nby))};
        for (int gi = 0; gi < 2 * g; ++gi) {
          const bool lo = gi < g;
          const int ig = lo ? gi : (stag ? nin[ax] + g + 1 + (gi - g) : nin[ax] + gi);
          int src = lo ? ig + nin[ax] : ig - nin[ax];
          int qs[3] = {qc[0], qc[1], qc[2]};
          const bool edge = lo ? (qc[ax] == 0) : (qc[ax] == nb[ax] - 1);
          if (edge && !periodic[ax]) src = lo ? g : (stag ? nin[ax] + g : nin[ax] + g - 1);
          else qs[ax] = (qc[ax] + (lo ? nb[ax] - 1 : 1)) % nb[ax];
          const int64_t qsrc = qof(qs);
          for (int b = 0; b < n[o2]; ++b)
            for (int a = 0; a < n[o1]; ++a) {
              int d[3], si[3];
              d[ax] = ig; d[o1] = a; d[o2] = b;
              si[ax] = src; si[o1] = a; si[o2] = b;
              const int64_t ld = d[0] + (int64_t)n[0] * (d[1] + (int64_t)n[1] * d[2]);
              const int64_t ls = si[0] + (int64_t)n[0] * (si[1] + (int64_t)n[1] * si[2]);
              for (int v = 0; v < nv; ++v) arr[ld + v * vstride + q * qstride] = arr[ls + v * vstride + qsrc * qstride];
            }
        }
      }
    }
  }
}

}  // extern "C"
