// Per-item kernels of the Cowling GRMHD stage (one thread per face, edge or
// cell).  Launch ranges and evaluation order follow the reference drivers:
//   compute_fluxes          src/evolution/evolve.cpp:813-1068, grmhd.hh:551-970
//   compute_emfs (GS / UCT) src/evolution/evolve.cpp:1069-1340, grmhd_helpers.hh:492-627
//   flag / apply FOFC       src/evolution/evolve.cpp:456-811
//   fluxes + sources        src/evolution/evolve.cpp:1342-1404, grmhd.hh:190-297
//   update_CT               src/evolution/evolve.cpp:1406-1479
//   aux (c2p, BDIV, E_c)    src/evolution/auxiliaries.cpp:81-162, grmhd.hh:306-434
//   linop_apply             include/grace/utils/tstep_utils.hh:54-229
#pragma once
#include "c2p.cuh"
#include "fastdiv.cuh"
#include "layout.cuh"

namespace grb {

struct StageBufs {
  double* flux;     // fluxes(i,j,k,v,dir,q)
  double* eface;    // GS face EMFs
  double* vbar;     // UCT face velocities and speeds
  double* ecenter;  // GS cell-centred E
  double* emf;      // edge EMFs
  int8_t* ftag;     // FOFC face tags
  int8_t* etag;     // FOFC edge tags
  unsigned long long* counters;  // [0] faces, [1] edges recomputed by FOFC
  uint32_t* flags;  // device status word
  // the deferred aux pass's list of cells (AuxDeferred records) and count
  void* adefer = nullptr;
  unsigned long long* nadefer = nullptr;
  int64_t adefer_cap = 0;
  // compacted list of the tagged faces (tuned mode): entries t << 2 | dir
  // (t the FOFC box index), *fcount of them, room for fcap
  uint32_t* flist = nullptr;
  uint32_t* fcount = nullptr;
  uint32_t fcap = 0;
};

// ---- the Riemann problem at one face (grmhd.hh:774-970) -------------------
template <int dir, bool FAST = false>
__device__ __forceinline__ void mhd_fluxes(const DevParams& P, bool rusanov,
                                           double* pl, double* pr, const Met& m, double f[7],
                                           double vb[4]) {
  const double alp = m.alp, sqrtg = m.sqrtg;
  double wl, wr, iwl = 0.0, iwr = 0.0;
  if (FAST) {
    // 1/W = rsqrt(1 + z^2), W = (1 + z^2) / W: no square root, no division
    const double ql = 1. + sqs(m.g, pl + GRB_P_ZX), qr = 1. + sqs(m.g, pr + GRB_P_ZX);
    iwl = rsqrt(ql);
    iwr = rsqrt(qr);
    wl = ql * iwl;
    wr = qr * iwr;
  } else {
    wl = lorentz(m.g, pl + GRB_P_ZX);
    wr = lorentz(m.g, pr + GRB_P_ZX);
  }
  double bl[4], br[4], b2l, b2r, vtl[3], vtr[3];
  const double gdd = dir == 0 ? m.gi[0] : dir == 1 ? m.gi[3] : m.gi[5];
  double cml, cpl, cmr, cpr, cmin, cmax;
  const double ialp = m.ialp;  // FAST: set by make_met<true>
  if (FAST) {
    comoving_b_f(alp, ialp, m.beta, m.g, pl + GRB_P_BX, pl + GRB_P_ZX, wl, iwl, bl, b2l);
    comoving_b_f(alp, ialp, m.beta, m.g, pr + GRB_P_BX, pr + GRB_P_ZX, wr, iwr, br, b2r);
    vtilde_f(alp, m.beta, pl + GRB_P_ZX, iwl, vtl);
    vtilde_f(alp, m.beta, pr + GRB_P_ZX, iwr, vtr);
    char_speeds_f2(ialp, m.beta[dir], gdd, pl, pr, wl, wr, b2l, b2r, vtl[dir], vtr[dir], cml, cpl, cmr, cpr);
  } else {
    comoving_b(alp, m.beta, m.g, pl + GRB_P_BX, pl + GRB_P_ZX, wl, bl, b2l);
    comoving_b(alp, m.beta, m.g, pr + GRB_P_BX, pr + GRB_P_ZX, wr, br, b2r);
    vtilde(alp, m.beta, pl + GRB_P_ZX, wl, vtl);
    vtilde(alp, m.beta, pr + GRB_P_ZX, wr, vtr);
    char_speeds(alp, m.beta[dir], pl[GRB_P_RHO], pl[GRB_P_PRESS], pl[GRB_P_EPS], pl[GRB_P_CS2], wl,
                b2l, vtl[dir], gdd, cml, cpl);
    char_speeds(alp, m.beta[dir], pr[GRB_P_RHO], pr[GRB_P_PRESS], pr[GRB_P_EPS], pr[GRB_P_CS2], wr,
                b2r, vtr[dir], gdd, cmr, cpr);
  }
  if (rusanov) {
    cmax = fmax(fmax(fabs(cml), fabs(cmr)), fmax(fabs(cpl), fabs(cpr)));
    if (fmin(pl[GRB_P_RHO], pr[GRB_P_RHO]) < P.rusanov_c_limit)
      cmax = fmax(cmax, alp * sqrt(gdd) + fabs(m.beta[dir]));
    cmin = cmax;
  } else {
    cmin = -fmin(0., fmin(cml, cmr));
    cmax = fmax(0., fmax(cpl, cpr));
  }
  if (cmin < 1e-12 && cmax < 1e-12) { cmin = 1; cmax = 1; }
  // FAST: one reciprocal for all HLL fluxes of the face
  const double isum = FAST ? 1.0 / (cmax + cmin) : 0.0;
  auto hll = [&](double fL, double fR, double uL, double uR, double cn, double cx) {
    return FAST ? hll_r(fL, fR, uL, uR, cn, cx, isum) : grb::hll(fL, fR, uL, uR, cn, cx);
  };
  if (P.emf == GRB_EMF_UCT) {
    const int a0 = dir == 0 ? 1 : 0, a1 = dir == 2 ? 1 : 2;
    vb[0] = hll(vtl[a0], vtr[a0], 0, 0, cmin, cmax);
    vb[1] = hll(vtl[a1], vtr[a1], 0, 0, cmin, cmax);
    vb[2] = cmin;
    vb[3] = cmax;
  }
  const ConsFlux L = cons_flux(alp, m.beta, m.g, pl[GRB_P_RHO], pl[GRB_P_PRESS], pl[GRB_P_EPS],
                               pl + GRB_P_ZX, pl[GRB_P_ENT], wl, b2l, bl, vtl, dir, ialp);
  const ConsFlux R = cons_flux(alp, m.beta, m.g, pr[GRB_P_RHO], pr[GRB_P_PRESS], pr[GRB_P_EPS],
                               pr + GRB_P_ZX, pr[GRB_P_ENT], wr, b2r, br, vtr, dir, ialp);
  f[GRB_DENS] = sqrtg * hll(L.fD, R.fD, L.D, R.D, cmin, cmax);
  f[GRB_ENTROPYSTAR] = sqrtg * hll(L.fent, R.fent, L.ents, R.ents, cmin, cmax);
  f[GRB_TAU] = sqrtg * hll(L.ftau, R.ftau, L.tau, R.tau, cmin, cmax);
#pragma unroll
  for (int c = 0; c < 3; ++c) f[GRB_SX + c] = sqrtg * hll(L.fS[c], R.fS[c], L.S[c], R.S[c], cmin, cmax);
  const double yl = pl[GRB_P_YE], yr = pr[GRB_P_YE];
  f[GRB_YESTAR] = sqrtg * hll(yl * L.fD, yr * R.fD, yl * L.D, yr * R.D, cmin, cmax);
  if (P.emf == GRB_EMF_GS) {
    const double* Bl = pl + GRB_P_BX;
    const double* Br = pr + GRB_P_BX;
    if (dir == 0) {
      vb[0] = sqrtg * hll(-Bl[0] * vtl[2] + Bl[2] * vtl[0], -Br[0] * vtr[2] + Br[2] * vtr[0], Bl[2], Br[2], cmin, cmax);
      vb[1] = -sqrtg * hll(-Bl[0] * vtl[1] + Bl[1] * vtl[0], -Br[0] * vtr[1] + Br[1] * vtr[0], Bl[1], Br[1], cmin, cmax);
    } else if (dir == 1) {
      vb[0] = -sqrtg * hll(-Bl[1] * vtl[2] + Bl[2] * vtl[1], -Br[1] * vtr[2] + Br[2] * vtr[1], Bl[2], Br[2], cmin, cmax);
      vb[1] = sqrtg * hll(Bl[0] * vtl[1] - Bl[1] * vtl[0], Br[0] * vtr[1] - Br[1] * vtr[0], Bl[0], Br[0], cmin, cmax);
    } else {
      vb[0] = sqrtg * hll(Bl[1] * vtl[2] - Bl[2] * vtl[1], Br[1] * vtr[2] - Br[2] * vtr[1], Bl[1], Br[1], cmin, cmax);
      vb[1] = -sqrtg * hll(Bl[0] * vtl[2] - Bl[2] * vtl[0], Br[0] * vtr[2] - Br[2] * vtr[0], Bl[0], Br[0], cmin, cmax);
    }
  }
}

// getflux<idir> (grmhd.hh:551-773) reading GRACE arrays through the cache.
template <int dir, bool FAST = false>
__device__ __forceinline__ void getflux(const DevParams& P, const Geo& G, int i, int j,
                                        int k, int64_t q, int recon, bool rusanov,
                                        const double* __restrict__ st,
                                        const double* __restrict__ aux,
                                        const double* __restrict__ bface, double f[7],
                                        double vb[4]) {
  const int64_t s = dir == 0 ? 1 : dir == 1 ? (int64_t)G.NX : (int64_t)G.NX * G.NY;
  const int64_t c0 = cvar(G, i, j, k, 0, GRB_N_EVOL_VARS, q);
  const int64_t a0 = cvar(G, i, j, k, 0, GRB_N_AUX_VARS, q);
  const double alpl = __ldg(st + c0 - s + G.cells * GRB_ALP);
  const double alpr = __ldg(st + c0 + G.cells * GRB_ALP);
  double gm[10];
#pragma unroll
  for (int a = 0; a < 10; ++a) {
    const double* p = st + c0 + G.cells * (GRB_GXX + a);
    gm[a] = face4(__ldg(p - 2 * s), __ldg(p - s), __ldg(p), __ldg(p + s));
  }
  const Met m = make_met<FAST>(gm, gm + 7, gm[6]);
  const int av[10] = {GRB_RHO, GRB_ZVECX, GRB_ZVECY, GRB_ZVECZ, GRB_YE, GRB_TEMP, GRB_ENTROPY, GRB_BX, GRB_BY, GRB_BZ};
  const int pv[10] = {GRB_P_RHO, GRB_P_ZX, GRB_P_ZY, GRB_P_ZZ, GRB_P_YE, GRB_P_TEMP, GRB_P_ENT, GRB_P_BX, GRB_P_BY, GRB_P_BZ};
  double pl[13], pr[13];
  const bool donor = (alpl <= P.alp_ex || alpr <= P.alp_ex);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const double* p = aux + a0 + G.cells * av[r];
    if (donor) {
      pl[pv[r]] = __ldg(p - s);
      pr[pv[r]] = __ldg(p);
    } else {
      double u[6];
#pragma unroll
      for (int o = 0; o < 6; ++o) u[o] = __ldg(p + (o - 3) * s);
      if (FAST) recon6_fast(recon, u, pl[pv[r]], pr[pv[r]]);
      else recon6(recon, u, pl[pv[r]], pr[pv[r]]);
    }
  }
  const int64_t bi = dir == 0 ? bxi(G, i, j, k, q) : dir == 1 ? byi(G, i, j, k, q) : bzi(G, i, j, k, q);
  const double bn = FAST ? __ldg(bface + bi) * m.isqrtg : __ldg(bface + bi) / m.sqrtg;
  pl[GRB_P_BX + dir] = bn;
  pr[GRB_P_BX + dir] = bn;
  uint32_t q0 = 0;
  pl[GRB_P_PRESS] = eos_PT(P.eos, pl[GRB_P_EPS], pl[GRB_P_CS2], nullptr, pl[GRB_P_TEMP], pl[GRB_P_RHO], q0);
  pr[GRB_P_PRESS] = eos_PT(P.eos, pr[GRB_P_EPS], pr[GRB_P_CS2], nullptr, pr[GRB_P_TEMP], pr[GRB_P_RHO], q0);
  mhd_fluxes<dir, FAST>(P, rusanov, pl, pr, m, f, vb);
}

__device__ __forceinline__ void store_face(const Geo& G, const StageBufs& B, int emf_kind, int dir,
                                           int i, int j, int k, int64_t q, const double f[7],
                                           const double vb[4]) {
#pragma unroll
  for (int v = 0; v < 7; ++v) B.flux[flx(G, i, j, k, v, dir, q)] = f[v];
  if (emf_kind == GRB_EMF_GS) {
    B.eface[efi(G, i, j, k, 0, dir, q)] = vb[0];
    B.eface[efi(G, i, j, k, 1, dir, q)] = vb[1];
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) B.vbar[vbi(G, i, j, k, c, dir, q)] = vb[c];
  }
}

// Box of items: [lo, hi) per axis, decoded from a linear thread index.
// dv: the divisors n[0..2], set by the host (box()); an unset or stale
// divisor sends decode to the 64-bit division path.  list (optional): the
// items are instead the nlist cells of list[] in every block, each packed as
// i | j << 8 | k << 16 (dl: the divisor nlist; nlist * nq < 2^32).
struct Box {
  int lo[3], n[3];
  int64_t nq;
  FastDiv dv[3];
  const uint32_t* list = nullptr;
  uint32_t nlist = 0;
  FastDiv dl;
  __host__ __device__ int64_t count() const {
    return list ? (int64_t)nlist * nq : (int64_t)n[0] * n[1] * n[2] * nq;
  }
};
__device__ __forceinline__ bool decode(const Box& b, int64_t t, int& i, int& j, int& k, int64_t& q) {
  if (t >= b.count()) return false;
  if (b.list) {
    const uint32_t u = (uint32_t)t;
    const uint32_t qq = fast_div(u, b.dl);
    const uint32_t c = __ldg(b.list + (u - qq * b.nlist));
    i = (int)(c & 0xffu);
    j = (int)((c >> 8) & 0xffu);
    k = (int)(c >> 16);
    q = qq;
    return true;
  }
  if (t <= 0xffffffffll && b.dv[0].d == (uint32_t)b.n[0] && b.dv[1].d == (uint32_t)b.n[1] &&
      b.dv[2].d == (uint32_t)b.n[2]) {
    const uint32_t u = (uint32_t)t;
    const uint32_t u1 = fast_div(u, b.dv[0]), u2 = fast_div(u1, b.dv[1]), u3 = fast_div(u2, b.dv[2]);
    i = b.lo[0] + (int)(u - u1 * (uint32_t)b.n[0]);
    j = b.lo[1] + (int)(u1 - u2 * (uint32_t)b.n[1]);
    k = b.lo[2] + (int)(u2 - u3 * (uint32_t)b.n[2]);
    q = u3;
    return true;
  }
  i = b.lo[0] + (int)(t % b.n[0]); t /= b.n[0];
  j = b.lo[1] + (int)(t % b.n[1]); t /= b.n[1];
  k = b.lo[2] + (int)(t % b.n[2]); t /= b.n[2];
  q = t;
  return true;
}

template <int dir, bool FAST = false, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) k_flux(DevParams P, Geo G, Box box,
                                               const double* __restrict__ st,
                                               const double* __restrict__ aux,
                                               const double* __restrict__ bface, StageBufs B) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  double f[7], vb[4];
  getflux<dir, FAST>(P, G, i, j, k, q, P.recon, P.riemann == GRB_RIEMANN_LLF, st, aux, bface, f, vb);
  store_face(G, B, P.emf, dir, i, j, k, q, f, vb);
}

// ---- Gardiner-Stone edge EMF (grmhd_helpers.hh:492-627) -------------------
__device__ __forceinline__ double gs_edge(const Geo& G, const StageBufs& B, int dir, int i, int j,
                                          int k, int64_t q) {
  // (a, b): the two face directions feeding this edge; da/db: their
  // transverse neighbour offsets; component slots in Eface.
  const double* EF = B.eface;
  const double* EC = B.ecenter;
  const double* FL = B.flux;
  auto sg = [](double x) { return copysign(1., x); };
  if (dir == 0) {
    const double Ezf = EF[efi(G, i, j, k, 0, 2, q)], Ezfm = EF[efi(G, i, j - 1, k, 0, 2, q)];
    const double Eyf = EF[efi(G, i, j, k, 0, 1, q)], Eyfm = EF[efi(G, i, j, k - 1, 0, 1, q)];
    const double NE = EC[eci(G, i, j, k, 0, q)], NW = EC[eci(G, i, j - 1, k, 0, q)];
    const double SE = EC[eci(G, i, j, k - 1, 0, q)], SW = EC[eci(G, i, j - 1, k - 1, 0, q)];
    const double a = sg(FL[flx(G, i, j, k, GRB_DENS, 1, q)]), am = sg(FL[flx(G, i, j, k - 1, GRB_DENS, 1, q)]);
    const double b = sg(FL[flx(G, i, j, k, GRB_DENS, 2, q)]), bm = sg(FL[flx(G, i, j - 1, k, GRB_DENS, 2, q)]);
    const double avg = 0.25 * (Ezf + Ezfm + Eyf + Eyfm);
    const double dN = (1. - a) * (NE - Ezf) + (1. + a) * (NW - Ezfm);
    const double dS = (1. - am) * (Ezf - SE) + (1. + am) * (Ezfm - SW);
    const double dE = (1. - b) * (NE - Eyf) + (1. + b) * (SE - Eyfm);
    const double dW = (1. - bm) * (Eyf - NW) + (1. + bm) * (Eyfm - SW);
    return avg + (1. / 8.) * (dS - dN) + (1. / 8.) * (dW - dE);
  } else if (dir == 1) {
    const double Ezf = EF[efi(G, i, j, k, 1, 2, q)], Ezfm = EF[efi(G, i - 1, j, k, 1, 2, q)];
    const double Exf = EF[efi(G, i, j, k, 0, 0, q)], Exfm = EF[efi(G, i, j, k - 1, 0, 0, q)];
    const double NE = EC[eci(G, i, j, k, 1, q)], NW = EC[eci(G, i - 1, j, k, 1, q)];
    const double SE = EC[eci(G, i, j, k - 1, 1, q)], SW = EC[eci(G, i - 1, j, k - 1, 1, q)];
    const double a = sg(FL[flx(G, i, j, k, GRB_DENS, 0, q)]), am = sg(FL[flx(G, i, j, k - 1, GRB_DENS, 0, q)]);
    const double b = sg(FL[flx(G, i, j, k, GRB_DENS, 2, q)]), bm = sg(FL[flx(G, i - 1, j, k, GRB_DENS, 2, q)]);
    const double avg = 0.25 * (Ezf + Ezfm + Exf + Exfm);
    const double dN = (1. - a) * (NE - Ezf) + (1. + a) * (NW - Ezfm);
    const double dS = (1. - am) * (Ezf - SE) + (1. + am) * (Ezfm - SW);
    const double dE = (1. - b) * (NE - Exf) + (1. + b) * (SE - Exfm);
    const double dW = (1. - bm) * (Exf - NW) + (1. + bm) * (Exfm - SW);
    return avg + (1. / 8.) * (dS - dN) + (1. / 8.) * (dW - dE);
  } else {
    const double Eyf = EF[efi(G, i, j, k, 1, 1, q)], Eyfm = EF[efi(G, i - 1, j, k, 1, 1, q)];
    const double Exf = EF[efi(G, i, j, k, 1, 0, q)], Exfm = EF[efi(G, i, j - 1, k, 1, 0, q)];
    const double NE = EC[eci(G, i, j, k, 2, q)], NW = EC[eci(G, i - 1, j, k, 2, q)];
    const double SE = EC[eci(G, i, j - 1, k, 2, q)], SW = EC[eci(G, i - 1, j - 1, k, 2, q)];
    const double a = sg(FL[flx(G, i, j, k, GRB_DENS, 0, q)]), am = sg(FL[flx(G, i, j - 1, k, GRB_DENS, 0, q)]);
    const double b = sg(FL[flx(G, i, j, k, GRB_DENS, 1, q)]), bm = sg(FL[flx(G, i - 1, j, k, GRB_DENS, 1, q)]);
    const double avg = 0.25 * (Eyf + Eyfm + Exf + Exfm);
    const double dN = (1. - a) * (NE - Eyf) + (1. + a) * (NW - Eyfm);
    const double dS = (1. - am) * (Eyf - SE) + (1. + am) * (Eyfm - SW);
    const double dE = (1. - b) * (NE - Exf) + (1. + b) * (SE - Exfm);
    const double dW = (1. - bm) * (Exf - NW) + (1. + bm) * (Exfm - SW);
    return avg + (1. / 8.) * (dS - dN) + (1. / 8.) * (dW - dE);
  }
}

// edge range of compute_emfs: [g, n+g] per axis, minus the top along the
// edge's own direction (evolve.cpp:1089-1103)
__global__ void __launch_bounds__(128) k_emf_gs(Geo G, Box box, StageBufs B) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  if (i < G.nx + G.g) B.emf[emi(G, i, j, k, 0, q)] = gs_edge(G, B, 0, i, j, k, q);
  if (j < G.ny + G.g) B.emf[emi(G, i, j, k, 1, q)] = gs_edge(G, B, 1, i, j, k, q);
  if (k < G.nz + G.g) B.emf[emi(G, i, j, k, 2, q)] = gs_edge(G, B, 2, i, j, k, q);
}

// ---- UCT edge EMF (evolve.cpp:1131-1340) ----------------------------------
__device__ __forceinline__ void recon_line(int recon, const double* p, int64_t s, double& L, double& R) {
  double u[6];
#pragma unroll
  for (int o = 0; o < 6; ++o) u[o] = __ldg(p + (o - 3) * s);
  recon6(recon, u, L, R);
}
__global__ void __launch_bounds__(128) k_emf_uct(DevParams P, Geo G, Box box,
                                                  const double* __restrict__ bx,
                                                  const double* __restrict__ by,
                                                  const double* __restrict__ bz, StageBufs B) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  const int rk = P.recon;
  const double* VB = B.vbar;
  // strides of the three face arrays along x, y, z
  const int64_t sxx = 1, sxy = G.NX + 1, sxz = (int64_t)(G.NX + 1) * G.NY;
  const int64_t syx = 1, syy = G.NX, syz = (int64_t)G.NX * (G.NY + 1);
  const int64_t szx = 1, szy = G.NX, szz = (int64_t)G.NX * G.NY;
  const int64_t vs[3] = {1, G.FX, (int64_t)G.FX * G.FY};
  if (i < G.nx + G.g) {  // E^x at (i, j-1/2, k-1/2)
    double ByL, ByR, vzL, vzR, BzL, BzR, vyL, vyR;
    recon_line(rk, by + byi(G, i, j, k, q), syz, ByL, ByR);
    recon_line(rk, VB + vbi(G, i, j, k, 1, 1, q), vs[2], vzL, vzR);
    recon_line(rk, bz + bzi(G, i, j, k, q), szy, BzL, BzR);
    recon_line(rk, VB + vbi(G, i, j, k, 1, 2, q), vs[1], vyL, vyR);
    const double cmin_y = fmax(VB[vbi(G, i, j, k, 2, 1, q)], VB[vbi(G, i, j, k - 1, 2, 1, q)]);
    const double cmax_y = fmax(VB[vbi(G, i, j, k, 3, 1, q)], VB[vbi(G, i, j, k - 1, 3, 1, q)]);
    const double cmin_z = fmax(VB[vbi(G, i, j, k, 2, 2, q)], VB[vbi(G, i, j - 1, k, 2, 2, q)]);
    const double cmax_z = fmax(VB[vbi(G, i, j, k, 3, 2, q)], VB[vbi(G, i, j - 1, k, 3, 2, q)]);
    B.emf[emi(G, i, j, k, 0, q)] = hll(vzL * ByL, vzR * ByR, ByL, ByR, cmin_z, cmax_z) -
                                   hll(vyL * BzL, vyR * BzR, BzL, BzR, cmin_y, cmax_y);
  }
  if (j < G.ny + G.g) {  // E^y at (i-1/2, j, k-1/2)
    double BzL, BzR, vxL, vxR, BxL, BxR, vzL, vzR;
    recon_line(rk, bz + bzi(G, i, j, k, q), szx, BzL, BzR);
    recon_line(rk, VB + vbi(G, i, j, k, 0, 2, q), vs[0], vxL, vxR);
    recon_line(rk, bx + bxi(G, i, j, k, q), sxz, BxL, BxR);
    recon_line(rk, VB + vbi(G, i, j, k, 1, 0, q), vs[2], vzL, vzR);
    const double cmin_z = fmax(VB[vbi(G, i, j, k, 2, 2, q)], VB[vbi(G, i - 1, j, k, 2, 2, q)]);
    const double cmax_z = fmax(VB[vbi(G, i, j, k, 3, 2, q)], VB[vbi(G, i - 1, j, k, 3, 2, q)]);
    const double cmin_x = fmax(VB[vbi(G, i, j, k, 2, 0, q)], VB[vbi(G, i, j, k - 1, 2, 0, q)]);
    const double cmax_x = fmax(VB[vbi(G, i, j, k, 3, 0, q)], VB[vbi(G, i, j, k - 1, 3, 0, q)]);
    B.emf[emi(G, i, j, k, 1, q)] = hll(vxL * BzL, vxR * BzR, BzL, BzR, cmin_x, cmax_x) -
                                   hll(vzL * BxL, vzR * BxR, BxL, BxR, cmin_z, cmax_z);
  }
  if (k < G.nz + G.g) {  // E^z at (i-1/2, j-1/2, k)
    double BxL, BxR, vyL, vyR, ByL, ByR, vxL, vxR;
    recon_line(rk, bx + bxi(G, i, j, k, q), sxy, BxL, BxR);
    recon_line(rk, VB + vbi(G, i, j, k, 0, 0, q), vs[1], vyL, vyR);
    recon_line(rk, by + byi(G, i, j, k, q), syx, ByL, ByR);
    recon_line(rk, VB + vbi(G, i, j, k, 0, 1, q), vs[0], vxL, vxR);
    const double cmin_x = fmax(VB[vbi(G, i, j, k, 2, 0, q)], VB[vbi(G, i, j - 1, k, 2, 0, q)]);
    const double cmax_x = fmax(VB[vbi(G, i, j, k, 3, 0, q)], VB[vbi(G, i, j - 1, k, 3, 0, q)]);
    const double cmin_y = fmax(VB[vbi(G, i, j, k, 2, 1, q)], VB[vbi(G, i - 1, j, k, 2, 1, q)]);
    const double cmax_y = fmax(VB[vbi(G, i, j, k, 3, 1, q)], VB[vbi(G, i - 1, j, k, 3, 1, q)]);
    B.emf[emi(G, i, j, k, 2, q)] = hll(vyL * BxL, vyR * BxR, BxL, BxR, cmin_y, cmax_y) -
                                   hll(vxL * ByL, vxR * ByR, ByL, ByR, cmin_x, cmax_x);
  }
  (void)sxx; (void)syx; (void)szx; (void)szz; (void)syy;
}

// ---- FOFC ------------------------------------------------------------------
__device__ __forceinline__ double ct_bx(const Geo& G, const double* bx, const double* E, const double* ix,
                                        int i, int j, int k, int64_t q, double dte) {
  return bx[bxi(G, i, j, k, q)] + dte * ((E[emi(G, i, j, k + 1, 1, q)] - E[emi(G, i, j, k, 1, q)]) * ix[2] +
                                         (E[emi(G, i, j, k, 2, q)] - E[emi(G, i, j + 1, k, 2, q)]) * ix[1]);
}
__device__ __forceinline__ double ct_by(const Geo& G, const double* by, const double* E, const double* ix,
                                        int i, int j, int k, int64_t q, double dte) {
  return by[byi(G, i, j, k, q)] + dte * ((E[emi(G, i + 1, j, k, 2, q)] - E[emi(G, i, j, k, 2, q)]) * ix[0] +
                                         (E[emi(G, i, j, k, 0, q)] - E[emi(G, i, j, k + 1, 0, q)]) * ix[2]);
}
__device__ __forceinline__ double ct_bz(const Geo& G, const double* bz, const double* E, const double* ix,
                                        int i, int j, int k, int64_t q, double dte) {
  return bz[bzi(G, i, j, k, q)] + dte * ((E[emi(G, i, j + 1, k, 0, q)] - E[emi(G, i, j, k, 0, q)]) * ix[1] +
                                         (E[emi(G, i, j, k, 1, q)] - E[emi(G, i + 1, j, k, 1, q)]) * ix[0]);
}

template <bool FAST = false>
__device__ __forceinline__ Met cell_met(const Geo& G, const double* st, int i, int j, int k, int64_t q) {
  const int64_t c0 = cvar(G, i, j, k, 0, GRB_N_EVOL_VARS, q);
  double g[6], b[3];
#pragma unroll
  for (int a = 0; a < 6; ++a) g[a] = st[c0 + G.cells * (GRB_GXX + a)];
#pragma unroll
  for (int a = 0; a < 3; ++a) b[a] = st[c0 + G.cells * (GRB_BETAX + a)];
  return make_met<FAST>(g, b, st[c0 + G.cells * GRB_ALP]);
}
__device__ __forceinline__ double cell_r(const Geo& G, const double* coords, const double* ix, int i,
                                         int j, int k, int64_t q) {
  if (!coords) return 0.0;
  const double x = coords[3 * q] + i / ix[0], y = coords[3 * q + 1] + j / ix[1], z = coords[3 * q + 2] + k / ix[2];
  return sqrt(x * x + y * y + z * z);
}

// Cells per work-queue item of the persistent launches: 8 tiles of 128.
constexpr int kAuxChunk = 8;

// The persistent loop of a one-thread-per-item kernel: the CTA takes chunks
// of kAuxChunk 128-item tiles of the box from the device work queue *queue
// (zeroed before the launch) until the box is exhausted, and calls
// item(i, j, k, q) for each of its items.  Every thread reaches every
// barrier.
template <class Item>
__device__ __forceinline__ void for_queue_items(const Box& box, unsigned long long* queue, Item&& item) {
  __shared__ unsigned long long chunk;
  const int64_t ntiles = (box.count() + 127) / 128;
  for (;;) {
    if (threadIdx.x == 0) chunk = atomicAdd(queue, (unsigned long long)kAuxChunk);
    __syncthreads();
    const int64_t first = (int64_t)chunk;
    __syncthreads();
    if (first >= ntiles) break;
    for (int c = 0; c < kAuxChunk; ++c) {
      int i, j, k;
      int64_t q;
      if (first + c < ntiles && decode(box, (first + c) * 128 + threadIdx.x, i, j, k, q)) item(i, j, k, q);
    }
  }
}

// k_flux as a persistent launch (tuned candidate); per face the same work.
template <int dir, bool FAST = false, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) k_flux_queue(DevParams P, Geo G, Box box,
                                                     const double* __restrict__ st,
                                                     const double* __restrict__ aux,
                                                     const double* __restrict__ bface, StageBufs B,
                                                     unsigned long long* __restrict__ queue) {
  for_queue_items(box, queue, [&](int i, int j, int k, int64_t q) {
    double f[7], vb[4];
    getflux<dir, FAST>(P, G, i, j, k, q, P.recon, P.riemann == GRB_RIEMANN_LLF, st, aux, bface, f, vb);
    store_face(G, B, P.emf, dir, i, j, k, q, f, vb);
  });
}

// flag_fofc_cells (evolve.cpp:456-635) for one cell of [g-1, n+g]^3
template <bool kFast>
__device__ __forceinline__ void fofc_flag_cell(const DevParams& P, const Geo& G, int i, int j, int k, int64_t q,
                                               double dt, double dtfact, const double* __restrict__ ns,
                                               const double* __restrict__ os, const double* __restrict__ obx,
                                               const double* __restrict__ oby, const double* __restrict__ obz,
                                               const double* __restrict__ idx,
                                               const double* __restrict__ coords, const StageBufs& B) {
  const double ix[3] = {idx[3 * q], idx[3 * q + 1], idx[3 * q + 2]};
  double c[10];
  const double* F = B.flux;
#pragma unroll
  for (int v = 0; v < 7; ++v)
    c[v] = ns[cvar(G, i, j, k, v, GRB_N_EVOL_VARS, q)] +
           dt * dtfact *
               ((F[flx(G, i, j, k, v, 0, q)] - F[flx(G, i + 1, j, k, v, 0, q)]) * ix[0] +
                (F[flx(G, i, j, k, v, 1, q)] - F[flx(G, i, j + 1, k, v, 1, q)]) * ix[1] +
                (F[flx(G, i, j, k, v, 2, q)] - F[flx(G, i, j, k + 1, v, 2, q)]) * ix[2]);
  const double dte = dt * dtfact;
  c[7] = 0.5 * (ct_bx(G, obx, B.emf, ix, i, j, k, q, dte) + ct_bx(G, obx, B.emf, ix, i + 1, j, k, q, dte));
  c[8] = 0.5 * (ct_by(G, oby, B.emf, ix, i, j, k, q, dte) + ct_by(G, oby, B.emf, ix, i, j + 1, k, q, dte));
  c[9] = 0.5 * (ct_bz(G, obz, B.emf, ix, i, j, k, q, dte) + ct_bz(G, obz, B.emf, ix, i, j, k + 1, q, dte));
  bool dmp = false;
  if (P.dmp_enable) {
    const double invM = 1.0 / P.dmp_M;
    const int lv[2] = {GRB_DENS, GRB_TAU};
    for (int n = 0; n < 2 && !dmp; ++n) {
      double vmax = -1.7976931348623157e308, vmin = 1.7976931348623157e308;
      for (int kt = -1; kt <= 1; ++kt)
        for (int jt = -1; jt <= 1; ++jt)
          for (int it = -1; it <= 1; ++it) {
            const double v = ns[cvar(G, i + it, j + jt, k + kt, lv[n], GRB_N_EVOL_VARS, q)];
            vmax = fmax(vmax, v);
            vmin = fmin(vmin, v);
          }
      const double t = c[lv[n]];
      if (t > P.dmp_M * vmax || t < vmin * invM) dmp = true;
    }
  }
  bool floored = false;
  if (!dmp) {  // the c2p dry run only matters when the DMP test passed
    const Met m = cell_met(G, os, i, j, k, q);
    double pr[13];
    floored = c2p_floored<kFast>(c, pr, m, P, cell_r(G, coords, ix, i, j, k, q));
  }
  if (floored || dmp) {
    int8_t* T = B.ftag;
    T[emi(G, i, j, k, 0, q)] = 1; T[emi(G, i + 1, j, k, 0, q)] = 1;
    T[emi(G, i, j, k, 1, q)] = 1; T[emi(G, i, j + 1, k, 1, q)] = 1;
    T[emi(G, i, j, k, 2, q)] = 1; T[emi(G, i, j, k + 1, 2, q)] = 1;
    int8_t* E = B.etag;
    E[emi(G, i, j, k, 0, q)] = 1; E[emi(G, i, j + 1, k, 0, q)] = 1; E[emi(G, i, j, k + 1, 0, q)] = 1; E[emi(G, i, j + 1, k + 1, 0, q)] = 1;
    E[emi(G, i, j, k, 1, q)] = 1; E[emi(G, i + 1, j, k, 1, q)] = 1; E[emi(G, i, j, k + 1, 1, q)] = 1; E[emi(G, i + 1, j, k + 1, 1, q)] = 1;
    E[emi(G, i, j, k, 2, q)] = 1; E[emi(G, i + 1, j, k, 2, q)] = 1; E[emi(G, i, j + 1, k, 2, q)] = 1; E[emi(G, i + 1, j + 1, k, 2, q)] = 1;
  }
}

// over cells [g-1, n+g]^3, one thread per cell
template <int MINB = 1, bool kFast = false>
__global__ void __launch_bounds__(128, MINB) k_fofc_flag(DevParams P, Geo G, Box box, double dt,
                                                    double dtfact, const double* __restrict__ ns,
                                                    const double* __restrict__ os,
                                                    const double* __restrict__ obx,
                                                    const double* __restrict__ oby,
                                                    const double* __restrict__ obz,
                                                    const double* __restrict__ idx,
                                                    const double* __restrict__ coords, StageBufs B) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  fofc_flag_cell<kFast>(P, G, i, j, k, q, dt, dtfact, ns, os, obx, oby, obz, idx, coords, B);
}

// The same as a persistent launch (tuned candidate): one wave of CTAs
// pulling chunks of kAuxChunk tiles of 128 cells, numbered block by block,
// from the device work queue *queue (zeroed before the launch) until the
// box is exhausted; per-cell work unchanged.  For uneven per-block cost
// (the c2p dry run's iterations vary with the state).
template <int MINB = 1, bool kFast = false>
__global__ void __launch_bounds__(128, MINB) k_fofc_flag_queue(DevParams P, Geo G, Box box, double dt,
                                                          double dtfact, const double* __restrict__ ns,
                                                          const double* __restrict__ os,
                                                          const double* __restrict__ obx,
                                                          const double* __restrict__ oby,
                                                          const double* __restrict__ obz,
                                                          const double* __restrict__ idx,
                                                          const double* __restrict__ coords, StageBufs B,
                                                          unsigned long long* __restrict__ queue) {
  __shared__ unsigned long long item;
  const int64_t ntiles = (box.count() + 127) / 128;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(queue, (unsigned long long)kAuxChunk);
    __syncthreads();
    const int64_t first = (int64_t)item;
    __syncthreads();
    if (first >= ntiles) break;
    for (int c = 0; c < kAuxChunk; ++c) {
      int i, j, k;
      int64_t q;
      if (first + c < ntiles && decode(box, (first + c) * 128 + threadIdx.x, i, j, k, q))
        fofc_flag_cell<kFast>(P, G, i, j, k, q, dt, dtfact, ns, os, obx, oby, obz, idx, coords, B);
    }
  }
}

// correct_{x,y,z}_fluxes_fofc: donor + LLF on tagged faces.  The box is the
// compaction range [g-1, n+g]^3; a face of direction d needs index_d >= g.
template <bool FAST = false>
__global__ void __launch_bounds__(128) k_fofc_faces(DevParams P, Geo G, Box box,
                                                     const double* __restrict__ st,
                                                     const double* __restrict__ aux,
                                                     const double* __restrict__ bx,
                                                     const double* __restrict__ by,
                                                     const double* __restrict__ bz, StageBufs B) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  unsigned cnt = 0;
  double f[7], vb[4];
  if (i >= G.g && B.ftag[emi(G, i, j, k, 0, q)]) {
    getflux<0, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, bx, f, vb);
    store_face(G, B, P.emf, 0, i, j, k, q, f, vb);
    ++cnt;
  }
  if (j >= G.g && B.ftag[emi(G, i, j, k, 1, q)]) {
    getflux<1, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, by, f, vb);
    store_face(G, B, P.emf, 1, i, j, k, q, f, vb);
    ++cnt;
  }
  if (k >= G.g && B.ftag[emi(G, i, j, k, 2, q)]) {
    getflux<2, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, bz, f, vb);
    store_face(G, B, P.emf, 2, i, j, k, q, f, vb);
    ++cnt;
  }
  if (cnt) atomicAdd(&B.counters[0], (unsigned long long)cnt);
}

// The FOFC box's tagged faces compacted into B.flist (the faces
// k_fofc_faces recomputes: face (i, j, k, d) of a box cell with index_d >=
// ngz), warp-aggregated appends; entries past B.fcap are dropped and the
// count still grows, which sends k_fofc_faces_list to its whole-box loop.
// Needs box.count() < 2^30.
__global__ void __launch_bounds__(256) k_fofc_scan(Geo G, Box box, StageBufs B) {
  int i, j, k;
  int64_t q;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool tg[3] = {false, false, false};
  if (decode(box, t, i, j, k, q)) {
    tg[0] = i >= G.g && B.ftag[emi(G, i, j, k, 0, q)];
    tg[1] = j >= G.g && B.ftag[emi(G, i, j, k, 1, q)];
    tg[2] = k >= G.g && B.ftag[emi(G, i, j, k, 2, q)];
  }
  const int nm = (int)tg[0] + (int)tg[1] + (int)tg[2];
  const int lane = threadIdx.x & 31;
  int incl = nm;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  uint32_t base = 0;
  if (lane == 31 && total) base = atomicAdd(B.fcount, (uint32_t)total);
  base = __shfl_sync(0xffffffffu, base, 31);
  uint32_t at = base + (uint32_t)(incl - nm);
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (tg[d]) {
      if (at < B.fcap) B.flist[at] = (uint32_t)t << 2 | (uint32_t)d;
      ++at;
    }
}

// k_fofc_faces over the compacted list: a grid-stride loop over the listed
// faces, each recomputed as there (donor reconstruction, LLF); when the
// list overflowed, a grid-stride loop over the whole box instead, reading
// the tags as k_fofc_faces does.
template <bool FAST = false>
__global__ void __launch_bounds__(128) k_fofc_faces_list(DevParams P, Geo G, Box box,
                                                          const double* __restrict__ st,
                                                          const double* __restrict__ aux,
                                                          const double* __restrict__ bx,
                                                          const double* __restrict__ by,
                                                          const double* __restrict__ bz, StageBufs B) {
  const uint32_t n = *B.fcount;
  if (n > B.fcap) {
    unsigned cnt = 0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < box.count();
         t += (int64_t)gridDim.x * blockDim.x) {
      int i, j, k;
      int64_t q;
      decode(box, t, i, j, k, q);
      double f[7], vb[4];
      if (i >= G.g && B.ftag[emi(G, i, j, k, 0, q)]) {
        getflux<0, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, bx, f, vb);
        store_face(G, B, P.emf, 0, i, j, k, q, f, vb);
        ++cnt;
      }
      if (j >= G.g && B.ftag[emi(G, i, j, k, 1, q)]) {
        getflux<1, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, by, f, vb);
        store_face(G, B, P.emf, 1, i, j, k, q, f, vb);
        ++cnt;
      }
      if (k >= G.g && B.ftag[emi(G, i, j, k, 2, q)]) {
        getflux<2, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, bz, f, vb);
        store_face(G, B, P.emf, 2, i, j, k, q, f, vb);
        ++cnt;
      }
    }
    if (cnt) atomicAdd(&B.counters[0], (unsigned long long)cnt);
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && n) atomicAdd(&B.counters[0], (unsigned long long)n);
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const uint32_t w = B.flist[e];
    const int dir = (int)(w & 3u);
    int i, j, k;
    int64_t q;
    decode(box, (int64_t)(w >> 2), i, j, k, q);
    double f[7], vb[4];
    if (dir == 0) getflux<0, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, bx, f, vb);
    else if (dir == 1) getflux<1, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, by, f, vb);
    else getflux<2, FAST>(P, G, i, j, k, q, GRB_RECON_DONOR, true, st, aux, bz, f, vb);
    store_face(G, B, P.emf, dir, i, j, k, q, f, vb);
  }
}
__global__ void __launch_bounds__(128) k_fofc_edges(Geo G, Box box, StageBufs B) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  if (i < G.g || j < G.g || k < G.g) return;
  unsigned cnt = 0;
  if (i < G.nx + G.g && B.etag[emi(G, i, j, k, 0, q)]) { B.emf[emi(G, i, j, k, 0, q)] = gs_edge(G, B, 0, i, j, k, q); ++cnt; }
  if (j < G.ny + G.g && B.etag[emi(G, i, j, k, 1, q)]) { B.emf[emi(G, i, j, k, 1, q)] = gs_edge(G, B, 1, i, j, k, q); ++cnt; }
  if (k < G.nz + G.g && B.etag[emi(G, i, j, k, 2, q)]) { B.emf[emi(G, i, j, k, 2, q)] = gs_edge(G, B, 2, i, j, k, q); ++cnt; }
  if (cnt) atomicAdd(&B.counters[1], (unsigned long long)cnt);
}

// ---- flux divergence + geometric sources on interior cells -----------------
// Sixth-order centred derivatives of the lapse, shift and 3-metric at one
// cell (os + c0: the cell's variable 0), one spacing h for all axes as in
// grmhd.hh:232-235: dalp[jd], db[3 jd + c] = d_jd beta^c,
// dg[6 jd + c] = d_jd g_c.  The 30 values in this order are also the
// layout of the static-metric cache (kMetDer doubles per cell).
constexpr int kMetDer = 30;
__device__ __forceinline__ void metric_derivs(const Geo& G, const double* __restrict__ os, int64_t c0, double h,
                                              double dalp[3], double db[9], double dg[18]) {
  const int64_t sy = G.NX, sz = (int64_t)G.NX * G.NY;
  auto der = [&](int v, double o[3]) {
    const double* p = os + c0 + G.cells * v;
    o[0] = fd6(p[-3], p[-2], p[-1], p[1], p[2], p[3], h);
    o[1] = fd6(p[-3 * sy], p[-2 * sy], p[-sy], p[sy], p[2 * sy], p[3 * sy], h);
    o[2] = fd6(p[-3 * sz], p[-2 * sz], p[-sz], p[sz], p[2 * sz], p[3 * sz], h);
  };
  double t3[3];
  der(GRB_ALP, dalp);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    der(GRB_BETAX + c, t3);
    db[c] = t3[0]; db[3 + c] = t3[1]; db[6 + c] = t3[2];
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    der(GRB_GXX + c, t3);
    dg[c] = t3[0]; dg[6 + c] = t3[1]; dg[12 + c] = t3[2];
  }
}
// Offset of derivative d of interior cell (i, j, k) of block q in the
// static-metric cache: [q][d][k - g][j - g][i - g].
__device__ __forceinline__ int64_t mdi(const Geo& G, int i, int j, int k, int d, int64_t q) {
  return (((q * kMetDer + d) * G.nz + (k - G.g)) * G.ny + (j - G.g)) * G.nx + (i - G.g);
}
// Fills the static-metric cache on interior cells.
__global__ void __launch_bounds__(128) k_metric_derivs(Geo G, Box box, const double* __restrict__ os,
                                                       const double* __restrict__ idx, double* __restrict__ md) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  double d[kMetDer];
  metric_derivs(G, os, cvar(G, i, j, k, 0, GRB_N_EVOL_VARS, q), idx[3 * q], d, d + 3, d + 12);
#pragma unroll
  for (int c = 0; c < kMetDer; ++c) md[mdi(G, i, j, k, c, q)] = d[c];
}

// add_fluxes_and_source_terms for one interior cell.  kCached: the metric
// derivatives from the static-metric cache md (tuned mode, Cowling) instead
// of differentiating the metric here.
template <bool kCached>
__device__ __forceinline__ void update_cell(const DevParams& P, const Geo& G, int i, int j, int k, int64_t q,
                                            double dt, double dtfact, double* __restrict__ ns,
                                            const double* __restrict__ os, const double* __restrict__ aux,
                                            const double* __restrict__ idx, const StageBufs& B,
                                            const double* __restrict__ md) {
  const double ix[3] = {idx[3 * q], idx[3 * q + 1], idx[3 * q + 2]};
  const Met m = cell_met(G, os, i, j, k, q);
  const int64_t a0 = cvar(G, i, j, k, 0, GRB_N_AUX_VARS, q);
  const double z[3] = {aux[a0 + G.cells * GRB_ZVECX], aux[a0 + G.cells * GRB_ZVECY], aux[a0 + G.cells * GRB_ZVECZ]};
  const double Bv[3] = {aux[a0 + G.cells * GRB_BX], aux[a0 + G.cells * GRB_BY], aux[a0 + G.cells * GRB_BZ]};
  const double W = lorentz(m.g, z);
  const int64_t c0 = cvar(G, i, j, k, 0, GRB_N_EVOL_VARS, q);
  double d[kMetDer];
  if (kCached) {
    const int64_t m0 = mdi(G, i, j, k, 0, q), ms = (int64_t)G.nx * G.ny * G.nz;
#pragma unroll
    for (int c = 0; c < kMetDer; ++c) d[c] = md[m0 + c * ms];
  } else {
    metric_derivs(G, os, c0, ix[0], d, d + 3, d + 12);
  }
  double K[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) K[c] = os[c0 + G.cells * (GRB_KXX + c)];
  double stau, sS[3];
  geom_sources(m, K, d, d + 12, d + 3, aux[a0 + G.cells * GRB_RHO], aux[a0 + G.cells * GRB_PRESS],
               aux[a0 + G.cells * GRB_EPS], Bv, z, W, stau, sS);
  const double* F = B.flux;
  const double sd = m.sqrtg * dt * dtfact;
  double src[7] = {0., sd * sS[0], sd * sS[1], sd * sS[2], sd * stau, 0., 0.};
#pragma unroll
  for (int v = 0; v < GRB_N_HRSC; ++v) {
    double* p = ns + c0 + G.cells * v;
    double u = *p;
    if (v >= 1 && v <= 4) u += src[v];
    const double dFx = (F[flx(G, i, j, k, v, 0, q)] - F[flx(G, i + 1, j, k, v, 0, q)]) * ix[0];
    const double dFy = (F[flx(G, i, j, k, v, 1, q)] - F[flx(G, i, j + 1, k, v, 1, q)]) * ix[1];
    const double dFz = (F[flx(G, i, j, k, v, 2, q)] - F[flx(G, i, j, k + 1, v, 2, q)]) * ix[2];
    *p = u + dt * dtfact * ((dFx + dFy) + dFz);
  }
}

template <int MINB = 1, bool kCached = false>
__global__ void __launch_bounds__(128, MINB) k_update(DevParams P, Geo G, Box box, double dt, double dtfact,
                                                 double* __restrict__ ns, const double* __restrict__ os,
                                                 const double* __restrict__ aux,
                                                 const double* __restrict__ idx, StageBufs B,
                                                 const double* __restrict__ md = nullptr) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  update_cell<kCached>(P, G, i, j, k, q, dt, dtfact, ns, os, aux, idx, B, md);
}

// k_update as a persistent launch (tuned candidate); per cell the same work.
template <int MINB = 1, bool kCached = false>
__global__ void __launch_bounds__(128, MINB) k_update_queue(DevParams P, Geo G, Box box, double dt,
                                                       double dtfact, double* __restrict__ ns,
                                                       const double* __restrict__ os,
                                                       const double* __restrict__ aux,
                                                       const double* __restrict__ idx, StageBufs B,
                                                       const double* __restrict__ md,
                                                       unsigned long long* __restrict__ queue) {
  for_queue_items(box, queue, [&](int i, int j, int k, int64_t q) {
    update_cell<kCached>(P, G, i, j, k, q, dt, dtfact, ns, os, aux, idx, B, md);
  });
}

// update_CT on faces [g, n+g] (+1 on the face's own axis)
__global__ void __launch_bounds__(128) k_ct(Geo G, Box box, double dt, double dtfact,
                                             double* __restrict__ bx, double* __restrict__ by,
                                             double* __restrict__ bz, const double* __restrict__ idx,
                                             StageBufs B) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  const double ix[3] = {idx[3 * q], idx[3 * q + 1], idx[3 * q + 2]};
  const double* E = B.emf;
  const double dd = dt * dtfact;
  if (j < G.ny + G.g && k < G.nz + G.g)
    bx[bxi(G, i, j, k, q)] += dd * ((E[emi(G, i, j, k + 1, 1, q)] - E[emi(G, i, j, k, 1, q)]) * ix[2] +
                                    (E[emi(G, i, j, k, 2, q)] - E[emi(G, i, j + 1, k, 2, q)]) * ix[1]);
  if (i < G.nx + G.g && k < G.nz + G.g)
    by[byi(G, i, j, k, q)] += dd * ((E[emi(G, i + 1, j, k, 2, q)] - E[emi(G, i, j, k, 2, q)]) * ix[0] +
                                    (E[emi(G, i, j, k, 0, q)] - E[emi(G, i, j, k + 1, 0, q)]) * ix[2]);
  if (i < G.nx + G.g && j < G.ny + G.g)
    bz[bzi(G, i, j, k, q)] += dd * ((E[emi(G, i, j + 1, k, 0, q)] - E[emi(G, i, j, k, 0, q)]) * ix[1] +
                                    (E[emi(G, i, j, k, 1, q)] - E[emi(G, i + 1, j, k, 1, q)]) * ix[0]);
}

// ---- time step: compute_max_eigenspeed (grmhd.hh:444-519) ----------------
// Largest |characteristic speed| over the three directions of one cell from
// its primitives (as stored in aux) and the cell metric.
GRB_HD double max_eigenspeed(const DevEos& e, const Met& m, const double pr[13]) {
  double rho = pr[GRB_P_RHO], T = pr[GRB_P_TEMP];
  uint32_t q = 0;
  const double cs2 = eos_cs2_T(e, T, rho, q);
  const double W = lorentz(m.g, pr + GRB_P_ZX);
  double b[4], b2, vt[3];
  comoving_b(m.alp, m.beta, m.g, pr + GRB_P_BX, pr + GRB_P_ZX, W, b, b2);
  vtilde(m.alp, m.beta, pr + GRB_P_ZX, W, vt);
  const double gdd[3] = {m.gi[0], m.gi[3], m.gi[5]};
  double cmax = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double cm, cp;
    char_speeds(m.alp, m.beta[d], rho, pr[GRB_P_PRESS], pr[GRB_P_EPS], cs2, W, b2, vt[d], gdd[d], cm, cp);
    cmax = fmax(cmax, fmax(fabs(cp), fabs(cm)));
  }
  return cmax;
}
// find_stable_timestep_impl (find_stable_timestep.cpp:73-125): the minimum
// of cfl / cmax * dx(0, q) over interior cells, reduced into *out as the
// bit pattern of a positive double (ordered like an unsigned integer).
struct DtArgs {
  const double* dx;  // spacings (3, nq)
  double cfl;
  unsigned long long* out;
};
__device__ __forceinline__ void dt_reduce(double v, unsigned long long* out) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v < INFINITY) atomicMin(out, (unsigned long long)__double_as_longlong(v));
}
__global__ void k_dt_init(unsigned long long* out) { *out = (unsigned long long)__double_as_longlong(INFINITY); }

// Separate reduction pass over interior cells (one thread per cell); every
// thread of the CTA reaches the warp reduction.
__global__ void __launch_bounds__(128) k_dt(DevParams P, Geo G, Box box, const double* __restrict__ st,
                                            const double* __restrict__ aux, DtArgs dt) {
  int i = 0, j = 0, k = 0;
  int64_t q = 0;
  double v = INFINITY;
  if (decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) {
    const int64_t a0 = cvar(G, i, j, k, 0, GRB_N_AUX_VARS, q);
    double pr[13];
    pr[GRB_P_RHO] = aux[a0 + G.cells * GRB_RHO];
    pr[GRB_P_TEMP] = aux[a0 + G.cells * GRB_TEMP];
    pr[GRB_P_EPS] = aux[a0 + G.cells * GRB_EPS];
    pr[GRB_P_PRESS] = aux[a0 + G.cells * GRB_PRESS];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      pr[GRB_P_ZX + a] = aux[a0 + G.cells * (GRB_ZVECX + a)];
      pr[GRB_P_BX + a] = aux[a0 + G.cells * (GRB_BX + a)];
    }
    const Met m = cell_met(G, st, i, j, k, q);
    v = dt.cfl / max_eigenspeed(P.eos, m, pr) * dt.dx[3 * q];
  }
  dt_reduce(v, dt.out);
}

// ---- aux: c2p on every cell + resets + C2P_ERR + BDIV + cell-centred E -----
// kDt: also the time-step reduction over the interior cells, from the
// primitives just computed (the aux pass that ends an RK step).
// One cell of the aux pass in three parts: aux_load (the cell's densitized
// cons and cell-centred B, the metric, aux B), the c2p (in one piece, or
// deferred at the entropy backup), aux_finish (prims, resets, C2P_ERR,
// BDIV, the cell-centred E, the dt candidate of an interior cell (kDt) or
// +inf).
struct AuxIn {
  double c[10];
  double bf[6];  // bx0, bx1, by0, by1, bz0, bz1
};
__device__ __forceinline__ Met aux_load(const DevParams& P, const Geo& G, int i, int j, int k, int64_t q,
                                        const double* __restrict__ st, const double* __restrict__ bx,
                                        const double* __restrict__ by, const double* __restrict__ bz,
                                        double* __restrict__ aux, bool write_b, bool kFast, AuxIn& A) {
  const int64_t c0 = cvar(G, i, j, k, 0, GRB_N_EVOL_VARS, q);
  const int64_t a0 = cvar(G, i, j, k, 0, GRB_N_AUX_VARS, q);
  A.bf[0] = bx[bxi(G, i, j, k, q)]; A.bf[1] = bx[bxi(G, i + 1, j, k, q)];
  A.bf[2] = by[byi(G, i, j, k, q)]; A.bf[3] = by[byi(G, i, j + 1, k, q)];
  A.bf[4] = bz[bzi(G, i, j, k, q)]; A.bf[5] = bz[bzi(G, i, j, k + 1, q)];
#pragma unroll
  for (int v = 0; v < 7; ++v) A.c[v] = st[c0 + G.cells * v];
  A.c[7] = 0.5 * (A.bf[0] + A.bf[1]);
  A.c[8] = 0.5 * (A.bf[2] + A.bf[3]);
  A.c[9] = 0.5 * (A.bf[4] + A.bf[5]);
  const Met m = cell_met(G, st, i, j, k, q);
  if (write_b) {
    const double isg = kFast ? 1.0 / m.sqrtg : 0.0;
    aux[a0 + G.cells * GRB_BX] = kFast ? A.c[7] * isg : A.c[7] / m.sqrtg;
    aux[a0 + G.cells * GRB_BY] = kFast ? A.c[8] * isg : A.c[8] / m.sqrtg;
    aux[a0 + G.cells * GRB_BZ] = kFast ? A.c[9] * isg : A.c[9] / m.sqrtg;
  }
  (void)P;
  return m;
}
// After the c2p: c, pr the c2p's output; A the cell's inputs (A.c its
// cons before the c2p).
template <bool kDt, bool kFast>
__device__ __forceinline__ double aux_finish(const DevParams& P, const Geo& G, int i, int j, int k, int64_t q,
                                             double* __restrict__ st, double* __restrict__ aux,
                                             const double* __restrict__ idx, const Met& m, const AuxIn& A,
                                             const double c[10], const double pr[13], const C2POut& o,
                                             const StageBufs& B, const DtArgs& dta) {
  double dtc = INFINITY;
  const double ix[3] = {idx[3 * q], idx[3 * q + 1], idx[3 * q + 2]};
  const int64_t c0 = cvar(G, i, j, k, 0, GRB_N_EVOL_VARS, q);
  const int64_t a0 = cvar(G, i, j, k, 0, GRB_N_AUX_VARS, q);
  if (o.fatal) atomicOr(B.flags, o.fatal);
  aux[a0 + G.cells * GRB_RHO] = pr[GRB_P_RHO];
  aux[a0 + G.cells * GRB_EPS] = pr[GRB_P_EPS];
  aux[a0 + G.cells * GRB_PRESS] = pr[GRB_P_PRESS];
  aux[a0 + G.cells * GRB_TEMP] = pr[GRB_P_TEMP];
  aux[a0 + G.cells * GRB_ENTROPY] = pr[GRB_P_ENT];
  aux[a0 + G.cells * GRB_YE] = pr[GRB_P_YE];
  aux[a0 + G.cells * GRB_ZVECX] = pr[GRB_P_ZX];
  aux[a0 + G.cells * GRB_ZVECY] = pr[GRB_P_ZY];
  aux[a0 + G.cells * GRB_ZVECZ] = pr[GRB_P_ZZ];
  if (o.err & ERR_RESET_DENS) {
    aux[a0 + G.cells * GRB_C2P_DENS_ERR] += A.c[GRB_DENS] - c[0];
    st[c0] = c[0];
  }
  if (o.err & ERR_RESET_STILDE)
    for (int v = 1; v <= 3; ++v) st[c0 + G.cells * v] = c[v];
  if (o.err & ERR_RESET_TAU) st[c0 + G.cells * GRB_TAU] = c[4];
  if (o.err & ERR_RESET_ENTROPY) st[c0 + G.cells * GRB_ENTROPYSTAR] = c[6];
  if (o.err & ERR_RESET_YE) st[c0 + G.cells * GRB_YESTAR] = c[5];
  {
    const uint64_t prev = (uint64_t)aux[a0 + G.cells * GRB_C2P_ERR];
    aux[a0 + G.cells * GRB_C2P_ERR] = (double)(prev | (uint64_t)o.err);
  }
  {
    const double isg = kFast ? 1.0 / m.sqrtg : 0.0;
    const double dv = (A.bf[1] - A.bf[0]) * ix[0] + (A.bf[3] - A.bf[2]) * ix[1] + (A.bf[5] - A.bf[4]) * ix[2];
    aux[a0 + G.cells * GRB_BDIV] = kFast ? dv * isg : dv / m.sqrtg;
  }
  if (P.emf == GRB_EMF_GS) {
    const double cbx = A.c[7], cby = A.c[8], cbz = A.c[9];
    // tuned mode: 1/W of the final primitives from the c2p
    const double W = kFast ? o.W : sqrt(1. + sqs(m.g, pr + GRB_P_ZX));
    double vt[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      vt[a] = (kFast ? m.alp * pr[GRB_P_ZX + a] * o.iW : m.alp * pr[GRB_P_ZX + a] / W) - m.beta[a];
    B.ecenter[eci(G, i, j, k, 0, q)] = cby * vt[2] - cbz * vt[1];
    B.ecenter[eci(G, i, j, k, 1, q)] = -cbx * vt[2] + cbz * vt[0];
    B.ecenter[eci(G, i, j, k, 2, q)] = cbx * vt[1] - cby * vt[0];
  }
  if (kDt && i >= G.g && i < G.nx + G.g && j >= G.g && j < G.ny + G.g && k >= G.g && k < G.nz + G.g)
    dtc = dta.cfl / max_eigenspeed(P.eos, m, pr) * dta.dx[3 * q];
  return dtc;
}

template <bool kDt, bool kFast>
__device__ __forceinline__ double aux_cell(const DevParams& P, const Geo& G, int i, int j, int k, int64_t q,
                                           double* __restrict__ st, const double* __restrict__ bx,
                                           const double* __restrict__ by, const double* __restrict__ bz,
                                           double* __restrict__ aux, const double* __restrict__ idx,
                                           const double* __restrict__ coords, const StageBufs& B,
                                           const DtArgs& dta) {
  AuxIn A;
  const Met m = aux_load(P, G, i, j, k, q, st, bx, by, bz, aux, true, kFast, A);
  double c[10], pr[13];
#pragma unroll
  for (int v = 0; v < 10; ++v) c[v] = A.c[v];
  const double ix[3] = {idx[3 * q], idx[3 * q + 1], idx[3 * q + 2]};
  const Guess none = no_guess();
  const C2POut o =
      c2p<kFast, !kFast>(c, pr, m, P, cell_r(G, coords, ix, i, j, k, q), false, P.alp_bh_thresh, none);
  return aux_finish<kDt, kFast>(P, G, i, j, k, q, st, aux, idx, m, A, c, pr, o, B, dta);
}

// The aux pass with the entropy backups deferred (tuned candidate, for
// blocks where many cells take the backup: a cold atmosphere, magnetised
// regions): k_aux_front runs each cell up to the decision to distrust its
// Kastaun result and finishes the trusted ones; the distrusted ones go to
// a list (up to B.adefer_cap; beyond it a cell finishes in place), and
// k_aux_backup runs the backup and the rest for the listed cells.  Every
// cell's operations and their order are those of aux_cell.
struct AuxDeferred {
  double c[10];
  double pr[13];
  C2PState F;
  int32_t i, j, k;
  int64_t q;
};

// One thread per cell over the box.
template <int MINB = 1, bool kDt = false, bool kFast = false>
__global__ void __launch_bounds__(128, MINB) k_aux(DevParams P, Geo G, Box box, double* __restrict__ st,
                                              const double* __restrict__ bx,
                                              const double* __restrict__ by,
                                              const double* __restrict__ bz,
                                              double* __restrict__ aux,
                                              const double* __restrict__ idx,
                                              const double* __restrict__ coords, StageBufs B,
                                              DtArgs dta = DtArgs{nullptr, 0.0, nullptr}) {
  int i = 0, j = 0, k = 0;
  int64_t q = 0;
  double dtc = INFINITY;
  if (decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q))
    dtc = aux_cell<kDt, kFast>(P, G, i, j, k, q, st, bx, by, bz, aux, idx, coords, B, dta);
  if (kDt) dt_reduce(dtc, dta.out);
}

// Persistent form: one wave of CTAs; each pulls chunks of kAuxChunk tiles of
// 128 cells (tiles numbered block by block, so a chunk stays inside one or
// two blocks) from the device work queue *queue (zeroed before the launch)
// until the box is exhausted.  Per-cell work is the same function.
template <int MINB = 1, bool kDt = false, bool kFast = false>
__global__ void __launch_bounds__(128, MINB) k_aux_queue(DevParams P, Geo G, Box box, double* __restrict__ st,
                                                    const double* __restrict__ bx,
                                                    const double* __restrict__ by,
                                                    const double* __restrict__ bz,
                                                    double* __restrict__ aux,
                                                    const double* __restrict__ idx,
                                                    const double* __restrict__ coords, StageBufs B,
                                                    unsigned long long* __restrict__ queue,
                                                    DtArgs dta = DtArgs{nullptr, 0.0, nullptr}) {
  __shared__ unsigned long long item;
  const int64_t ntiles = (box.count() + 127) / 128;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(queue, (unsigned long long)kAuxChunk);
    __syncthreads();
    const int64_t first = (int64_t)item;
    __syncthreads();
    if (first >= ntiles) break;
    for (int c = 0; c < kAuxChunk; ++c) {
      int i = 0, j = 0, k = 0;
      int64_t q = 0;
      double dtc = INFINITY;
      if (first + c < ntiles && decode(box, (first + c) * 128 + threadIdx.x, i, j, k, q))
        dtc = aux_cell<kDt, kFast>(P, G, i, j, k, q, st, bx, by, bz, aux, idx, coords, B, dta);
      if (kDt) dt_reduce(dtc, dta.out);
    }
  }
}

template <int MINB = 1, bool kDt = false, bool kFast = false>
__global__ void __launch_bounds__(128, MINB) k_aux_front(DevParams P, Geo G, Box box, double* __restrict__ st,
                                                    const double* __restrict__ bx,
                                                    const double* __restrict__ by,
                                                    const double* __restrict__ bz,
                                                    double* __restrict__ aux,
                                                    const double* __restrict__ idx,
                                                    const double* __restrict__ coords, StageBufs B,
                                                    DtArgs dta = DtArgs{nullptr, 0.0, nullptr}) {
  int i = 0, j = 0, k = 0;
  int64_t q = 0;
  double dtc = INFINITY;
  const bool active = decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q);
  AuxIn A;
  Met m;
  double c[10], pr[13];
  C2PState F{};
  double r = 0.0;
  if (active) {
    m = aux_load(P, G, i, j, k, q, st, bx, by, bz, aux, true, kFast, A);
#pragma unroll
    for (int v = 0; v < 10; ++v) c[v] = A.c[v];
    const double ix[3] = {idx[3 * q], idx[3 * q + 1], idx[3 * q + 2]};
    r = cell_r(G, coords, ix, i, j, k, q);
    F = c2p_front<kFast>(c, pr, m, P, false, P.alp_bh_thresh, no_guess());
  }
  const bool later = active && !F.done && F.backup;
  const unsigned mask = __ballot_sync(0xffffffffu, later);
  unsigned long long base = 0;
  const int lane = threadIdx.x & 31;
  if (lane == 0 && mask) base = atomicAdd(B.nadefer, (unsigned long long)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, 0);
  const unsigned long long slot = base + __popc(mask & ((1u << lane) - 1u));
  if (active) {
    if (later && slot < (unsigned long long)B.adefer_cap) {
      AuxDeferred& d = static_cast<AuxDeferred*>(B.adefer)[slot];
#pragma unroll
      for (int v = 0; v < 10; ++v) d.c[v] = c[v];
#pragma unroll
      for (int v = 0; v < 13; ++v) d.pr[v] = pr[v];
      d.F = F;
      d.i = i; d.j = j; d.k = k; d.q = q;
    } else {
      if (!F.done) {
        if (F.backup) c2p_backup(F, c, pr, m, P);
        c2p_back<kFast, !kFast>(F, c, pr, m, P, r);
      }
      dtc = aux_finish<kDt, kFast>(P, G, i, j, k, q, st, aux, idx, m, A, c, pr, F.o, B, dta);
    }
  }
  if (kDt) dt_reduce(dtc, dta.out);
}
template <int MINB = 1, bool kDt = false, bool kFast = false>
__global__ void __launch_bounds__(128, MINB) k_aux_backup(DevParams P, Geo G, double* __restrict__ st,
                                                     const double* __restrict__ bx,
                                                     const double* __restrict__ by,
                                                     const double* __restrict__ bz,
                                                     double* __restrict__ aux,
                                                     const double* __restrict__ idx,
                                                     const double* __restrict__ coords, StageBufs B,
                                                     DtArgs dta = DtArgs{nullptr, 0.0, nullptr}) {
  const int64_t nd = (int64_t)min(*B.nadefer, (unsigned long long)B.adefer_cap);
  double dtc = INFINITY;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nd; e += (int64_t)gridDim.x * blockDim.x) {
    const AuxDeferred& d = static_cast<const AuxDeferred*>(B.adefer)[e];
    const int i = d.i, j = d.j, k = d.k;
    const int64_t q = d.q;
    AuxIn A;
    const Met m = aux_load(P, G, i, j, k, q, st, bx, by, bz, aux, false, kFast, A);
    double c[10], pr[13];
#pragma unroll
    for (int v = 0; v < 10; ++v) c[v] = d.c[v];
#pragma unroll
    for (int v = 0; v < 13; ++v) pr[v] = d.pr[v];
    C2PState F = d.F;
    const double ix[3] = {idx[3 * q], idx[3 * q + 1], idx[3 * q + 2]};
    c2p_backup(F, c, pr, m, P);
    c2p_back<kFast, !kFast>(F, c, pr, m, P, cell_r(G, coords, ix, i, j, k, q));
    dtc = fmin(dtc, aux_finish<kDt, kFast>(P, G, i, j, k, q, st, aux, idx, m, A, c, pr, F.o, B, dta));
  }
  if (kDt) dt_reduce(dtc, dta.out);
}

// reset_c2p_diagnostics (evolve.cpp:154-161)
__global__ void k_reset_diag(Geo G, double* __restrict__ aux) {
  const int64_t n = G.cells * G.nq;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / G.cells, c = t % G.cells;
    aux[c + G.cells * (GRB_C2P_DENS_ERR + (int64_t)GRB_N_AUX_VARS * q)] = 0.0;
    aux[c + G.cells * (GRB_C2P_ERR + (int64_t)GRB_N_AUX_VARS * q)] = 0.0;
  }
}

// linop_apply: a = b*x (+ c*y) elementwise, 2 doubles per thread
__global__ void k_linop(int64_t n, double* __restrict__ a, const double* __restrict__ x,
                        const double* __restrict__ y, double b, double c) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    a[t] = y ? b * x[t] + c * y[t] : b * x[t];
}
// the three-term linop_apply: a = b*x + c*y + d*z elementwise, the sums
// left to right.  a may be any of x, y, z (each element is read before it
// is written by the same thread).
__global__ void k_linop3(int64_t n, double* a, const double* x, const double* y, const double* z, double b,
                         double c, double d) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    a[t] = b * x[t] + c * y[t] + d * z[t];
}


// ---- ghost fill for a brick of same-level blocks ---------------------------
// Periodic axes copy from the neighbouring block (wrapping), the others copy
// the nearest interior cell or face (zero-gradient outflow).  These copies
// compose axis by axis, so each ghost cell (edges and corners included) is
// copied once, directly from the interior cell that the x, y and z sweeps
// of phys_bc / copy kernels would carry into it, with identical values.
// Only the 7 evolved HRSC variables and the three face-B arrays are
// exchanged; the Cowling metric is static.
struct Brick {
  int nbx, nby, nbz;
  int periodic[3];
  int q0;  // first block filled: the launch's blockIdx.y counts from it
};
// One coordinate along one axis: true when x is a ghost index; then (sx,
// off) is the source index and the block offset (-1, 0, +1) along the axis.
// stag: the array is staggered along this axis (faces 0 .. nin + 2g).
__device__ __forceinline__ bool ghost_map(int x, int nin, int g, bool stag, bool periodic, int qc, int nb,
                                          int& sx, int& off) {
  off = 0;
  sx = x;
  if (x < g) {
    if (qc == 0 && !periodic) sx = g;
    else { sx = x + nin; off = -1; }
    return true;
  }
  if (x >= (stag ? nin + g + 1 : nin + g)) {
    if (qc == nb - 1 && !periodic) sx = stag ? nin + g : nin + g - 1;
    else { sx = x - nin; off = 1; }
    return true;
  }
  return false;
}
// Invariant divisors by the x and y extents of the four arrays (cells, x,
// y, z faces), for the per-cell ghost kernel's index decoding.
struct GhostDivs {
  FastDiv x[4], y[4];
};
// One launch for the four arrays: blockIdx.z = 0 the cell-centred HRSC
// variables, 1..3 the face array staggered along blockIdx.z - 1.  One
// thread per cell of one block (blockIdx.y = q - br.q0), x fastest; 32-bit index
// arithmetic (q < 65536, a block's cells < 2^31).
__global__ void __launch_bounds__(256) k_ghost(Geo G, Brick br, GhostDivs D, double* __restrict__ cells,
                                              double* __restrict__ fx, double* __restrict__ fy,
                                              double* __restrict__ fz) {
  const int fd = (int)blockIdx.z - 1;
  const int q = br.q0 + (int)blockIdx.y;
  int n[3] = {G.NX, G.NY, G.NZ};
  if (fd >= 0) n[fd] += 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n[0] * n[1] * n[2]) return;
  // the array's divisors by select (a dynamic index into the parameter
  // would copy it to local memory)
  const FastDiv dx = fd < 0 ? D.x[0] : fd == 0 ? D.x[1] : fd == 1 ? D.x[2] : D.x[3];
  const FastDiv dy = fd < 0 ? D.y[0] : fd == 0 ? D.y[1] : fd == 1 ? D.y[2] : D.y[3];
  double* a = fd < 0 ? cells : fd == 0 ? fx : fd == 1 ? fy : fz;
  const int nin[3] = {G.nx, G.ny, G.nz};
  const int nb[3] = {br.nbx, br.nby, br.nbz};
  const int qyz = q / br.nbx;
  const int qc[3] = {q - qyz * br.nbx, qyz % br.nby, qyz / br.nby};
  const uint32_t u1 = fast_div((uint32_t)t, dx), u2 = fast_div(u1, dy);
  const int c[3] = {(int)((uint32_t)t - u1 * (uint32_t)n[0]), (int)(u1 - u2 * (uint32_t)n[1]), (int)u2};
  int sidx[3], off[3];
  bool ghost = false;
#pragma unroll
  for (int ax = 0; ax < 3; ++ax)
    ghost |= ghost_map(c[ax], nin[ax], G.g, fd == ax, br.periodic[ax] != 0, qc[ax], nb[ax], sidx[ax], off[ax]);
  if (!ghost) return;
  int qs[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) qs[ax] = (qc[ax] + off[ax] + nb[ax]) % nb[ax];
  const int qsrc = qs[0] + br.nbx * (qs[1] + br.nby * qs[2]);
  const int nv = fd < 0 ? GRB_N_HRSC : 1;
  const int64_t vstride = (int64_t)n[0] * n[1] * n[2];
  const int64_t qstride = vstride * (fd < 0 ? GRB_N_EVOL_VARS : 1);
  const int64_t ld = (c[0] + n[0] * (c[1] + n[1] * c[2])) + (int64_t)q * qstride;
  const int64_t ls = (sidx[0] + n[0] * (sidx[1] + n[1] * sidx[2])) + (int64_t)qsrc * qstride;
  double tmp[GRB_N_HRSC];
#pragma unroll
  for (int v = 0; v < GRB_N_HRSC; ++v)
    if (v < nv) tmp[v] = a[ls + v * vstride];
#pragma unroll
  for (int v = 0; v < GRB_N_HRSC; ++v)
    if (v < nv) a[ld + v * vstride] = tmp[v];
}

// The x face array (rows of NX + 1 faces, staggered along x), one thread
// per row of one block (blockIdx.y = q - br.q0): a row whose y and z are interior
// has 2 ngz ghost faces (x < ngz and x > nx + ngz), any other row is ghost
// throughout.  Each thread loads up to 8 of its row's sources before it
// stores them, so the copies of a row overlap; the source of every face is
// the one k_ghost maps it to.
__global__ void __launch_bounds__(128) k_ghost_xfaces(Geo G, Brick br, FastDiv dny, double* __restrict__ fx) {
  const int N0 = G.NX + 1, N1 = G.NY;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= N1 * G.NZ) return;
  const int q = br.q0 + (int)blockIdx.y;
  const int k = (int)fast_div((uint32_t)row, dny), j = row - k * N1;
  const int nb[3] = {br.nbx, br.nby, br.nbz};
  const int qyz = q / br.nbx;
  const int qc[3] = {q - qyz * br.nbx, qyz % br.nby, qyz / br.nby};
  int sy, oy, sz, oz;
  const bool gy = ghost_map(j, G.ny, G.g, false, br.periodic[1] != 0, qc[1], nb[1], sy, oy);
  const bool gz = ghost_map(k, G.nz, G.g, false, br.periodic[2] != 0, qc[2], nb[2], sz, oz);
  const bool full = gy || gz;
  const int cnt = full ? N0 : 2 * G.g;
  const int64_t vst = (int64_t)N0 * N1 * G.NZ;
  const int qyzs = (qc[1] + oy + nb[1]) % nb[1] + br.nby * ((qc[2] + oz + nb[2]) % nb[2]);
  const int64_t drow = (int64_t)q * vst + (int64_t)N0 * (j + (int64_t)N1 * k);
  const int64_t srow = (int64_t)N0 * (sy + (int64_t)N1 * sz);
  for (int m0 = 0; m0 < cnt; m0 += 8) {
    double v[8];
    int xs[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int m = m0 + u;
      xs[u] = -1;
      if (m < cnt) {
        const int x = full ? m : (m < G.g ? m : G.nx + G.g + 1 + (m - G.g));
        int sx, ox;
        ghost_map(x, G.nx, G.g, true, br.periodic[0] != 0, qc[0], nb[0], sx, ox);
        const int qs = (qc[0] + ox + nb[0]) % nb[0] + br.nbx * qyzs;
        v[u] = fx[(int64_t)qs * vst + srow + sx];
        xs[u] = x;
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (xs[u] >= 0) fx[drow + xs[u]] = v[u];
  }
}

// The same fill in runs of 4 cells along x, for ghost width 4 and interior
// extents along x that are multiples of 4 (so runs never straddle the
// interior's edge) on arrays whose rows are 4-aligned (not staggered along
// x): blockIdx.z = 0 the cell-centred HRSC variables, 1, 2 the face arrays
// staggered along y, z; runs + off[a] lists array a's ghost runs, packed
// r | j << 8 | k << 16 (x in [4r, 4r + 4) of row (j, k)).  Each thread
// copies one run with 16-byte loads and stores: the matching run of its
// source row, or one cell repeated where zero-gradient applies along x.
__global__ void __launch_bounds__(128) k_ghost_runs(Geo G, Brick br, const uint32_t* __restrict__ runs,
                                                   int3 off, int3 cnt, double* __restrict__ cells,
                                                   double* __restrict__ fy, double* __restrict__ fz) {
  const int arr = blockIdx.z;
  const int len = arr == 0 ? cnt.x : arr == 1 ? cnt.y : cnt.z;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= len) return;
  const uint32_t e = __ldg(runs + (arr == 0 ? off.x : arr == 1 ? off.y : off.z) + t);
  const int r = (int)(e & 0xffu), c1 = (int)((e >> 8) & 0xffu), c2 = (int)(e >> 16);
  const int fd = arr == 0 ? -1 : arr;  // staggered axis (1: y, 2: z)
  int n[3] = {G.NX, G.NY, G.NZ};
  if (fd > 0) n[fd] += 1;
  double* a = arr == 0 ? cells : arr == 1 ? fy : fz;
  const int q = br.q0 + (int)blockIdx.y;
  const int nin[3] = {G.nx, G.ny, G.nz};
  const int nb[3] = {br.nbx, br.nby, br.nbz};
  const int qyz = q / br.nbx;
  const int qc[3] = {q - qyz * br.nbx, qyz % br.nby, qyz / br.nby};
  int sx, sy, sz, ox, oy, oz;
  const int x0 = 4 * r;
  ghost_map(x0, nin[0], G.g, false, br.periodic[0] != 0, qc[0], nb[0], sx, ox);
  ghost_map(c1, nin[1], G.g, fd == 1, br.periodic[1] != 0, qc[1], nb[1], sy, oy);
  ghost_map(c2, nin[2], G.g, fd == 2, br.periodic[2] != 0, qc[2], nb[2], sz, oz);
  // along x: a ghost run whose first cell maps to the boundary cell is a
  // zero-gradient run (every cell copies that one cell); otherwise the
  // run maps to the run at the same offset
  int sxe;
  int oxe;
  ghost_map(x0 + 3, nin[0], G.g, false, br.periodic[0] != 0, qc[0], nb[0], sxe, oxe);
  const bool bcast = sxe == sx;
  const int qs = (qc[0] + ox + nb[0]) % nb[0] +
                 br.nbx * ((qc[1] + oy + nb[1]) % nb[1] + br.nby * ((qc[2] + oz + nb[2]) % nb[2]));
  const int nv = arr == 0 ? GRB_N_HRSC : 1;
  const int64_t vstride = (int64_t)n[0] * n[1] * n[2];
  const int64_t qstride = vstride * (arr == 0 ? GRB_N_EVOL_VARS : 1);
  const int64_t ld = (x0 + n[0] * (c1 + n[1] * c2)) + (int64_t)q * qstride;
  const int64_t ls = (sx + n[0] * (sy + n[1] * sz)) + (int64_t)qs * qstride;
  for (int v = 0; v < nv; ++v) {
    double2* d = reinterpret_cast<double2*>(a + ld + v * vstride);
    if (bcast) {
      const double x = a[ls + v * vstride];
      d[0] = make_double2(x, x);
      d[1] = make_double2(x, x);
    } else {
      const double2* sp = reinterpret_cast<const double2*>(a + ls + v * vstride);
      const double2 u0 = sp[0], u1 = sp[1];
      d[0] = u0;
      d[1] = u1;
    }
  }
}

// Interior of one array between the device layout and a packed interior
// layout [nq][nv][n2][n1][n0] (no ghosts): box = the interior (lo = g),
// x (nv variables x nq blocks) folded into the box's block index;
// qdev: block stride of the device array; to_packed selects the direction.
__global__ void __launch_bounds__(256) k_pack_interior(Box box, int nv, FastDiv dnv, int N0, int N1,
                                                       int64_t vstride, int64_t qdev, bool to_packed,
                                                       double* __restrict__ dev, double* __restrict__ packed) {
  int i, j, k;
  int64_t qv;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (!decode(box, t, i, j, k, qv)) return;
  const uint32_t q = fast_div((uint32_t)qv, dnv);
  const uint32_t v = (uint32_t)qv - q * (uint32_t)nv;
  const int64_t o = (int64_t)q * qdev + (int64_t)v * vstride + ((int64_t)k * N1 + j) * N0 + i;
  if (to_packed) packed[t] = dev[o];
  else dev[o] = packed[t];
}

// Interior rows of one array between device memory and mapped host
// memory.  box: rows at full x extent (x = 0 .. N0-1) of the interior y and
// z ranges, x (nv variables x nq blocks) folded into the box's block index,
// so each (variable, block, z) plane is one contiguous run of memory that
// the bus moves in whole lines; dst and src are LayoutLeft arrays with the
// same cell layout, variable stride vstride and block strides qdst, qsrc
// (doubles).  Only x in [xlo, xhi) is stored (the loads cover the whole
// row, volatile so that they are not narrowed to the stored part).
__global__ void __launch_bounds__(256) k_copy_rows(Box box, int xlo, int xhi, int nv, FastDiv dnv, int N0,
                                                    int N1, int64_t vstride, int64_t qdst, int64_t qsrc,
                                                    double* dst, const double* src) {
  int i, j, k;
  int64_t qv;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, qv)) return;
  const uint32_t q = fast_div((uint32_t)qv, dnv);
  const uint32_t v = (uint32_t)qv - q * (uint32_t)nv;
  const int64_t o = (int64_t)v * vstride + ((int64_t)k * N1 + j) * N0 + i;
  const double x = *reinterpret_cast<const volatile double*>(src + o + (int64_t)q * qsrc);
  if (i >= xlo && i < xhi) dst[o + (int64_t)q * qdst] = x;
}

}  // namespace grb
