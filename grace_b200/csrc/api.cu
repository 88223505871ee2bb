// C ABI of the B200 Cowling GRMHD stage library (include/grace_b200.h).
//
// Host orchestration only: validates arguments, owns the scratch arrays
// (the reference keeps them in the variable_list singleton,
// src/data_structures/variables.cpp:100-211), and launches the kernels of
// stage_kernels.cuh / fused_kernels.cuh on the caller's stream.  No call
// here synchronises the stream except grb_get_status and grb_reserve.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <tuple>
#include <utility>
#include <new>
#include <vector>

#include "grace_b200.h"
#include "amr.cuh"
#include "outflow.cuh"
#include "flux_tma.cuh"
#include "reflux.cuh"
#include "mlp.cuh"
#include "stage_kernels.cuh"

using namespace grb;

struct grb_handle {
  grb_params p;
  DevParams dp;
  Geo geo;
  bool reserved = false;
  int64_t cap_f = 0, cap_c = 0;  // capacities (elements) of face-grid / cell scratch
  StageBufs B{};
  uint32_t* d_flags = nullptr;
  unsigned long long* d_counters = nullptr;
  int last_error = GRB_OK;
  int64_t launches = 0;  // kernels launched through this handle
  int mode = GRB_MODE_PLAIN;
  // tuned mode: register-cap variant per kernel family (index into kMinB)
  int var_flux = 0, var_flag = 0, var_update = 0, var_aux = 0;
  bool autotuned = false;
  float tune_ms[4][3] = {};
  // optional per-kernel-kind timing with events on the launching stream
  bool timing = false;
  struct Mark { int kind; cudaEvent_t a, b; };
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> pool;
  double kind_ms[GRB_KIND_COUNT] = {0};
  int64_t kind_n[GRB_KIND_COUNT] = {0};
  // learned c2p bracket: FP32 parameter block on the device
  float* d_mlp = nullptr;
  MlpSmem* d_mlp_pack = nullptr;  // shared-memory image of the network
  unsigned long long* d_queue = nullptr;  // work-queue counters: [0] aux pass, [1] FOFC flag, [2] flux, [3] update
  double* d_metder = nullptr;             // static-metric cache (grb_set_static_metric)
  size_t metder_bytes = 0;
  int metder_key[4] = {0, 0, 0, 0};       // nx, ny, nz, ngz it was built for
  int64_t metder_nq = 0;                  // blocks it covers
  const double* metder_idx = nullptr;     // the spacings it was built with
  double* d_stage_io = nullptr;           // staging of grb_copy_evolved_packed
  size_t stage_io_bytes = 0;
  uint32_t* d_ghostruns = nullptr;        // ghost runs of k_ghost_runs, 3 arrays
  int ghost_off[3] = {0, 0, 0}, ghost_cnt[3] = {0, 0, 0};
  int ghost_key[4] = {0, 0, 0, 0};        // nx, ny, nz, ngz they were built for
  uint32_t* d_auxlist = nullptr;          // cells of the tuned aux pass in one block
  uint32_t auxlist_n = 0;
  int auxlist_key[4] = {0, 0, 0, 0};      // nx, ny, nz, ngz it was built for
  float tune_aux_queue_ms = 0.f;
  float tune_aux_defer_ms = 0.f;
  float tune_flag_queue_ms = 0.f;
  float tune_flux_queue_ms = 0.f;
  float tune_update_queue_ms = 0.f;
  const double* res_idx = nullptr;        // spacings of the grid passed to grb_reserve
  bool mlp_ready = false;
  uint32_t fcap_alloc = 0;  // entries allocated for the compacted FOFC face list
  // the tuned batch c2p's deferred entropy backups: records and their count
  C2PDeferred* d_defer = nullptr;
  int64_t defer_cap = 0;
  unsigned long long* d_ndefer = nullptr;
  // refluxing (grb_set_reflux): the caller's descriptor lists and the edge
  // accumulation buffers
  bool reflux = false;
  bool reflux_flux_same = false;
  RefluxDev rf{};
  double* d_refacc = nullptr;
  size_t refacc_bytes = 0;
};

namespace {

int fail(grb_handle* h, int code) {
  if (h) h->last_error = code;
  return code;
}
#define CK(call)                                       \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return fail(h, GRB_ERR_CUDA); \
  } while (0)

DevParams to_dev(const grb_params& p) {
  DevParams d{};
  DevEos& e = d.eos;
  e.kind = p.eos.kind;
  e.eps_max = p.eos.eps_max;
  if (p.eos.kind == GRB_EOS_IDEAL_GAS) {
    // ideal_gas_eos.hh:56-86
    e.rhomax = 1e100; e.rhomin = 1e-100; e.tempmax = 1e100; e.yemax = 1e100;
    e.h_min = 1. + 1e-15;
    e.gm1 = p.eos.gamma - 1.;
    e.g = e.gm1 + 1.;
    e.ggm1 = e.g * e.gm1;
    e.igm1 = 1.0 / e.gm1;
    e.ent_min = (p.eos.temp_atm > 0.0) ? (p.eos.temp_atm / e.gm1) : 1e-100;
    e.n = 1;
  } else {
    // hybrid_eos.hh:62-75 with the polytrope bounds of eos_storage.cpp:143-150
    e.rhomax = 1e10; e.rhomin = 1e-100; e.tempmax = 1e99; e.yemax = 1e99;
    e.h_min = 1. + 1e-10;
    e.gthm1 = p.eos.gamma_th - 1.;
    e.entropy_min = p.eos.entropy_min;
    e.n = p.eos.n_pieces;
    for (int i = 0; i < GRB_MAX_PIECES; ++i) {
      e.K[i] = p.eos.pw_kappa[i]; e.G[i] = p.eos.pw_gamma[i];
      e.R[i] = p.eos.pw_rho[i]; e.E[i] = p.eos.pw_eps[i];
    }
  }
  e.ih0 = 1.0 / e.h_min;
  d.rho_fl = p.rho_fl; d.ye_fl = p.ye_fl; d.temp_fl = p.temp_fl; d.atmo_tol = p.atmo_tol;
  d.excise_by_radius = p.excise_by_radius; d.r_ex = p.r_ex; d.alp_ex = p.alp_ex;
  d.tol = p.c2p_tol; d.max_w = p.max_w; d.max_sigma = p.max_sigma;
  d.beta_fallback = p.beta_fallback; d.alp_bh_thresh = p.alp_bh_thresh;
  d.use_ent_backup = p.use_ent_backup;
  d.rusanov_c_limit = p.rusanov_use_c_limit;
  d.fofc = p.fofc_enable; d.dmp_enable = p.dmp_enable; d.dmp_M = p.dmp_M;
  d.recon = p.recon; d.riemann = p.riemann; d.emf = p.emf;
  return d;
}

bool valid_params(const grb_params* p) {
  if (!p) return false;
  if (p->eos.kind != GRB_EOS_IDEAL_GAS && p->eos.kind != GRB_EOS_HYBRID_PWPOLY) return false;
  if (p->eos.kind == GRB_EOS_HYBRID_PWPOLY && (p->eos.n_pieces < 1 || p->eos.n_pieces > GRB_MAX_PIECES)) return false;
  if (p->recon < GRB_RECON_WENOZ || p->recon > GRB_RECON_DONOR) return false;
  if (p->riemann != GRB_RIEMANN_HLL && p->riemann != GRB_RIEMANN_LLF) return false;
  if (p->emf != GRB_EMF_GS && p->emf != GRB_EMF_UCT) return false;
  if (p->ranges != GRB_RANGES_FULL && p->ranges != GRB_RANGES_NEXT_STAGE) return false;
  // flag_fofc_cells asserts on UCT (evolve.cpp:479-481)
  if (p->fofc_enable && p->emf == GRB_EMF_UCT) return false;
  return true;
}

bool same_geo(const Geo& a, const grb_grid* g) {
  return a.nx == g->nx && a.ny == g->ny && a.nz == g->nz && a.g == g->ngz && a.nq == g->nq;
}

int check_grid(grb_handle* h, const grb_grid* g) {
  if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->nq < 1 || !g->idx) return GRB_ERR_INVALID;
  if (g->ngz < 4) return GRB_ERR_INVALID;  // WENO-Z + FOFC need ngz >= 4 (evolve.cpp:476-478)
  if (!h->reserved) return GRB_ERR_NOT_RESERVED;
  const Geo t = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  if (t.fcells * t.nq > h->cap_f || t.cells * t.nq > h->cap_c) return GRB_ERR_NOT_RESERVED;
  if (h->p.excise_by_radius && !g->coords) return GRB_ERR_INVALID;
  return GRB_OK;
}

inline Box box(int l0, int l1, int l2, int n0, int n1, int n2, int64_t nq) {
  Box b;
  b.lo[0] = l0; b.lo[1] = l1; b.lo[2] = l2;
  b.n[0] = n0; b.n[1] = n1; b.n[2] = n2;
  b.nq = nq;
  for (int a = 0; a < 3; ++a) b.dv[a] = make_fastdiv((uint32_t)std::max(b.n[a], 1));
  return b;
}
inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

cudaEvent_t take_event(grb_handle* h) {
  if (!h->pool.empty()) {
    cudaEvent_t e = h->pool.back();
    h->pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
// Brackets the launches between begin() and end() with a pair of events
// when timing is on; a no-op otherwise.
struct KScope {
  grb_handle* h;
  cudaStream_t s;
  int kind;
  cudaEvent_t a = nullptr;
  KScope(grb_handle* h_, cudaStream_t s_, int k) : h(h_), s(s_), kind(k) {
    if (h->timing) { a = take_event(h); cudaEventRecord(a, s); }
  }
  ~KScope() {
    if (h->timing) {
      cudaEvent_t b = take_event(h);
      cudaEventRecord(b, s);
      h->marks.push_back({kind, a, b});
    }
  }
};


// ---- tuned-mode variant dispatch (launch-bounds register caps) -------------
// kMinB[v]: minimum resident CTAs of 128 threads per SM requested from the
// compiler; 1 leaves the register count free, 4 caps it at 128, 5 at 102.
constexpr int kMaxDevices = 64;  // device ordinals tracked by per-device launch set-up
constexpr int kMinB[3] = {1, 4, 5};
// The c2p-bearing kernels (FOFC flag, aux pass) in their tuned forms: 3, 4,
// 5 (uncapped they need 180-250 registers, two CTAs per SM at most).
constexpr int kMinBC2p[3] = {3, 4, 5};
// The update kernel that reads the static-metric cache: 1, 3, 4.
constexpr int kMinBCached[3] = {1, 3, 4};
constexpr int kNumVar = 3;

// ---- TMA-staged flux kernel: tensor maps and tile geometry ----------------
// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}
// Tile of direction dir for the face box b (one block's face ranges), for
// CTAs of nt threads.
FluxTile flux_tile(int dir, const Geo& G, const Box& b, int nt) {
  FluxTile T;
  for (int a = 0; a < 3; ++a) { T.lo[a] = b.lo[a]; T.n[a] = b.n[a]; }
  T.R = nt / T.n[0];
  T.BY = dir == 0 ? T.R : dir == 1 ? T.R + 5 : 1;
  T.BZ = dir == 2 ? T.R + 5 : 1;
  (void)G;
  return T;
}
// Tensor map over a LayoutLeft (NX, NY, NZ, nv, nq) double array, box
// (NX, BY, BZ, 10 variables, 1 block).  False when the array or the box does
// not meet the copy engine's rules (then the global-load kernel runs).
bool make_tmap(CUtensorMap* tm, const double* base, const Geo& G, int nv, int64_t nq, const FluxTile& T) {
  auto enc = tma_encoder();
  if (!enc || ((uintptr_t)base & 15) || (G.NX * sizeof(double)) % 16 || G.NX > 256 || T.BY > 256 ||
      T.BZ > 256 || T.R < 1)
    return false;
  const cuuint64_t dims[5] = {(cuuint64_t)G.NX, (cuuint64_t)G.NY, (cuuint64_t)G.NZ, (cuuint64_t)nv,
                              (cuuint64_t)nq};
  const cuuint64_t strides[4] = {(cuuint64_t)G.NX * 8, (cuuint64_t)G.NX * G.NY * 8, (cuuint64_t)G.cells * 8,
                                 (cuuint64_t)G.cells * nv * 8};
  const cuuint32_t box[5] = {(cuuint32_t)G.NX, (cuuint32_t)T.BY, (cuuint32_t)T.BZ, 10u, 1u};
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
template <int dir, int MINB, int NT = 128>
bool launch_flux_tma(cudaStream_t s, const DevParams& P, const Geo& G, const Box& b, const double* st,
                     const double* aux, const double* bf, const StageBufs& B) {
  const FluxTile T = flux_tile(dir, G, b, NT);
  if (T.n[0] > NT || b.nq > 65535) return false;
  CUtensorMap ta, tm;
  if (!make_tmap(&ta, aux, G, GRB_N_AUX_VARS, b.nq, T) || !make_tmap(&tm, st, G, GRB_N_EVOL_VARS, b.nq, T))
    return false;
  const size_t smem = flux_tile_smem(G, T);
  // the attribute is per device: remember what each device ordinal got
  static size_t attr[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return false;
  if (smem > attr[dev]) {
    if (cudaFuncSetAttribute(k_flux_tma<dir, MINB, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return false;
    attr[dev] = smem;
  }
  const int nrow = dir == 2 ? T.n[2] : T.n[1];
  const int nother = dir == 2 ? T.n[1] : T.n[2];
  const dim3 grid((unsigned)((nrow + T.R - 1) / T.R), (unsigned)nother, (unsigned)b.nq);
  k_flux_tma<dir, MINB, NT><<<grid, NT, smem, s>>>(P, G, T, ta, tm, bf, B);
  return true;
}

// One wave of a persistent one-thread-per-item kernel (occupancy x SMs CTAs
// of 128 threads, per device ordinal and kernel), after zeroing its queue
// counter on the stream; the kernel's last argument is the counter.
template <class... KArgs, class... Args>
void launch_item_queue(cudaStream_t s, void (*kernel)(KArgs...), Args&&... args) {
  static int grids[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int grid = dev >= 0 && dev < kMaxDevices ? grids[dev] : 0;
  if (grid == 0) {
    int sms = 0, occ = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, 128, 0);
    grid = (sms > 0 ? sms : 1) * (occ > 0 ? occ : 1);
    if (dev >= 0 && dev < kMaxDevices) grids[dev] = grid;
  }
  unsigned long long* queue = std::get<sizeof...(Args) - 1>(std::forward_as_tuple(args...));
  cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
  kernel<<<grid, 128, 0, s>>>(std::forward<Args>(args)...);
}

// The TMA-staged flux as one wave of persistent CTAs pulling tiles from the
// queue counter (zeroed first on the stream); false when the tile does not
// fit (the caller then launches another form).
template <int dir, int MINB, int NT = 128>
bool launch_flux_tma_queue(cudaStream_t s, const DevParams& P, const Geo& G, const Box& b, const double* st,
                           const double* aux, const double* bf, const StageBufs& B, unsigned long long* queue) {
  const FluxTile T = flux_tile(dir, G, b, NT);
  if (T.n[0] > NT || !queue) return false;
  CUtensorMap ta, tm;
  if (!make_tmap(&ta, aux, G, GRB_N_AUX_VARS, b.nq, T) || !make_tmap(&tm, st, G, GRB_N_EVOL_VARS, b.nq, T))
    return false;
  const size_t smem = flux_tile_smem(G, T);
  static size_t attr[kMaxDevices] = {};
  static int occ_for[kMaxDevices] = {};
  static size_t occ_smem[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return false;
  if (smem > attr[dev]) {
    if (cudaFuncSetAttribute(k_flux_tma_queue<dir, MINB, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return false;
    attr[dev] = smem;
  }
  if (occ_smem[dev] != smem) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_flux_tma_queue<dir, MINB, NT>, NT, smem) !=
            cudaSuccess || occ < 1)
      return false;
    occ_for[dev] = occ;
    occ_smem[dev] = smem;
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int nrow = dir == 2 ? T.n[2] : T.n[1];
  const int nother = dir == 2 ? T.n[1] : T.n[2];
  const int ntx = (nrow + T.R - 1) / T.R;
  if (cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s) != cudaSuccess) return false;
  k_flux_tma_queue<dir, MINB, NT><<<(unsigned)(std::max(sms, 1) * occ_for[dev]), NT, smem, s>>>(
      P, G, T, ta, tm, bf, B, queue, ntx, nother);
  return true;
}

// Flux candidates of the tuned mode (tile shapes and register caps): the
// global-load kernel at 4 CTAs/SM of 128 threads, the TMA-staged kernel
// with 128-thread tiles at 4 CTAs/SM, and with 256-thread tiles (twice the
// rows per tile, less halo re-read along y and z) at 2 CTAs/SM (the same
// register budget).  Reported by grb_get_tuning as min CTAs/SM, plus 100
// for the TMA-staged kernel.
constexpr int kFluxMinB[3] = {4, 4, 2};
constexpr bool kFluxTma[3] = {false, true, true};

// Candidates 3..5: the same three as persistent launches pulling work from
// the queue counter (given): the global-load kernel's 128-face tiles, or
// the TMA-staged kernel's tiles.
template <int dir>
void launch_flux_tuned(int v, unsigned nb, cudaStream_t s, const DevParams& P, const Geo& G, const Box& b,
                       const double* st, const double* aux, const double* bf, const StageBufs& B,
                       unsigned long long* queue = nullptr) {
  if (v >= 3 && queue) {
    if (v == 4 && launch_flux_tma_queue<dir, 4>(s, P, G, b, st, aux, bf, B, queue)) return;
    if (v == 5 && launch_flux_tma_queue<dir, 2, 256>(s, P, G, b, st, aux, bf, B, queue)) return;
    launch_item_queue(s, k_flux_queue<dir, true, 4>, P, G, b, st, aux, bf, B, queue);
    return;
  }
  if (v >= 3) v -= 3;
  if (v == 1 && launch_flux_tma<dir, 4>(s, P, G, b, st, aux, bf, B)) return;
  if (v == 2 && launch_flux_tma<dir, 2, 256>(s, P, G, b, st, aux, bf, B)) return;
  k_flux<dir, true, 4><<<nb, 128, 0, s>>>(P, G, b, st, aux, bf, B);
}
// One wave of the persistent FOFC flag kernel (per device ordinal), after
// zeroing its queue counter.
template <int MINB>
void launch_flag_queue(cudaStream_t s, const DevParams& P, const Geo& G, const Box& b, double dt, double dtfact,
                       const double* ns, const double* os, const double* bx, const double* by, const double* bz,
                       const double* idx, const double* crd, const StageBufs& B, unsigned long long* queue) {
  static int grids[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int grid = 0;
  if (dev >= 0 && dev < kMaxDevices) grid = grids[dev];
  if (grid == 0) {
    int sms = 0, occ = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fofc_flag_queue<MINB, true>, 128, 0);
    grid = (sms > 0 ? sms : 1) * (occ > 0 ? occ : 1);
    if (dev >= 0 && dev < kMaxDevices) grids[dev] = grid;
  }
  cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
  k_fofc_flag_queue<MINB, true><<<grid, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, bx, by, bz, idx, crd, B, queue);
}
// Flag candidates: 0..2 one thread per cell at 3, 4, 5 CTAs/SM; 3..5 the
// persistent work-queue form at the same caps (given the queue counter).
void launch_flag_tuned(int v, unsigned nb, cudaStream_t s, const DevParams& P, const Geo& G, const Box& b,
                       double dt, double dtfact, const double* ns, const double* os, const double* bx,
                       const double* by, const double* bz, const double* idx, const double* crd,
                       const StageBufs& B, unsigned long long* queue = nullptr) {
  if (v >= 3 && queue) {
    if (v == 4) launch_flag_queue<4>(s, P, G, b, dt, dtfact, ns, os, bx, by, bz, idx, crd, B, queue);
    else if (v == 5) launch_flag_queue<5>(s, P, G, b, dt, dtfact, ns, os, bx, by, bz, idx, crd, B, queue);
    else launch_flag_queue<3>(s, P, G, b, dt, dtfact, ns, os, bx, by, bz, idx, crd, B, queue);
    return;
  }
  if (v >= 3) v -= 3;
  if (v == 1) k_fofc_flag<4, true><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, bx, by, bz, idx, crd, B);
  else if (v == 2) k_fofc_flag<5, true><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, bx, by, bz, idx, crd, B);
  else k_fofc_flag<3, true><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, bx, by, bz, idx, crd, B);
}
// Update candidates: 0..2 at 1, 4, 5 CTAs/SM; with the static-metric
// cache md the kernel that reads it (capped at 1, 3, 4 CTAs/SM).
// 3..5: the same caps as persistent launches pulling 128-cell tiles from the
// queue counter (given).
void launch_update_tuned(int v, unsigned nb, cudaStream_t s, const DevParams& P, const Geo& G, const Box& b,
                         double dt, double dtfact, double* ns, const double* os, const double* aux,
                         const double* idx, const StageBufs& B, const double* md = nullptr,
                         unsigned long long* queue = nullptr) {
  if (v >= 3 && queue) {
    const int m = v - 3;
    if (md) {
      if (m == 1) launch_item_queue(s, k_update_queue<3, true>, P, G, b, dt, dtfact, ns, os, aux, idx, B, md, queue);
      else if (m == 2) launch_item_queue(s, k_update_queue<4, true>, P, G, b, dt, dtfact, ns, os, aux, idx, B, md, queue);
      else launch_item_queue(s, k_update_queue<1, true>, P, G, b, dt, dtfact, ns, os, aux, idx, B, md, queue);
    } else {
      const double* none = nullptr;
      if (m == 1) launch_item_queue(s, k_update_queue<4, false>, P, G, b, dt, dtfact, ns, os, aux, idx, B, none, queue);
      else if (m == 2) launch_item_queue(s, k_update_queue<5, false>, P, G, b, dt, dtfact, ns, os, aux, idx, B, none, queue);
      else launch_item_queue(s, k_update_queue<1, false>, P, G, b, dt, dtfact, ns, os, aux, idx, B, none, queue);
    }
    return;
  }
  if (v >= 3) v -= 3;
  if (md) {
    static_assert(kMinBCached[1] == 3 && kMinBCached[2] == 4, "update candidates");
    if (v == 1) k_update<3, true><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, aux, idx, B, md);
    else if (v == 2) k_update<4, true><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, aux, idx, B, md);
    else k_update<1, true><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, aux, idx, B, md);
    return;
  }
  if (v == 1) k_update<4><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, aux, idx, B);
  else if (v == 2) k_update<5><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, aux, idx, B);
  else k_update<1><<<nb, 128, 0, s>>>(P, G, b, dt, dtfact, ns, os, aux, idx, B);
}
// Work-queue aux pass: one wave of CTAs (occupancy x SMs) pulling tiles.
template <int MINB, bool kDt>
void launch_aux_queue(cudaStream_t s, const DevParams& P, const Geo& G, const Box& b, double* st, const double* bx,
                      const double* by, const double* bz, double* aux, const double* idx, const double* crd,
                      const StageBufs& B, unsigned long long* queue, const DtArgs& dta) {
  // one wave of CTAs, per device ordinal
  static int grids[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int grid = 0;
  if (dev >= 0 && dev < kMaxDevices) grid = grids[dev];
  if (grid == 0) {
    int sms = 0, occ = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_aux_queue<MINB, kDt, true>, 128, 0);
    grid = (sms > 0 ? sms : 1) * (occ > 0 ? occ : 1);
    if (dev >= 0 && dev < kMaxDevices) grids[dev] = grid;
  }
  cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
  k_aux_queue<MINB, kDt, true><<<grid, 128, 0, s>>>(P, G, b, st, bx, by, bz, aux, idx, crd, B, queue, dta);
}

// The aux pass with the entropy backups deferred to a second kernel over
// the listed cells (when the handle holds the list).
template <int MINB, bool kDt>
void launch_aux_deferred(unsigned nb, cudaStream_t s, const DevParams& P, const Geo& G, const Box& b, double* st,
                         const double* bx, const double* by, const double* bz, double* aux, const double* idx,
                         const double* crd, const StageBufs& B, const DtArgs& dta) {
  cudaMemsetAsync(B.nadefer, 0, sizeof(unsigned long long), s);
  k_aux_front<MINB, kDt, true><<<nb, 128, 0, s>>>(P, G, b, st, bx, by, bz, aux, idx, crd, B, dta);
  k_aux_backup<MINB, kDt, true><<<std::min(nb, 148u * 8u), 128, 0, s>>>(P, G, st, bx, by, bz, aux, idx, crd, B,
                                                                       dta);
}

// Aux candidates: 0..2 one thread per cell at kMinBC2p[v] CTAs/SM; 3..5
// the work-queue form at kMinBC2p[v - 3]; 6..8 the deferred-backup form at
// kMinBC2p[v - 6].
void launch_aux_tuned(int v, unsigned nb, cudaStream_t s, const DevParams& P, const Geo& G, const Box& b,
                      double* st, const double* bx, const double* by, const double* bz, double* aux,
                      const double* idx, const double* crd, const StageBufs& B,
                      const DtArgs* dta = nullptr, unsigned long long* queue = nullptr) {
  if (v >= 6 && B.adefer) {
    const DtArgs d0{nullptr, 0.0, nullptr};
    const int m = v - 6;
    if (dta) {
      if (m == 1) launch_aux_deferred<4, true>(nb, s, P, G, b, st, bx, by, bz, aux, idx, crd, B, *dta);
      else if (m == 2) launch_aux_deferred<5, true>(nb, s, P, G, b, st, bx, by, bz, aux, idx, crd, B, *dta);
      else launch_aux_deferred<3, true>(nb, s, P, G, b, st, bx, by, bz, aux, idx, crd, B, *dta);
    } else {
      if (m == 1) launch_aux_deferred<4, false>(nb, s, P, G, b, st, bx, by, bz, aux, idx, crd, B, d0);
      else if (m == 2) launch_aux_deferred<5, false>(nb, s, P, G, b, st, bx, by, bz, aux, idx, crd, B, d0);
      else launch_aux_deferred<3, false>(nb, s, P, G, b, st, bx, by, bz, aux, idx, crd, B, d0);
    }
    return;
  }
  if (v >= 6) v -= 6;
  if (v >= 3 && queue) {
    const DtArgs d0{nullptr, 0.0, nullptr};
    const int m = v - 3;
    if (dta) {
      if (m == 1) launch_aux_queue<4, true>(s, P, G, b, st, bx, by, bz, aux, idx, crd, B, queue, *dta);
      else if (m == 2) launch_aux_queue<5, true>(s, P, G, b, st, bx, by, bz, aux, idx, crd, B, queue, *dta);
      else launch_aux_queue<3, true>(s, P, G, b, st, bx, by, bz, aux, idx, crd, B, queue, *dta);
    } else {
      if (m == 1) launch_aux_queue<4, false>(s, P, G, b, st, bx, by, bz, aux, idx, crd, B, queue, d0);
      else if (m == 2) launch_aux_queue<5, false>(s, P, G, b, st, bx, by, bz, aux, idx, crd, B, queue, d0);
      else launch_aux_queue<3, false>(s, P, G, b, st, bx, by, bz, aux, idx, crd, B, queue, d0);
    }
    return;
  }
  if (v >= 3) v -= 3;
  if (dta) {
    if (v == 1) k_aux<4, true, true><<<nb, 128, 0, s>>>(P, G, b, st, bx, by, bz, aux, idx, crd, B, *dta);
    else if (v == 2) k_aux<5, true, true><<<nb, 128, 0, s>>>(P, G, b, st, bx, by, bz, aux, idx, crd, B, *dta);
    else k_aux<3, true, true><<<nb, 128, 0, s>>>(P, G, b, st, bx, by, bz, aux, idx, crd, B, *dta);
    return;
  }
  if (v == 1) k_aux<4, false, true><<<nb, 128, 0, s>>>(P, G, b, st, bx, by, bz, aux, idx, crd, B);
  else if (v == 2) k_aux<5, false, true><<<nb, 128, 0, s>>>(P, G, b, st, bx, by, bz, aux, idx, crd, B);
  else k_aux<3, false, true><<<nb, 128, 0, s>>>(P, G, b, st, bx, by, bz, aux, idx, crd, B);
}

// A = b X (+ c Y) on the planes z in [zlo, zlo + nz) and rows y in [ylo,
// ylo + ny) of a LayoutLeft array (N0, N1, N2, nv_total, nq) at full x
// extent, for nv variables: each plane's rows are one contiguous span, so
// every warp reads and writes consecutive doubles.  grid (span / 256,
// nz * nv, nq); no 64-bit index division.
struct LinBox {
  int N0, N1, N2;
  int ylo, ny, zlo, nz;
  int64_t vstride, qstride;
};
__global__ void __launch_bounds__(256) k_linop_box(LinBox L, int nv, double* __restrict__ a,
                                                   const double* __restrict__ x, const double* __restrict__ y,
                                                   double b, double c) {
  const int span = L.ny * L.N0;
  const int e = blockIdx.x * 256 + threadIdx.x;
  if (e >= span) return;
  const int zi = blockIdx.y % L.nz, v = blockIdx.y / L.nz;
  const int64_t o = (int64_t)v * L.vstride + (int64_t)blockIdx.z * L.qstride +
                    ((int64_t)(L.zlo + zi) * L.N1 + L.ylo) * L.N0 + e;
  a[o] = y ? b * x[o] + c * y[o] : b * x[o];
}
void launch_linop_box(cudaStream_t s, const LinBox& L, int nv, int64_t nq, double* a, const double* x,
                      const double* y, double b, double c) {
  const dim3 grid((unsigned)((L.ny * L.N0 + 255) / 256), (unsigned)(L.nz * nv), (unsigned)nq);
  k_linop_box<<<grid, 256, 0, s>>>(L, nv, a, x, y, b, c);
}

// The deferred aux pass's cell list: one record per aux cell of the grid, at
// most 2^24 (cells past the capacity finish in place).  Not inside a
// stream capture.
bool ensure_aux_defer(grb_handle* h, int64_t cells) {
  const int64_t cap = std::min<int64_t>(cells, 1ll << 24);
  if (h->B.adefer && h->B.adefer_cap >= cap) return true;
  cudaFree(h->B.adefer);
  h->B.adefer = nullptr;
  h->B.adefer_cap = 0;
  if (!h->B.nadefer && cudaMalloc(&h->B.nadefer, sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (cudaMalloc(&h->B.adefer, sizeof(AuxDeferred) * (size_t)cap) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  h->B.adefer_cap = cap;
  return true;
}
void free_aux_defer(grb_handle* h) {
  cudaFree(h->B.adefer);
  h->B.adefer = nullptr;
  h->B.adefer_cap = 0;
}

// Aux pass and linop on the next stage's cells only (tuned mode with
// GRB_RANGES_NEXT_STAGE); otherwise every cell, the drop-in contract.
inline bool trimmed(const grb_handle* h) {
  return h->mode == GRB_MODE_TUNED && h->p.ranges == GRB_RANGES_NEXT_STAGE;
}

// A grid that is a run of blocks of the reserved grid — the same block
// geometry, idx pointing into the reserved grid's spacings at block q0 (its
// field pointers offset alike) — has block offset q0; any other grid 0.
int64_t run_offset(const grb_handle* h, const grb_grid* g) {
  if (!h->reserved || !h->res_idx || !g->idx || h->geo.nx != g->nx || h->geo.ny != g->ny ||
      h->geo.nz != g->nz || h->geo.g != g->ngz)
    return 0;
  const uintptr_t a = (uintptr_t)g->idx, b = (uintptr_t)h->res_idx;
  if (a < b || (a - b) % (3 * sizeof(double))) return 0;
  const int64_t q0 = (int64_t)((a - b) / (3 * sizeof(double)));
  return q0 + g->nq <= h->geo.nq ? q0 : 0;
}
// The handle's scratch for a call on grid g: the scratch that outlives a
// call (the Gardiner-Stone cell-centred E, written by the aux pass and read
// by the next substep) is addressed from the run's first block, so that
// calls on runs of blocks of the reserved grid see their own blocks'.
StageBufs run_bufs(const grb_handle* h, const grb_grid* g) {
  StageBufs B = h->B;
  if (B.ecenter) B.ecenter += run_offset(h, g) * 3 * h->geo.cells;
  return B;
}

// The static-metric cache when it was built for this geometry and these
// spacings and covers these blocks, else null.  A grid whose idx points
// into the cached spacings at block q0 (a run of blocks of the cached grid,
// with its field pointers offset alike) gets the cache from block q0 on.
const double* static_metric(const grb_handle* h, const Geo& G, const double* idx) {
  if (!h->d_metder || !idx || !h->metder_idx) return nullptr;
  const int key[4] = {G.nx, G.ny, G.nz, G.g};
  if (!std::equal(key, key + 4, h->metder_key)) return nullptr;
  const uintptr_t a = (uintptr_t)idx, b = (uintptr_t)h->metder_idx;
  if (a < b || (a - b) % (3 * sizeof(double))) return nullptr;
  const int64_t q0 = (int64_t)((a - b) / (3 * sizeof(double)));
  if (q0 + G.nq > h->metder_nq) return nullptr;
  return h->d_metder + q0 * (int64_t)kMetDer * G.nx * G.ny * G.nz;
}

// Refluxing of the stage (grb_set_reflux): the fluxes after FOFC, the edge
// EMFs after the update.  Returns the kernels launched.
int reflux_fluxes(grb_handle* h, const Geo& G, cudaStream_t s, const StageBufs& B) {
  if (!h->reflux) return 0;
  const RefluxDev& R = h->rf;
  const int64_t n2 = (int64_t)G.nx * G.nx * GRB_N_HRSC;
  int l = 0;
  if (R.nfaces) { k_reflux_faces<<<nblk(n2 * R.nfaces, 128), 128, 0, s>>>(G, R, B.flux); ++l; }
  if (R.nsame && h->reflux_flux_same) {
    k_reflux_same_faces<<<nblk(n2 * R.nsame, 128), 128, 0, s>>>(G, R, B.flux);
    ++l;
  }
  return l;
}
int reflux_emfs(grb_handle* h, const Geo& G, cudaStream_t s, const StageBufs& B) {
  if (!h->reflux) return 0;
  const RefluxDev& R = h->rf;
  const int64_t n = G.nx;
  int l = 0;
  if (R.nfaces) { k_reflux_emf_faces<<<nblk(n / 2 * (n / 2) * R.nfaces, 128), 128, 0, s>>>(G, R, B.emf); ++l; }
  if (R.nsame) { k_reflux_emf_same_faces<<<nblk(n * n * R.nsame, 128), 128, 0, s>>>(G, R, B.emf); ++l; }
  if (R.nedges) {
    k_reflux_emf_edges_compute<<<nblk(n * R.nedges, 128), 128, 0, s>>>(G, R, B.emf);
    k_reflux_emf_edges_apply<<<nblk(n * R.nedges, 128), 128, 0, s>>>(G, R, B.emf);
    l += 2;
  }
  if (R.nsame_edges) {
    k_reflux_emf_same_edges_compute<<<nblk(n * R.nsame_edges, 128), 128, 0, s>>>(G, R, B.emf);
    k_reflux_emf_same_edges_apply<<<nblk(n * R.nsame_edges, 128), 128, 0, s>>>(G, R, B.emf);
    l += 2;
  }
  return l;
}

// Grid of the FOFC list kernel: three 128-thread CTAs per SM (its register
// footprint) for a grid-stride loop over the listed faces.
static unsigned fofc_list_grid() {
  static int sms[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 444;
  if (!sms[dev] && cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms[dev] = 148;
  return (unsigned)(3 * sms[dev]);
}

// The stage in tuned mode: only the faces the stage reads, FAST flux math,
// tuned register caps.  Returns the number of kernels launched, or -1 when
// a scratch reset could not be enqueued.
int stage_tuned(grb_handle* h, const Geo& G, const grb_grid* g, double dt, double dtfact,
                const grb_fields* nw, const grb_fields* old, const double* aux, cudaStream_t s,
                StageBufs B, bool count_fofc) {
  const DevParams& P = h->dp;
  const int gz = G.g, T = 128;
  int launches = 0;
  const double* bf[3] = {old->bx, old->by, old->bz};
  const int nn[3] = {G.nx, G.ny, G.nz};
  for (int dir = 0; dir < 3; ++dir) {
    KScope ks(h, s, GRB_KIND_FLUX);
    int lo[3], n[3];
    for (int a = 0; a < 3; ++a) {
      if (a == dir) { lo[a] = gz - 1; n[a] = nn[a] + 3; }
      else if (P.emf == GRB_EMF_GS) { lo[a] = gz - 1; n[a] = nn[a] + 2; }
      else { lo[a] = gz - 3; n[a] = nn[a] + 6; }  // UCT reconstructs face data across
    }
    const Box b = box(lo[0], lo[1], lo[2], n[0], n[1], n[2], G.nq);
    const unsigned nb = nblk(b.count(), T);
    if (dir == 0) launch_flux_tuned<0>(h->var_flux, nb, s, P, G, b, old->state, aux, bf[0], B, h->d_queue + 2);
    if (dir == 1) launch_flux_tuned<1>(h->var_flux, nb, s, P, G, b, old->state, aux, bf[1], B, h->d_queue + 2);
    if (dir == 2) launch_flux_tuned<2>(h->var_flux, nb, s, P, G, b, old->state, aux, bf[2], B, h->d_queue + 2);
    ++launches;
  }
  const Box eb = box(gz, gz, gz, G.nx + 1, G.ny + 1, G.nz + 1, G.nq);
  {
    KScope ks(h, s, GRB_KIND_EMF);
    if (P.emf == GRB_EMF_GS) k_emf_gs<<<nblk(eb.count(), T), T, 0, s>>>(G, eb, B);
    else k_emf_uct<<<nblk(eb.count(), T), T, 0, s>>>(P, G, eb, old->bx, old->by, old->bz, B);
    ++launches;
  }
  if (P.fofc && P.emf == GRB_EMF_GS) {
    const int64_t nf = G.fcells * G.nq * 3;
    if (cudaMemsetAsync(B.ftag, 0, (size_t)nf, s) != cudaSuccess ||
        cudaMemsetAsync(B.etag, 0, (size_t)nf, s) != cudaSuccess ||
        (count_fofc && cudaMemsetAsync(B.counters, 0, 2 * sizeof(unsigned long long), s) != cudaSuccess))
      return -1;
    const Box fb = box(gz - 1, gz - 1, gz - 1, G.nx + 2, G.ny + 2, G.nz + 2, G.nq);
    const bool listed = B.flist && fb.count() < (1ll << 30);
    if (listed && cudaMemsetAsync(B.fcount, 0, sizeof(uint32_t), s) != cudaSuccess) return -1;
    {
      KScope ks(h, s, GRB_KIND_FOFC_FLAG);
      launch_flag_tuned(h->var_flag, nblk(fb.count(), T), s, P, G, fb, dt, dtfact, nw->state, old->state,
                        old->bx, old->by, old->bz, g->idx, g->coords, B, h->d_queue + 1);
      ++launches;
    }
    {
      KScope ks(h, s, GRB_KIND_FOFC_FIX);
      if (listed) {
        // the few tagged faces compacted first: the recompute kernel's
        // register footprint then costs occupancy only where there is work
        k_fofc_scan<<<nblk(fb.count(), 256), 256, 0, s>>>(G, fb, B);
        k_fofc_faces_list<true><<<fofc_list_grid(), T, 0, s>>>(P, G, fb, old->state, aux, old->bx, old->by,
                                                              old->bz, B);
        ++launches;
      } else {
        k_fofc_faces<true><<<nblk(fb.count(), T), T, 0, s>>>(P, G, fb, old->state, aux, old->bx, old->by,
                                                            old->bz, B);
      }
      k_fofc_edges<<<nblk(fb.count(), T), T, 0, s>>>(G, fb, B);
      launches += 2;
    }
  }
  if (h->reflux) {
    KScope ks(h, s, GRB_KIND_OTHER);
    launches += reflux_fluxes(h, G, s, B);
  }
  const Box ub = box(gz, gz, gz, G.nx, G.ny, G.nz, G.nq);
  {
    KScope ks(h, s, GRB_KIND_UPDATE);
    launch_update_tuned(h->var_update, nblk(ub.count(), T), s, P, G, ub, dt, dtfact, nw->state, old->state,
                        aux, g->idx, B, static_metric(h, G, g->idx), h->d_queue + 3);
    ++launches;
  }
  if (h->reflux) {
    KScope ks(h, s, GRB_KIND_OTHER);
    launches += reflux_emfs(h, G, s, B);
  }
  {
    KScope ks(h, s, GRB_KIND_CT);
    k_ct<<<nblk(eb.count(), T), T, 0, s>>>(G, eb, dt, dtfact, nw->bx, nw->by, nw->bz, g->idx, B);
    ++launches;
  }
  return launches;
}

}  // namespace

extern "C" {

void grb_params_defaults(grb_params* p, int32_t eos_kind) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->eos.kind = eos_kind;
  p->eos.n_pieces = 1;
  p->eos.gamma = 5.0 / 3.0;
  p->eos.gamma_th = 1.8;
  p->eos.eps_max = 1.0e5;
  p->eos.entropy_min = 1.0e-13;
  p->eos.temp_atm = 0.0;
  p->rho_fl = 1.0e-14; p->ye_fl = 0.0; p->temp_fl = 0.0; p->atmo_tol = 1.0e-3;
  p->excise_by_radius = 0; p->r_ex = 1.0; p->alp_ex = 0.05; p->rho_ex = 1.0e-14;
  p->temp_ex = 0.0; p->ye_ex = 0.0;
  p->c2p_tol = 1.0e-10; p->max_w = 50.0; p->max_sigma = 100.0; p->beta_fallback = 1.0e-2;
  p->alp_bh_thresh = 0.2; p->use_ent_backup = 1;
  p->rusanov_use_c_limit = 0.0;
  p->fofc_enable = 1; p->dmp_enable = 1; p->dmp_M = 1.2;
  p->recon = GRB_RECON_WENOZ; p->riemann = GRB_RIEMANN_HLL; p->emf = GRB_EMF_GS;
  p->ranges = GRB_RANGES_FULL;
}

int grb_eos_setup_pwpoly(grb_eos_params* e, int32_t n, double kappa_0, const double* gammas,
                         const double* rhos) {
  if (!e || n < 1 || n > GRB_MAX_PIECES || !gammas || (n > 1 && !rhos)) return GRB_ERR_INVALID;
  double r[GRB_MAX_PIECES] = {0.0};
  for (int i = 1; i < n; ++i) r[i] = rhos[i - 1];
  for (int i = 0; i + 1 < n; ++i)
    if (!(r[i + 1] > r[i])) return GRB_ERR_INVALID;
  double k[GRB_MAX_PIECES] = {0}, ep[GRB_MAX_PIECES] = {0}, pr[GRB_MAX_PIECES] = {0};
  k[0] = kappa_0;
  for (int i = 1; i < n; ++i) {
    k[i] = k[i - 1] * std::pow(r[i], gammas[i - 1] - gammas[i]);
    ep[i] = ep[i - 1] + k[i - 1] * std::pow(r[i], gammas[i - 1] - 1.) / (gammas[i - 1] - 1.) -
            k[i] * std::pow(r[i], gammas[i] - 1.) / (gammas[i] - 1.);
    pr[i] = k[i] * std::pow(r[i], gammas[i]);
  }
  e->n_pieces = n;
  for (int i = 0; i < GRB_MAX_PIECES; ++i) {
    e->pw_kappa[i] = i < n ? k[i] : 0.0;
    e->pw_gamma[i] = i < n ? gammas[i] : 0.0;
    e->pw_rho[i] = i < n ? r[i] : 0.0;
    e->pw_eps[i] = i < n ? ep[i] : 0.0;
    e->pw_press[i] = i < n ? pr[i] : 0.0;
  }
  return GRB_OK;
}

int grb_create(grb_handle** out, const grb_params* p) {
  if (!out) return GRB_ERR_INVALID;
  *out = nullptr;
  if (!valid_params(p)) return GRB_ERR_INVALID;
  grb_handle* h = new (std::nothrow) grb_handle();
  if (!h) return GRB_ERR_NOMEM;
  h->p = *p;
  h->dp = to_dev(*p);
  if (cudaMalloc(&h->d_flags, sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&h->d_counters, 2 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&h->d_queue, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(h->d_flags);
    cudaFree(h->d_counters);
    delete h;
    return GRB_ERR_CUDA;
  }
  cudaMemset(h->d_flags, 0, sizeof(uint32_t));
  cudaMemset(h->d_counters, 0, 2 * sizeof(unsigned long long));
  *out = h;
  return GRB_OK;
}

static void free_scratch(grb_handle* h) {
  cudaFree(h->B.flux); cudaFree(h->B.eface); cudaFree(h->B.vbar); cudaFree(h->B.ecenter);
  cudaFree(h->B.emf); cudaFree(h->B.ftag); cudaFree(h->B.etag);
  cudaFree(h->B.flist); cudaFree(h->B.fcount);
  h->B.flux = h->B.eface = h->B.vbar = h->B.ecenter = h->B.emf = nullptr;
  h->B.ftag = h->B.etag = nullptr;
  h->B.flist = h->B.fcount = nullptr;
  h->B.fcap = h->fcap_alloc = 0;
  h->reserved = false;
  h->cap_f = h->cap_c = 0;
}

int grb_destroy(grb_handle* h) {
  if (!h) return GRB_ERR_INVALID;
  for (auto& m : h->marks) { cudaEventDestroy(m.a); cudaEventDestroy(m.b); }
  for (auto e : h->pool) cudaEventDestroy(e);
  free_scratch(h);
  cudaFree(h->d_flags);
  cudaFree(h->d_counters);
  cudaFree(h->d_mlp);
  cudaFree(h->d_mlp_pack);
  cudaFree(h->d_queue);
  cudaFree(h->d_auxlist);
  cudaFree(h->d_ghostruns);
  cudaFree(h->d_stage_io);
  cudaFree(h->d_metder);
  cudaFree(h->d_refacc);
  cudaFree(h->B.adefer);
  cudaFree(h->B.nadefer);
  cudaFree(h->d_defer);
  cudaFree(h->d_ndefer);
  delete h;
  return GRB_OK;
}

int grb_reserve(grb_handle* h, const grb_grid* g) {
  if (!h || !g || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->nq < 1 || g->ngz < 4) return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  h->res_idx = g->idx;
  if (h->reserved && same_geo(h->geo, g)) return GRB_OK;
  free_scratch(h);
  const int64_t nf = G.fcells * G.nq, nc = G.cells * G.nq;
  auto al = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
  bool ok = al((void**)&h->B.flux, sizeof(double) * nf * 7 * 3) &&
            al((void**)&h->B.emf, sizeof(double) * nf * 3) &&
            al((void**)&h->B.ftag, (size_t)nf * 3) && al((void**)&h->B.etag, (size_t)nf * 3);
  if (ok && h->p.emf == GRB_EMF_GS)
    ok = al((void**)&h->B.eface, sizeof(double) * nf * 2 * 3) &&
         al((void**)&h->B.ecenter, sizeof(double) * nc * 3);
  if (ok && h->p.emf == GRB_EMF_UCT) ok = al((void**)&h->B.vbar, sizeof(double) * nf * 4 * 3);
  if (ok && h->p.emf == GRB_EMF_GS && h->p.fofc_enable) {
    // the compacted FOFC face list: up to 4 Mi faces a substep (more falls
    // back to the full recompute launch)
    h->B.fcap = h->fcap_alloc = (uint32_t)std::min<int64_t>(nf * 3, 1 << 22);
    ok = al((void**)&h->B.flist, sizeof(uint32_t) * h->B.fcap) && al((void**)&h->B.fcount, sizeof(uint32_t));
  }
  if (!ok) {
    free_scratch(h);
    cudaGetLastError();
    return fail(h, GRB_ERR_NOMEM);
  }
  // Edge EMFs outside the computed range stay zero for the lifetime of the
  // scratch, as the zero-initialised reference view does; the FOFC
  // tentative CT update of ghost-layer cells reads them.
  CK(cudaMemset(h->B.emf, 0, sizeof(double) * nf * 3));
  CK(cudaMemset(h->B.flux, 0, sizeof(double) * nf * 7 * 3));
  if (h->B.eface) CK(cudaMemset(h->B.eface, 0, sizeof(double) * nf * 2 * 3));
  if (h->B.ecenter) CK(cudaMemset(h->B.ecenter, 0, sizeof(double) * nc * 3));
  if (h->B.vbar) CK(cudaMemset(h->B.vbar, 0, sizeof(double) * nf * 4 * 3));
  CK(cudaDeviceSynchronize());
  h->geo = G;
  h->cap_f = nf;
  h->cap_c = nc;
  h->reserved = true;
  h->B.counters = h->d_counters;
  h->B.flags = h->d_flags;
  return GRB_OK;
}

int grb_get_status(grb_handle* h, grb_status* st) {
  if (!h || !st) return GRB_ERR_INVALID;
  uint32_t f = 0;
  unsigned long long c[2] = {0, 0};
  CK(cudaMemcpy(&f, h->d_flags, sizeof(f), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(c, h->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
  st->device_flags = f;
  st->last_error = h->last_error;
  st->fofc_faces = (int64_t)c[0];
  st->fofc_edges = (int64_t)c[1];
  st->launches = h->launches;
  return GRB_OK;
}

int grb_clear_status(grb_handle* h) {
  if (!h) return GRB_ERR_INVALID;
  CK(cudaMemset(h->d_flags, 0, sizeof(uint32_t)));
  h->last_error = GRB_OK;
  return GRB_OK;
}

int grb_advance_substep(grb_handle* h, const grb_grid* g, double t, double dt, double dtfact,
                        const grb_fields* nw, const grb_fields* old, const double* aux,
                        void* stream) {
  (void)t;
  if (!h) return GRB_ERR_INVALID;
  int rc = check_grid(h, g);
  if (rc) return fail(h, rc);
  if (!nw || !old || !aux || !nw->state || !old->state || !nw->bx || !old->bx) return fail(h, GRB_ERR_INVALID);
  cudaStream_t s = (cudaStream_t)stream;
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  const DevParams& P = h->dp;
  const int gz = G.g, T = 128;
  // refluxing descriptors name blocks of the reserved grid
  if (h->reflux && (run_offset(h, g) != 0 || g->nq != h->geo.nq)) return fail(h, GRB_ERR_INVALID);
  StageBufs B = run_bufs(h, g);
  if (h->mode == GRB_MODE_TUNED) {
    const int nl = stage_tuned(h, G, g, dt, dtfact, nw, old, aux, s, B, true);
    if (nl < 0) return fail(h, GRB_ERR_CUDA);
    h->launches += nl;
    CK(cudaGetLastError());
    return GRB_OK;
  }
  // compute_fluxes: reference ranges (evolve.cpp:908-922)
  const double* bf[3] = {old->bx, old->by, old->bz};
  for (int dir = 0; dir < 3; ++dir) {
    int lo[3] = {0, 0, 0}, n[3] = {G.NX, G.NY, G.NZ};
    lo[dir] = gz - 1;
    n[dir] = (dir == 0 ? G.nx : dir == 1 ? G.ny : G.nz) + 3;
    const Box b = box(lo[0], lo[1], lo[2], n[0], n[1], n[2], G.nq);
    KScope ks(h, s, GRB_KIND_FLUX);
    if (dir == 0) k_flux<0><<<nblk(b.count(), T), T, 0, s>>>(P, G, b, old->state, aux, bf[0], B);
    if (dir == 1) k_flux<1><<<nblk(b.count(), T), T, 0, s>>>(P, G, b, old->state, aux, bf[1], B);
    if (dir == 2) k_flux<2><<<nblk(b.count(), T), T, 0, s>>>(P, G, b, old->state, aux, bf[2], B);
    ++h->launches;
  }
  const Box eb = box(gz, gz, gz, G.nx + 1, G.ny + 1, G.nz + 1, G.nq);
  {
  KScope ks(h, s, GRB_KIND_EMF);
  if (P.emf == GRB_EMF_GS)
    k_emf_gs<<<nblk(eb.count(), T), T, 0, s>>>(G, eb, B);
  else
    k_emf_uct<<<nblk(eb.count(), T), T, 0, s>>>(P, G, eb, old->bx, old->by, old->bz, B);
  ++h->launches;
  }
  if (P.fofc && P.emf == GRB_EMF_GS) {
    const int64_t nf = G.fcells * G.nq * 3;
    CK(cudaMemsetAsync(B.ftag, 0, (size_t)nf, s));
    CK(cudaMemsetAsync(B.etag, 0, (size_t)nf, s));
    CK(cudaMemsetAsync(B.counters, 0, 2 * sizeof(unsigned long long), s));
    const Box fb = box(gz - 1, gz - 1, gz - 1, G.nx + 2, G.ny + 2, G.nz + 2, G.nq);
    {
    KScope ks(h, s, GRB_KIND_FOFC_FLAG);
    k_fofc_flag<1><<<nblk(fb.count(), T), T, 0, s>>>(P, G, fb, dt, dtfact, nw->state, old->state, old->bx,
                                                   old->by, old->bz, g->idx, g->coords, B); ++h->launches;
    }
    {
    KScope ks(h, s, GRB_KIND_FOFC_FIX);
    k_fofc_faces<false><<<nblk(fb.count(), T), T, 0, s>>>(P, G, fb, old->state, aux, old->bx, old->by, old->bz, B); ++h->launches;
    k_fofc_edges<<<nblk(fb.count(), T), T, 0, s>>>(G, fb, B); ++h->launches;
    }
  }
  if (h->reflux) {
    KScope ks(h, s, GRB_KIND_OTHER);
    h->launches += reflux_fluxes(h, G, s, B);
  }
  const Box ub = box(gz, gz, gz, G.nx, G.ny, G.nz, G.nq);
  {
  KScope ks(h, s, GRB_KIND_UPDATE);
  k_update<1><<<nblk(ub.count(), T), T, 0, s>>>(P, G, ub, dt, dtfact, nw->state, old->state, aux, g->idx, B); ++h->launches;
  }
  if (h->reflux) {
    KScope ks(h, s, GRB_KIND_OTHER);
    h->launches += reflux_emfs(h, G, s, B);
  }
  {
  KScope ks(h, s, GRB_KIND_CT);
  k_ct<<<nblk(eb.count(), T), T, 0, s>>>(G, eb, dt, dtfact, nw->bx, nw->by, nw->bz, g->idx, B); ++h->launches;
  }
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_compute_auxiliary_quantities(grb_handle* h, const grb_grid* g, const grb_fields* st,
                                     double* aux, void* stream) {
  return grb_compute_auxiliary_quantities_dt(h, g, st, aux, nullptr, 0.0, nullptr, stream);
}

// The cells whose primitives (and c2p resets) the next tuned stage reads
// before the ghost exchange refills the rest, with the Gardiner-Stone EMF:
// the face fluxes reconstruct along each axis over the whole block from
// cells whose two other indices lie in [g-1, n+g+1) (cells with at least
// two indices there), and the FOFC flag's DMP test reads the new
// conservatives, which the c2p may reset, on [g-2, n+g+2)^3.  The flag, the
// FOFC face and edge corrections, the cell-centred E of the EMF and the
// update stay inside these.  Packed i | j << 8 | k << 16, x fastest.
std::vector<uint32_t> tuned_aux_cells(const Geo& G) {
  const int N[3] = {G.NX, G.NY, G.NZ}, n[3] = {G.nx, G.ny, G.nz};
  std::vector<uint32_t> v;
  for (int k = 0; k < N[2]; ++k)
    for (int j = 0; j < N[1]; ++j)
      for (int i = 0; i < N[0]; ++i) {
        const int c[3] = {i, j, k};
        int in_t = 0, in_d = 0;
        for (int a = 0; a < 3; ++a) {
          in_t += c[a] >= G.g - 1 && c[a] < n[a] + G.g + 1;
          in_d += c[a] >= G.g - 2 && c[a] < n[a] + G.g + 2;
        }
        if (in_t >= 2 || in_d == 3) v.push_back((uint32_t)i | (uint32_t)j << 8 | (uint32_t)k << 16);
      }
  return v;
}
// The aux box of the tuned mode: the cell list above when it applies (GS
// EMF, blocks up to 256 cells a side, the list already built for this
// geometry or buildable now, i.e. not inside a stream capture), else the
// whole block.
Box tuned_aux_box(grb_handle* h, const Geo& G, cudaStream_t s) {
  Box b = box(0, 0, 0, G.NX, G.NY, G.NZ, G.nq);
  if (h->dp.emf != GRB_EMF_GS || G.NX > 256 || G.NY > 256 || G.NZ > 256 || G.g < 2) return b;
  const int key[4] = {G.nx, G.ny, G.nz, G.g};
  if (!h->d_auxlist || !std::equal(key, key + 4, h->auxlist_key)) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return b;
    const std::vector<uint32_t> v = tuned_aux_cells(G);
    uint32_t* d = nullptr;
    if (cudaMalloc(&d, v.size() * sizeof(uint32_t)) != cudaSuccess) return b;
    if (cudaMemcpy(d, v.data(), v.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(d);
      return b;
    }
    cudaFree(h->d_auxlist);
    h->d_auxlist = d;
    h->auxlist_n = (uint32_t)v.size();
    std::copy(key, key + 4, h->auxlist_key);
  }
  if ((int64_t)h->auxlist_n * G.nq >= (1ll << 32)) return b;
  b.list = h->d_auxlist;
  b.nlist = h->auxlist_n;
  b.dl = make_fastdiv(h->auxlist_n);
  return b;
}

int grb_compute_auxiliary_quantities_dt(grb_handle* h, const grb_grid* g, const grb_fields* st, double* aux,
                                        const double* dx, double cfl, double* dt_out, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  int rc = check_grid(h, g);
  if (rc) return fail(h, rc);
  if (!st || !st->state || !st->bx || !st->by || !st->bz || !aux) return fail(h, GRB_ERR_INVALID);
  if (dt_out && (!dx || !(cfl > 0.0))) return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  const Box b = box(0, 0, 0, G.NX, G.NY, G.NZ, G.nq);
  cudaStream_t s = (cudaStream_t)stream;
  KScope ks(h, s, GRB_KIND_AUX);
  const DtArgs dta{dx, cfl, reinterpret_cast<unsigned long long*>(dt_out)};
  if (dt_out) {
    k_dt_init<<<1, 1, 0, s>>>(dta.out);
    ++h->launches;
  }
  const StageBufs B = run_bufs(h, g);
  if (h->mode == GRB_MODE_TUNED) {
    const Box tb = trimmed(h) ? tuned_aux_box(h, G, s) : b;
    launch_aux_tuned(h->var_aux, nblk(tb.count(), 128), s, h->dp, G, tb, st->state, st->bx, st->by, st->bz, aux,
                     g->idx, g->coords, B, dt_out ? &dta : nullptr, h->d_queue);
  } else if (dt_out) {
    k_aux<1, true><<<nblk(b.count(), 128), 128, 0, s>>>(h->dp, G, b, st->state, st->bx, st->by, st->bz, aux,
                                                        g->idx, g->coords, B, dta);
  } else {
    k_aux<1><<<nblk(b.count(), 128), 128, 0, s>>>(h->dp, G, b, st->state, st->bx, st->by, st->bz, aux, g->idx,
                                                  g->coords, B);
  }
  ++h->launches;
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_find_stable_timestep(grb_handle* h, const grb_grid* g, const grb_fields* st, const double* aux,
                             const double* dx, double cfl, double* dt_out, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  int rc = check_grid(h, g);
  if (rc) return fail(h, rc);
  if (!st || !st->state || !aux || !dx || !dt_out || !(cfl > 0.0)) return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  const Box b = box(G.g, G.g, G.g, G.nx, G.ny, G.nz, G.nq);
  cudaStream_t s = (cudaStream_t)stream;
  KScope ks(h, s, GRB_KIND_OTHER);
  const DtArgs dta{dx, cfl, reinterpret_cast<unsigned long long*>(dt_out)};
  k_dt_init<<<1, 1, 0, s>>>(dta.out);
  k_dt<<<nblk(b.count(), 128), 128, 0, s>>>(h->dp, G, b, st->state, aux, dta);
  h->launches += 2;
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_reset_c2p_diagnostics(grb_handle* h, const grb_grid* g, double* aux, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  int rc = check_grid(h, g);
  if (rc) return fail(h, rc);
  if (!aux) return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  KScope ks(h, (cudaStream_t)stream, GRB_KIND_OTHER);
  k_reset_diag<<<1184, 256, 0, (cudaStream_t)stream>>>(G, aux); ++h->launches;
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_linop_apply(grb_handle* h, const grb_grid* g, const grb_fields* A, const grb_fields* Bf,
                    const grb_fields* Cf, double b, double c, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g || g->nq < 1) return fail(h, GRB_ERR_INVALID);
  if (!A || !Bf || !A->state || !Bf->state) return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n[4] = {G.cells * GRB_N_EVOL_VARS * G.nq, (int64_t)(G.NX + 1) * G.NY * G.NZ * G.nq,
                        (int64_t)G.NX * (G.NY + 1) * G.NZ * G.nq, (int64_t)G.NX * G.NY * (G.NZ + 1) * G.nq};
  double* a[4] = {A->state, A->bx, A->by, A->bz};
  const double* x[4] = {Bf->state, Bf->bx, Bf->by, Bf->bz};
  const double* y[4] = {Cf ? Cf->state : nullptr, Cf ? Cf->bx : nullptr, Cf ? Cf->by : nullptr, Cf ? Cf->bz : nullptr};
  KScope ks(h, s, GRB_KIND_LINOP);
  if (trimmed(h)) {
    // The Cowling metric and curvature are static, and the next stage reads
    // the combination only on the HRSC variables of cells [g-2, n+g+2) (the
    // FOFC flag window) and on the faces the CT update advances before the
    // ghost exchange refills the rest: combine just those.
    const int gz = G.g;
    if (G.nq > 65535 || gz < 2) return fail(h, GRB_ERR_INVALID);
    LinBox Lc{G.NX, G.NY, G.NZ, gz - 2, G.ny + 4, gz - 2, G.nz + 4, (int64_t)G.cells,
              (int64_t)G.cells * GRB_N_EVOL_VARS};
    launch_linop_box(s, Lc, GRB_N_HRSC, G.nq, a[0], x[0], y[0], b, c);
    ++h->launches;
    for (int fd = 0; fd < 3; ++fd) {
      int N[3] = {G.NX, G.NY, G.NZ}, nn[3] = {G.nx, G.ny, G.nz};
      N[fd] += 1;
      nn[fd] += 1;
      const int64_t fc = (int64_t)N[0] * N[1] * N[2];
      LinBox Lf{N[0], N[1], N[2], gz, nn[1], gz, nn[2], fc, fc};
      launch_linop_box(s, Lf, 1, G.nq, a[1 + fd], x[1 + fd], y[1 + fd], b, c);
      ++h->launches;
    }
    CK(cudaGetLastError());
    return GRB_OK;
  }
  for (int v = 0; v < 4; ++v) {
    k_linop<<<148 * 16, 256, 0, s>>>(n[v], a[v], x[v], y[v], b, c);
    ++h->launches;
  }
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_linop_apply3(grb_handle* h, const grb_grid* g, const grb_fields* A, const grb_fields* Bf,
                     const grb_fields* Cf, const grb_fields* Df, double b, double c, double d, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g || g->nq < 1 || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->ngz < 0) return fail(h, GRB_ERR_INVALID);
  const grb_fields* f[4] = {A, Bf, Cf, Df};
  for (const grb_fields* x : f)
    if (!x || !x->state || !x->bx || !x->by || !x->bz) return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n[4] = {G.cells * GRB_N_EVOL_VARS * G.nq, (int64_t)(G.NX + 1) * G.NY * G.NZ * G.nq,
                        (int64_t)G.NX * (G.NY + 1) * G.NZ * G.nq, (int64_t)G.NX * G.NY * (G.NZ + 1) * G.nq};
  double* a[4] = {A->state, A->bx, A->by, A->bz};
  const double* x[4] = {Bf->state, Bf->bx, Bf->by, Bf->bz};
  const double* y[4] = {Cf->state, Cf->bx, Cf->by, Cf->bz};
  const double* z[4] = {Df->state, Df->bx, Df->by, Df->bz};
  KScope ks(h, s, GRB_KIND_LINOP);
  for (int v = 0; v < 4; ++v) {
    k_linop3<<<148 * 16, 256, 0, s>>>(n[v], a[v], x[v], y[v], z[v], b, c, d);
    ++h->launches;
  }
  CK(cudaGetLastError());
  return GRB_OK;
}

}  // extern "C"

namespace {

int launch_c2p(grb_handle* h, int64_t n, const double* cons, const double* metric, double* prims,
               double* cons_out, uint32_t* err, bool learned, const grb_c2p_diag* diag, cudaStream_t s) {
  C2PDiagDev d{nullptr, nullptr, nullptr, nullptr};
  if (diag) d = C2PDiagDev{diag->iters, diag->guess_used, diag->mu, diag->bracket};
  if (n > (int64_t)kC2PThreads * 0x7fffffff) return fail(h, GRB_ERR_INVALID);
  const unsigned nb = nblk(n, kC2PThreads);
  const bool fast = h->mode == GRB_MODE_TUNED;
  if (fast) {
    // tuned mode: the entropy backups deferred to a second, compacted pass
    if (n > h->defer_cap) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
        return fail(h, GRB_ERR_INVALID);  // the first call of a size must come before any capture
      cudaFree(h->d_defer);
      h->d_defer = nullptr;
      h->defer_cap = 0;
      if (!h->d_ndefer && cudaMalloc(&h->d_ndefer, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, GRB_ERR_NOMEM);
      }
      if (cudaMalloc(&h->d_defer, sizeof(C2PDeferred) * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, GRB_ERR_NOMEM);
      }
      h->defer_cap = n;
    }
    CK(cudaMemsetAsync(h->d_ndefer, 0, sizeof(unsigned long long), s));
    if (learned)
      k_c2p_batch_front<true, true><<<nb, kC2PThreads, 0, s>>>(h->dp, n, cons, metric, prims, cons_out, err, d,
                                                              h->d_mlp_pack, h->d_flags, h->d_defer, h->d_ndefer);
    else
      k_c2p_batch_front<false, true><<<nb, kC2PThreads, 0, s>>>(h->dp, n, cons, metric, prims, cons_out, err, d,
                                                               nullptr, h->d_flags, h->d_defer, h->d_ndefer);
    const unsigned gb = (unsigned)std::min<int64_t>(nb, 148 * 16);
    k_c2p_batch_backup<true><<<gb, kC2PThreads, 0, s>>>(h->dp, n, metric, prims, cons_out, err, h->d_flags,
                                                       h->d_defer, h->d_ndefer);
    h->launches += 2;
    CK(cudaGetLastError());
    return GRB_OK;
  }
  if (learned)
    k_c2p_batch<true><<<nb, kC2PThreads, 0, s>>>(h->dp, n, cons, metric, prims, cons_out, err, d, h->d_mlp_pack,
                                                 h->d_flags);
  else
    k_c2p_batch<false><<<nb, kC2PThreads, 0, s>>>(h->dp, n, cons, metric, prims, cons_out, err, d, nullptr,
                                                  h->d_flags);
  ++h->launches;
  CK(cudaGetLastError());
  return GRB_OK;
}

int ensure_mlp(grb_handle* h) {
  if (!h->d_mlp) CK(cudaMalloc(&h->d_mlp, sizeof(float) * kMlpNumParams));
  if (!h->d_mlp_pack) CK(cudaMalloc(&h->d_mlp_pack, sizeof(MlpSmem)));
  return GRB_OK;
}

// Rebuild the shared-memory image after the parameters changed.
int pack_mlp(grb_handle* h, cudaStream_t s) {
  k_mlp_pack<<<1, 256, 0, s>>>(h->d_mlp, h->d_mlp_pack);
  ++h->launches;
  CK(cudaGetLastError());
  return GRB_OK;
}

// He-uniform hidden weights, small output layer, zero biases (host RNG,
// reproducible for a seed).
void mlp_init(std::vector<float>& P, uint64_t seed) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  std::fill(P.begin(), P.end(), 0.f);
  const float a1 = std::sqrt(6.f / kMlpIn), a2 = std::sqrt(6.f / kMlpH), a4 = std::sqrt(3.f / kMlpH);
  // high parts and remainders of an input start with the same weight
  for (int o = 0; o < kMlpH; ++o)
    for (int k = 0; k < kMlpIn; ++k)
      P[kMlpOffW1 + o * kMlpK0 + k] = P[kMlpOffW1 + o * kMlpK0 + kMlpIn + k] = a1 * u(rng);
  for (int t = 0; t < kMlpH * kMlpH; ++t) P[kMlpOffW2 + t] = a2 * u(rng);
  for (int t = 0; t < kMlpH * kMlpH; ++t) P[kMlpOffW3 + t] = a2 * u(rng);
  for (int t = 0; t < kMlpH; ++t) P[kMlpOffW4 + t] = a4 * u(rng);
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { cudaFree(p); }
  template <class T>
  T* as() { return static_cast<T*>(p); }
};

}  // namespace

extern "C" {

static_assert(kMlpNumParams == GRB_MLP_NUM_PARAMS, "parameter block size");
static_assert(kMlpNumWeights == GRB_MLP_NUM_WEIGHTS, "trainable block size");

int grb_c2p_batch(grb_handle* h, int64_t n, const double* cons, const double* metric, double* prims,
                  double* cons_out, uint32_t* err, int32_t use_learned, void* stream) {
  return grb_c2p_batch_diag(h, n, cons, metric, prims, cons_out, err, use_learned, nullptr, stream);
}

int grb_c2p_batch_diag(grb_handle* h, int64_t n, const double* cons, const double* metric, double* prims,
                       double* cons_out, uint32_t* err, int32_t use_learned, const grb_c2p_diag* diag,
                       void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (n < 0 || (n > 0 && (!cons || !prims))) return fail(h, GRB_ERR_INVALID);
  if (use_learned && !h->mlp_ready) return fail(h, GRB_ERR_NO_MODEL);
  if (n == 0) return GRB_OK;
  KScope ks(h, (cudaStream_t)stream, GRB_KIND_C2P);
  return launch_c2p(h, n, cons, metric, prims, cons_out, err, use_learned != 0, diag, (cudaStream_t)stream);
}

int grb_c2p_features(grb_handle* h, int64_t n, const double* cons, const double* metric, const double* mu,
                     float* feat, float* target, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (n < 0 || (n > 0 && (!cons || !feat || !target))) return fail(h, GRB_ERR_INVALID);
  if (n == 0) return GRB_OK;
  KScope ks(h, (cudaStream_t)stream, GRB_KIND_OTHER);
  k_mlp_labels<<<(unsigned)std::min<int64_t>(nblk(n, 256), 148 * 8), 256, 0, (cudaStream_t)stream>>>(
      h->dp, n, cons, metric, mu, feat, target);
  ++h->launches;
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_mlp_eval(grb_handle* h, int64_t n, const float* params, const float* feat, float* out, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (n < 0 || (n > 0 && (!feat || !out))) return fail(h, GRB_ERR_INVALID);
  if (!params && !h->mlp_ready) return fail(h, GRB_ERR_NO_MODEL);
  if (n == 0) return GRB_OK;
  KScope ks(h, (cudaStream_t)stream, GRB_KIND_OTHER);
  const unsigned grid = (unsigned)std::min<int64_t>(nblk(n, kC2PThreads), 148 * 8);
  k_mlp_eval<<<grid, kC2PThreads, 0, (cudaStream_t)stream>>>(params ? params : h->d_mlp, n, feat, out);
  ++h->launches;
  CK(cudaGetLastError());
  return GRB_OK;
}

}  // extern "C"

namespace {
int grad_setup(grb_handle* h) {
  static bool done = false;
  if (!done) {
    CK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpGradSmem)));
    done = true;
  }
  return GRB_OK;
}
}  // namespace

// FMR prolongation launches of one element kind (grb_prolong_to_ghosts).
template <int kKind>
static void launch_prolong(const Geo& G, const int ext[3], const grb_fields* fine, const grb_fields* cbuf,
                           int64_t nelems, const int64_t* fine_q, const int64_t* cbuf_q, const uint8_t* elem_id,
                           const int8_t* have_fine, const RestrictVars* V, bool faces, cudaStream_t s) {
  if (V[0].n) {
    const Box b = box(0, 0, 0, ext[0] / 2, ext[1] / 2, ext[2] / 2, (int64_t)V[0].n * nelems);
    k_prolong_cells<kKind><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, V[0], make_fastdiv((uint32_t)V[0].n),
                                                                cbuf->state, fine->state, fine_q, cbuf_q, elem_id);
  }
  if (V[1].n) {
    // the kind's largest element cross-section in (x, y), in coarse cells
    const int ne = kKind == GRB_ELEM_FACE ? 6 : (kKind == GRB_ELEM_EDGE ? 12 : 8);
    int cols = 0;
    for (int e = 0; e < ne; ++e) {
      int r[2];
      for (int d = 0; d < 2; ++d) {
        int w, lp;
        ghost_axis<kKind>(e, d, w, lp);
        r[d] = w == 2 ? G.nx / 2 : G.g / 2;
      }
      cols = r[0] * r[1] > cols ? r[0] * r[1] : cols;
    }
    const Box b = box(0, 0, 0, cols, 1, 1, (int64_t)V[1].n * nelems);
    k_prolong_lag_zcol<kKind><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, V[1], make_fastdiv((uint32_t)V[1].n),
                                                                   cbuf->state, fine->state, fine_q, cbuf_q, elem_id);
  }
  if (!faces) return;
  const Box b = box(0, 0, 0, ext[0] / 2, ext[1] / 2, ext[2] / 2, nelems);
  k_prolong_faces<kKind, 1><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, fine->bx, fine->by, fine->bz, cbuf->bx,
                                                                 cbuf->by, cbuf->bz, fine_q, cbuf_q, elem_id, have_fine);
  k_prolong_faces<kKind, 2><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, fine->bx, fine->by, fine->bz, cbuf->bx,
                                                                 cbuf->by, cbuf->bz, fine_q, cbuf_q, elem_id, have_fine);
}

extern "C" {

int grb_mlp_grad(grb_handle* h, int64_t n, const float* params, const float* feat, const float* target,
                 float* grad, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (n < 1 || n > (int64_t)kGradRows * 65535 || !params || !feat || !target || !grad) return fail(h, GRB_ERR_INVALID);
  if (int rc = grad_setup(h)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int nparts = (int)nblk(n, kGradRows);
  DevBuf part;
  CK(cudaMalloc(&part.p, sizeof(float) * (size_t)nparts * kPW));
  KScope ks(h, s, GRB_KIND_OTHER);
  k_mlp_grad<<<nparts, kGradThreads, sizeof(MlpGradSmem), s>>>(params, n, feat, target, n, 0, 0, 1,
                                                              1.f / (float)n, part.as<float>());
  k_mlp_reduce<<<nblk(kPW, 256), 256, 0, s>>>(part.as<float>(), nparts, grad);
  h->launches += 2;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));  // part is freed on return
  return GRB_OK;
}

void grb_train_config_defaults(grb_train_config* c) {
  if (!c) return;
  c->steps = 8000;
  c->batch = 16384;
  c->lr = 3e-3f;
  c->lr_min = 3e-5f;
  c->seed = 0x6A5CEull;
  c->calib_states = 1 << 18;
}

int grb_c2p_train(grb_handle* h, int64_t n, const double* cons, const double* metric, const grb_train_config* cfg,
                  grb_train_report* rep, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  grb_train_config C;
  grb_train_config_defaults(&C);
  if (cfg) C = *cfg;
  if (n < kGradRows || !cons || C.steps < 1 || C.batch < kGradRows || C.batch % kGradRows ||
      C.batch > kGradRows * 65535 || !(C.lr > 0.f) || C.lr_min < 0.f || C.calib_states < 0)
    return fail(h, GRB_ERR_INVALID);
  if (int rc = ensure_mlp(h)) return rc;
  if (int rc = grad_setup(h)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  grb_train_report R{};
  R.states = n;
  const int nparts = C.batch / kGradRows;
  DevBuf prims, mu, feat, tgt, part, m1, m2, loss, stat, pred;
  CK(cudaMalloc(&prims.p, sizeof(double) * 13 * (size_t)n));
  CK(cudaMalloc(&mu.p, sizeof(double) * (size_t)n));
  CK(cudaMalloc(&feat.p, sizeof(float) * kMlpIn * (size_t)n));
  CK(cudaMalloc(&tgt.p, sizeof(float) * (size_t)n));
  CK(cudaMalloc(&pred.p, sizeof(float) * (size_t)n));
  CK(cudaMalloc(&part.p, sizeof(float) * (size_t)nparts * kPW));
  CK(cudaMalloc(&m1.p, sizeof(float) * kMlpNumWeights));
  CK(cudaMalloc(&m2.p, sizeof(float) * kMlpNumWeights));
  CK(cudaMalloc(&loss.p, sizeof(float) * (size_t)C.steps));
  CK(cudaMalloc(&stat.p, sizeof(double) * kStatBlocks * kStatN));
  CK(cudaMemsetAsync(m1.p, 0, sizeof(float) * kMlpNumWeights, s));
  CK(cudaMemsetAsync(m2.p, 0, sizeof(float) * kMlpNumWeights, s));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, s));
  h->mlp_ready = false;
  // 1. labels: roots of the plain FP64 c2p, features of the same states
  grb_c2p_diag dg{nullptr, nullptr, mu.as<double>(), nullptr};
  if (int rc = launch_c2p(h, n, cons, metric, prims.as<double>(), nullptr, nullptr, false, &dg, s)) return rc;
  k_mlp_labels<<<(unsigned)std::min<int64_t>(nblk(n, 256), 148 * 8), 256, 0, s>>>(
      h->dp, n, cons, metric, mu.as<double>(), feat.as<float>(), tgt.as<float>());
  k_mlp_stats<<<kStatBlocks, 256, 0, s>>>(n, feat.as<float>(), tgt.as<float>(), stat.as<double>());
  h->launches += 2;
  CK(cudaGetLastError());
  std::vector<double> st(kStatBlocks * kStatN);
  CK(cudaMemcpyAsync(st.data(), stat.p, sizeof(double) * st.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double sum[kStatN] = {0};
  for (int b = 0; b < kStatBlocks; ++b)
    for (int a = 0; a < kStatN; ++a) sum[a] += st[b * kStatN + a];
  const double cnt = sum[2 * kMlpIn + 2];
  R.labelled = (int64_t)cnt;
  if (cnt < kGradRows) return fail(h, GRB_ERR_INVALID);
  // 2. initial network and normalisation
  std::vector<float> P(kMlpNumParams);
  mlp_init(P, C.seed);
  for (int k = 0; k < kMlpIn; ++k) {
    const double m = sum[k] / cnt, v = std::max(sum[kMlpIn + k] / cnt - m * m, 0.0);
    P[kMlpOffNorm + k] = (float)m;
    P[kMlpOffNorm + kMlpIn + k] = (float)std::max(std::sqrt(v), 1e-3);
  }
  {
    const double m = sum[2 * kMlpIn] / cnt, v = std::max(sum[2 * kMlpIn + 1] / cnt - m * m, 0.0);
    P[kMlpOffNorm + 2 * kMlpIn] = (float)m;
    P[kMlpOffNorm + 2 * kMlpIn + 1] = (float)std::max(std::sqrt(v), 1e-6);
  }
  P[kMlpOffNorm + 2 * kMlpIn + 2] = 0.1f;
  CK(cudaMemcpyAsync(h->d_mlp, P.data(), sizeof(float) * kMlpNumParams, cudaMemcpyHostToDevice, s));
  // 3. Adam with linear warm-up and cosine decay
  const int64_t warm = std::min<int64_t>(100, C.steps / 10);
  double b1t = 1.0, b2t = 1.0;
  for (int64_t it = 0; it < C.steps; ++it) {
    double lr;
    if (it < warm) lr = C.lr * (double)(it + 1) / (double)warm;
    else lr = C.lr_min + 0.5 * (C.lr - C.lr_min) * (1.0 + std::cos(M_PI * (double)(it - warm) / (double)std::max<int64_t>(1, C.steps - warm)));
    b1t *= 0.9;
    b2t *= 0.999;
    k_mlp_grad<<<nparts, kGradThreads, sizeof(MlpGradSmem), s>>>(h->d_mlp, n, feat.as<float>(), tgt.as<float>(),
                                                                C.batch, C.seed, it, 0, 1.f / (float)C.batch,
                                                                part.as<float>());
    k_mlp_adam<<<nblk(kPW, 256), 256, 0, s>>>(h->d_mlp, m1.as<float>(), m2.as<float>(), part.as<float>(), nparts,
                                               (float)lr, (float)(1.0 - b1t), (float)(1.0 - b2t), loss.as<float>(), it);
    h->launches += 2;
  }
  CK(cudaGetLastError());
  // 4. prediction error on the training states -> candidate half-widths
  k_mlp_eval<<<(unsigned)std::min<int64_t>(nblk(n, kC2PThreads), 148 * 8), kC2PThreads, 0, s>>>(
      h->d_mlp, n, feat.as<float>(), pred.as<float>());
  ++h->launches;
  CK(cudaEventRecord(e1, s));
  std::vector<float> hp(n), ht(n), hl(2);
  CK(cudaMemcpyAsync(hp.data(), pred.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ht.data(), tgt.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&hl[0], loss.as<float>(), sizeof(float), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&hl[1], loss.as<float>() + C.steps - 1, sizeof(float), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  float tms = 0.f;
  cudaEventElapsedTime(&tms, e0, e1);
  R.train_ms = tms;
  R.loss_first = hl[0];
  R.loss_last = hl[1];
  std::vector<float> err;
  err.reserve(n);
  for (int64_t t = 0; t < n; ++t)
    if (std::isfinite(ht[t])) err.push_back(std::fabs(hp[t] - ht[t]));
  auto quant = [&](double q) {
    const size_t k = std::min(err.size() - 1, (size_t)(q * (double)(err.size() - 1)));
    std::nth_element(err.begin(), err.begin() + k, err.end());
    return err[k];
  };
  R.err_q50 = quant(0.5);
  R.err_q90 = quant(0.9);
  R.err_q99 = quant(0.99);
  R.err_q999 = quant(0.999);
  const float q9999 = quant(0.9999);
  R.err_max = *std::max_element(err.begin(), err.end());
  const float cand[4] = {1.2f * R.err_q90, 1.2f * R.err_q99, 1.2f * R.err_q999, 1.2f * q9999};
  // 5. choose delta on the calibration states by the learned c2p's cost in
  // Brent iterations as warps see it (deterministic), and time each choice
  h->mlp_ready = true;
  const int64_t nc = std::min<int64_t>(n, C.calib_states > 0 ? C.calib_states : n);
  DevBuf its, used;
  CK(cudaMalloc(&its.p, sizeof(int32_t) * (size_t)nc));
  CK(cudaMalloc(&used.p, sizeof(int8_t) * (size_t)nc));
  std::vector<int32_t> hits((size_t)nc);
  std::vector<int8_t> hused((size_t)nc);
  int best = 0;
  for (int ci = 0; ci < 4; ++ci) {
    const float dlt = std::max(cand[ci], 1e-6f);
    R.delta_cand[ci] = dlt;
    CK(cudaMemcpyAsync(h->d_mlp + kMlpOffNorm + 2 * kMlpIn + 2, &dlt, sizeof(float), cudaMemcpyHostToDevice, s));
    if (int rc = pack_mlp(h, s)) return rc;
    grb_c2p_diag cd{its.as<int32_t>(), used.as<int8_t>(), nullptr, nullptr};
    if (int rc = launch_c2p(h, nc, cons, metric, prims.as<double>(), nullptr, nullptr, true, &cd, s)) return rc;
    CK(cudaMemcpyAsync(hits.data(), its.p, sizeof(int32_t) * (size_t)nc, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hused.data(), used.p, sizeof(int8_t) * (size_t)nc, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double cost = 0.0;
    int64_t warps = 0;
    for (int64_t w0 = 0; w0 < nc; w0 += 32, ++warps) {
      int32_t m = 0;
      for (int64_t t = w0; t < std::min<int64_t>(nc, w0 + 32); ++t)
        m = std::max<int32_t>(m, hits[(size_t)t] + (hused[(size_t)t] ? 0 : 1));
      cost += m;
    }
    R.calib_cost[ci] = (float)(cost / (double)std::max<int64_t>(warps, 1));
    float bestms = 1e30f;
    for (int rep_i = 0; rep_i < 3; ++rep_i) {
      CK(cudaEventRecord(e0, s));
      if (int rc = launch_c2p(h, nc, cons, metric, prims.as<double>(), nullptr, nullptr, true, nullptr, s)) return rc;
      CK(cudaEventRecord(e1, s));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      bestms = std::min(bestms, ms);
    }
    R.calib_ms[ci] = bestms;
    if (R.calib_cost[ci] < R.calib_cost[best]) best = ci;
  }
  R.delta = R.delta_cand[best];
  CK(cudaMemcpyAsync(h->d_mlp + kMlpOffNorm + 2 * kMlpIn + 2, &R.delta, sizeof(float), cudaMemcpyHostToDevice, s));
  if (int rc = pack_mlp(h, s)) return rc;
  CK(cudaStreamSynchronize(s));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rep) *rep = R;
  return GRB_OK;
}

int grb_c2p_model_get(grb_handle* h, float* params, int64_t nparams) {
  if (!h) return GRB_ERR_INVALID;
  if (!params || nparams != kMlpNumParams) return fail(h, GRB_ERR_INVALID);
  if (!h->mlp_ready) return fail(h, GRB_ERR_NO_MODEL);
  CK(cudaMemcpy(params, h->d_mlp, sizeof(float) * kMlpNumParams, cudaMemcpyDeviceToHost));
  return GRB_OK;
}

int grb_c2p_model_set(grb_handle* h, const float* params, int64_t nparams) {
  if (!h) return GRB_ERR_INVALID;
  if (!params || nparams != kMlpNumParams) return fail(h, GRB_ERR_INVALID);
  for (int k = 0; k < kMlpNumParams; ++k)
    if (!std::isfinite(params[k])) return fail(h, GRB_ERR_INVALID);
  for (int k = 0; k < kMlpIn; ++k)
    if (!(params[kMlpOffNorm + kMlpIn + k] > 0.f)) return fail(h, GRB_ERR_INVALID);
  if (!(params[kMlpOffNorm + 2 * kMlpIn + 1] > 0.f) || !(params[kMlpOffNorm + 2 * kMlpIn + 2] > 0.f))
    return fail(h, GRB_ERR_INVALID);
  if (int rc = ensure_mlp(h)) return rc;
  CK(cudaMemcpy(h->d_mlp, params, sizeof(float) * kMlpNumParams, cudaMemcpyHostToDevice));
  if (int rc = pack_mlp(h, 0)) return rc;
  CK(cudaDeviceSynchronize());
  h->mlp_ready = true;
  return GRB_OK;
}

// Ghost runs of k_ghost_runs for this block geometry (ghost width 4,
// interiors multiples of 4 along x, blocks up to 255 rows a side), built
// now if needed and possible (not inside a stream capture); false when the
// run form does not apply.
static bool ghost_runs(grb_handle* h, const Geo& G, cudaStream_t s) {
  if (G.g != 4 || G.nx % 4 || G.NY + 1 > 255 || G.NZ + 1 > 255 || G.NX / 4 > 255) return false;
  const int key[4] = {G.nx, G.ny, G.nz, G.g};
  if (h->d_ghostruns && std::equal(key, key + 4, h->ghost_key)) return true;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
  std::vector<uint32_t> v;
  int off[3], cnt[3];
  const int nr = G.NX / 4;
  for (int a = 0; a < 3; ++a) {  // cells, faces staggered along y, z
    const int N1 = G.NY + (a == 1), N2 = G.NZ + (a == 2);
    const int hi1 = G.ny + G.g + (a == 1), hi2 = G.nz + G.g + (a == 2);
    off[a] = (int)v.size();
    for (int k = 0; k < N2; ++k)
      for (int j = 0; j < N1; ++j) {
        const bool row_ghost = j < G.g || j >= hi1 || k < G.g || k >= hi2;
        for (int r = 0; r < nr; ++r)
          if (row_ghost || r == 0 || r == nr - 1)
            v.push_back((uint32_t)r | (uint32_t)j << 8 | (uint32_t)k << 16);
      }
    cnt[a] = (int)v.size() - off[a];
  }
  uint32_t* d = nullptr;
  if (cudaMalloc(&d, v.size() * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (cudaMemcpy(d, v.data(), v.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    cudaGetLastError();
    return false;
  }
  cudaFree(h->d_ghostruns);
  h->d_ghostruns = d;
  std::copy(off, off + 3, h->ghost_off);
  std::copy(cnt, cnt + 3, h->ghost_cnt);
  std::copy(key, key + 4, h->ghost_key);
  return true;
}

int grb_fill_ghosts_brick(grb_handle* h, const grb_grid* g, const grb_fields* f, int32_t nbx,
                          int32_t nby, int32_t nbz, const int32_t* periodic, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g) return fail(h, GRB_ERR_INVALID);
  return grb_fill_ghosts_brick_range(h, g, f, nbx, nby, nbz, periodic, 0, g->nq, stream);
}

int grb_fill_ghosts_brick_range(grb_handle* h, const grb_grid* g, const grb_fields* f, int32_t nbx,
                                int32_t nby, int32_t nbz, const int32_t* periodic, int64_t q_begin,
                                int64_t q_end, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g || !f || !f->state || !f->bx || !f->by || !f->bz || !periodic || g->ngz < 1 ||
      nbx < 1 || nby < 1 || nbz < 1 || (int64_t)nbx * nby * nbz != g->nq || g->nq > 65535 ||
      q_begin < 0 || q_end > g->nq || q_begin >= q_end)
    return fail(h, GRB_ERR_INVALID);
  Brick br;
  br.nbx = nbx; br.nby = nby; br.nbz = nbz;
  br.q0 = (int)q_begin;
  for (int a = 0; a < 3; ++a) br.periodic[a] = periodic[a] != 0;
  // the launches cover blocks [q_begin, q_end) (blockIdx.y from br.q0); the
  // geometry keeps the whole brick's nq
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  const unsigned nfill = (unsigned)(q_end - q_begin);
  cudaStream_t s = (cudaStream_t)stream;
  double* bf[3] = {f->bx, f->by, f->bz};
  KScope ks(h, s, GRB_KIND_GHOST);
  // cells of the largest array (a face array)
  const int64_t total = (int64_t)std::max({G.NX + 1, G.NY + 1, G.NZ + 1}) *
                        std::max({G.NX * G.NY, G.NY * G.NZ, G.NX * G.NZ});
  if (total > (1ll << 31) - 256) return fail(h, GRB_ERR_INVALID);
  GhostDivs D;
  for (int a = 0; a < 4; ++a) {
    D.x[a] = make_fastdiv((uint32_t)(G.NX + (a == 1)));
    D.y[a] = make_fastdiv((uint32_t)(G.NY + (a == 2)));
  }
  const bool aligned = (((uintptr_t)f->state | (uintptr_t)bf[1] | (uintptr_t)bf[2]) & 15) == 0;
  if (aligned && ghost_runs(h, G, s)) {
    // 4-cell runs for the cells and the y, z face arrays; the x face array
    // (rows of NX+1) by rows
    const int* o = h->ghost_off;
    const int* c = h->ghost_cnt;
    const int mx = std::max({c[0], c[1], c[2]});
    const dim3 gr((unsigned)((mx + 127) / 128), nfill, 3u);
    k_ghost_runs<<<gr, 128, 0, s>>>(G, br, h->d_ghostruns, make_int3(o[0], o[1], o[2]), make_int3(c[0], c[1], c[2]),
                                    f->state, bf[1], bf[2]);
    const dim3 gx((unsigned)((G.NY * G.NZ + 127) / 128), nfill, 1u);
    k_ghost_xfaces<<<gx, 128, 0, s>>>(G, br, make_fastdiv((uint32_t)G.NY), bf[0]);
    h->launches += 2;
  } else {
    const dim3 grid((unsigned)((total + 255) / 256), nfill, 4u);
    k_ghost<<<grid, 256, 0, s>>>(G, br, D, f->state, bf[0], bf[1], bf[2]);
    ++h->launches;
  }
  CK(cudaGetLastError());
  return GRB_OK;
}


// Device view of a host array: the pointer the GPU uses for page-locked,
// mapped host memory, or null.
static double* host_view(double* p) {
  cudaPointerAttributes a;
  if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
  return static_cast<double*>(a.devicePointer);
}

int grb_copy_evolved_interior(grb_handle* h, const grb_grid* g, const grb_fields* host, int32_t host_state_nvars,
                              const grb_fields* dev, int32_t to_device, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g || !host || !dev || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->ngz < 1 || g->nq < 1 ||
      (host_state_nvars != GRB_N_HRSC && host_state_nvars != GRB_N_EVOL_VARS))
    return fail(h, GRB_ERR_INVALID);
  double* hv[4] = {host_view(host->state), host_view(host->bx), host_view(host->by), host_view(host->bz)};
  double* dv[4] = {dev->state, dev->bx, dev->by, dev->bz};
  for (int a = 0; a < 4; ++a)
    if (!hv[a] || !dv[a]) return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  if ((int64_t)GRB_N_HRSC * G.nq >= (1ll << 32) - 1) return fail(h, GRB_ERR_INVALID);
  cudaStream_t s = (cudaStream_t)stream;
  KScope ks(h, s, GRB_KIND_OTHER);
  for (int a = 0; a < 4; ++a) {
    int N[3] = {G.NX, G.NY, G.NZ}, n[3] = {G.nx, G.ny, G.nz};
    if (a > 0) { N[a - 1] += 1; n[a - 1] += 1; }
    const int nv = a == 0 ? GRB_N_HRSC : 1;
    const int64_t vstride = (int64_t)N[0] * N[1] * N[2];
    const int64_t qdev = vstride * (a == 0 ? GRB_N_EVOL_VARS : 1);
    const int64_t qhost = vstride * (a == 0 ? host_state_nvars : 1);
    double* dst = to_device ? dv[a] : hv[a];
    const double* src = to_device ? hv[a] : dv[a];
    const int64_t qd = to_device ? qdev : qhost, qs = to_device ? qhost : qdev;
    // whole rows of the interior (y, z) range; an upload stores only the
    // interior x, a download also the x-ghosts of those rows
    const Box b = box(0, G.g, G.g, N[0], n[1], n[2], (int64_t)nv * G.nq);
    const int xlo = to_device ? G.g : 0, xhi = to_device ? G.g + n[0] : N[0];
    k_copy_rows<<<nblk(b.count(), 256), 256, 0, s>>>(b, xlo, xhi, nv, make_fastdiv((uint32_t)nv), N[0], N[1],
                                                     vstride, qd, qs, dst, src);
    ++h->launches;
  }
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_set_static_metric(grb_handle* h, const grb_grid* g, const grb_fields* st, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!st) {
    cudaFree(h->d_metder);
    h->d_metder = nullptr;
    h->metder_bytes = 0;
    h->metder_idx = nullptr;
    h->metder_nq = 0;
    return GRB_OK;
  }
  if (!g || !st->state || !g->idx || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->ngz < 3 || g->nq < 1)
    return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  const size_t bytes = sizeof(double) * kMetDer * (size_t)G.nx * G.ny * G.nz * (size_t)G.nq;
  if (bytes > h->metder_bytes) {
    cudaFree(h->d_metder);
    h->d_metder = nullptr;
    h->metder_bytes = 0;
    if (cudaMalloc(&h->d_metder, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(h, GRB_ERR_NOMEM);
    }
    h->metder_bytes = bytes;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const Box b = box(G.g, G.g, G.g, G.nx, G.ny, G.nz, G.nq);
  k_metric_derivs<<<nblk(b.count(), 128), 128, 0, s>>>(G, b, st->state, g->idx, h->d_metder);
  ++h->launches;
  CK(cudaGetLastError());
  const int key[4] = {G.nx, G.ny, G.nz, G.g};
  std::copy(key, key + 4, h->metder_key);
  h->metder_nq = G.nq;
  h->metder_idx = g->idx;
  return GRB_OK;
}

int grb_copy_evolved_packed(grb_handle* h, const grb_grid* g, const grb_fields* host, const grb_fields* dev,
                            int32_t to_device, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g || !host || !dev || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->ngz < 1 || g->nq < 1)
    return fail(h, GRB_ERR_INVALID);
  double* hp[4] = {host->state, host->bx, host->by, host->bz};
  double* dp[4] = {dev->state, dev->bx, dev->by, dev->bz};
  for (int a = 0; a < 4; ++a)
    if (!hp[a] != !dp[a]) return fail(h, GRB_ERR_INVALID);  // both null: array skipped
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  if ((int64_t)GRB_N_HRSC * G.nq >= (1ll << 32) - 1) return fail(h, GRB_ERR_INVALID);
  cudaStream_t s = (cudaStream_t)stream;
  // packed sizes (doubles) and offsets of the four arrays in the staging:
  // each array and each direction has its own region, laid out for the
  // larger of this call's blocks and the reserved grid's (so calls on runs
  // of blocks find the same regions as whole-grid calls), and calls on
  // different streams that move different arrays, or the same array in
  // opposite directions, do not share staging
  const bool same_blocks = h->reserved && h->geo.nx == g->nx && h->geo.ny == g->ny && h->geo.nz == g->nz &&
                           h->geo.g == g->ngz;
  const int64_t nq_lay = same_blocks ? std::max(G.nq, h->geo.nq) : G.nq;
  int64_t cnt[4], off[4], tot = 0;
  for (int a = 0; a < 4; ++a) {
    int n[3] = {G.nx, G.ny, G.nz};
    if (a > 0) n[a - 1] += 1;
    const int64_t per_q = (int64_t)n[0] * n[1] * n[2] * (a == 0 ? GRB_N_HRSC : 1);
    cnt[a] = per_q * G.nq;
    off[a] = tot;
    tot += (per_q * nq_lay + 31) / 32 * 32;  // 256-byte aligned starts
  }
  if (cnt[0] >= (1ll << 32)) return fail(h, GRB_ERR_INVALID);
  if (to_device)
    for (int a = 0; a < 4; ++a) off[a] += tot;
  const size_t bytes = sizeof(double) * (size_t)(2 * tot);
  if (bytes > h->stage_io_bytes) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
      return fail(h, GRB_ERR_INVALID);  // first call must come before any capture
    cudaFree(h->d_stage_io);
    h->d_stage_io = nullptr;
    h->stage_io_bytes = 0;
    if (cudaMalloc(&h->d_stage_io, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(h, GRB_ERR_NOMEM);
    }
    h->stage_io_bytes = bytes;
  }
  KScope ks(h, s, GRB_KIND_OTHER);
  for (int a = 0; a < 4; ++a) {
    if (!hp[a]) continue;
    int N[3] = {G.NX, G.NY, G.NZ}, n[3] = {G.nx, G.ny, G.nz};
    if (a > 0) { N[a - 1] += 1; n[a - 1] += 1; }
    const int nv = a == 0 ? GRB_N_HRSC : 1;
    const int64_t vstride = (int64_t)N[0] * N[1] * N[2];
    const int64_t qdev = vstride * (a == 0 ? GRB_N_EVOL_VARS : 1);
    const Box b = box(G.g, G.g, G.g, n[0], n[1], n[2], (int64_t)nv * G.nq);
    double* stg = h->d_stage_io + off[a];
    const size_t nb = sizeof(double) * (size_t)cnt[a];
    if (to_device) {
      CK(cudaMemcpyAsync(stg, hp[a], nb, cudaMemcpyHostToDevice, s));
      k_pack_interior<<<nblk(b.count(), 256), 256, 0, s>>>(b, nv, make_fastdiv((uint32_t)nv), N[0], N[1],
                                                           vstride, qdev, false, dp[a], stg);
    } else {
      k_pack_interior<<<nblk(b.count(), 256), 256, 0, s>>>(b, nv, make_fastdiv((uint32_t)nv), N[0], N[1],
                                                           vstride, qdev, true, dp[a], stg);
      CK(cudaMemcpyAsync(hp[a], stg, nb, cudaMemcpyDeviceToHost, s));
    }
    ++h->launches;
  }
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_restrict_to_coarse(grb_handle* h, const grb_grid* g, const grb_fields* fine, const grb_fields* cbuf,
                           int64_t nquads, const int64_t* src_q, const int64_t* dst_q, const uint8_t* child_id,
                           const int32_t* vars_lo, int32_t nlo, const int32_t* vars_ho, int32_t nho,
                           void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g || !fine || !cbuf || nquads < 0 || g->nx < 2 || g->ny < 2 || g->nz < 2 || g->ngz < 3 ||
      g->nx % 2 || g->ny % 2 || g->nz % 2 || nlo < 0 || nho < 0 || nlo > GRB_N_EVOL_VARS ||
      nho > GRB_N_EVOL_VARS || (nlo && !vars_lo) || (nho && !vars_ho) || !src_q || !dst_q)
    return fail(h, GRB_ERR_INVALID);
  if (nquads == 0) return GRB_OK;
  if (nho && !child_id) return fail(h, GRB_ERR_INVALID);
  // the 5-point stencils reach 3 fine cells beyond the interior's edge cell
  if (nho && (g->nx < 4 || g->ny < 4 || g->nz < 4)) return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, nquads);
  cudaStream_t s = (cudaStream_t)stream;
  KScope ks(h, s, GRB_KIND_OTHER);
  for (int pass = 0; pass < 2; ++pass) {
    const int nl = pass == 0 ? nlo : nho;
    const int32_t* vl = pass == 0 ? vars_lo : vars_ho;
    if (!nl) continue;
    if (!fine->state || !cbuf->state) return fail(h, GRB_ERR_INVALID);
    RestrictVars V{};
    V.n = nl;
    for (int t = 0; t < nl; ++t) {
      if (vl[t] < 0 || vl[t] >= GRB_N_EVOL_VARS) return fail(h, GRB_ERR_INVALID);
      V.v[t] = vl[t];
    }
    if ((int64_t)nl * nquads >= (1ll << 32)) return fail(h, GRB_ERR_INVALID);
    const Box b = box(0, 0, 0, G.nx / 2, G.ny / 2, G.nz / 2, (int64_t)nl * nquads);
    if (pass == 0)
      k_restrict_cells<false><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, V, make_fastdiv((uint32_t)nl), fine->state,
                                                                   cbuf->state, src_q, dst_q, child_id);
    else if (G.nz >= 6) {
      // by z columns; with 4 cells along z the edge stencils' windows move
      // back along z, so those blocks keep one thread per coarse cell
      const Box bc = box(0, 0, 0, G.nx / 2, G.ny / 2, 1, (int64_t)nl * nquads);
      k_restrict_lag_zcol<<<nblk(bc.count(), 128), 128, 0, s>>>(G, bc, V, make_fastdiv((uint32_t)nl), fine->state,
                                                               cbuf->state, src_q, dst_q, child_id);
    } else
      k_restrict_cells<true><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, V, make_fastdiv((uint32_t)nl), fine->state,
                                                                  cbuf->state, src_q, dst_q, child_id);
    ++h->launches;
  }
  const double* fs[3] = {fine->bx, fine->by, fine->bz};
  double* cs[3] = {cbuf->bx, cbuf->by, cbuf->bz};
  for (int d = 0; d < 3; ++d) {
    if (!fs[d] && !cs[d]) continue;
    if (!fs[d] || !cs[d]) return fail(h, GRB_ERR_INVALID);
    const Box b = box(0, 0, 0, G.nx / 2 + (d == 0), G.ny / 2 + (d == 1), G.nz / 2 + (d == 2), nquads);
    if (d == 0) k_restrict_faces<0><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, fs[d], cs[d], src_q, dst_q);
    if (d == 1) k_restrict_faces<1><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, fs[d], cs[d], src_q, dst_q);
    if (d == 2) k_restrict_faces<2><<<nblk(b.count(), 128), 128, 0, s>>>(G, b, fs[d], cs[d], src_q, dst_q);
    ++h->launches;
  }
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_prolong_to_ghosts(grb_handle* h, const grb_grid* g, const grb_fields* fine, const grb_fields* cbuf,
                          int32_t elem_kind, int64_t nelems, const int64_t* fine_q, const int64_t* cbuf_q,
                          const uint8_t* elem_id, const int8_t* have_fine, const int32_t* vars_lo, int32_t nlo,
                          const int32_t* vars_ho, int32_t nho, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g || !fine || !cbuf || nelems < 0 || elem_kind < GRB_ELEM_FACE || elem_kind > GRB_ELEM_CORNER ||
      g->nx != g->ny || g->nx != g->nz || g->nx < 4 || g->nx % 2 || g->ngz < 4 || g->ngz % 2 || nlo < 0 ||
      nho < 0 || nlo > GRB_N_EVOL_VARS || nho > GRB_N_EVOL_VARS || (nlo && !vars_lo) || (nho && !vars_ho) ||
      !fine_q || !cbuf_q || !elem_id)
    return fail(h, GRB_ERR_INVALID);
  if (nelems == 0) return GRB_OK;
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, nelems);
  const int n = g->nx, ng = g->ngz;
  const int ext[3] = {ng, elem_kind == GRB_ELEM_FACE ? n : ng, elem_kind == GRB_ELEM_CORNER ? ng : n};
  RestrictVars V[2] = {};
  for (int pass = 0; pass < 2; ++pass) {
    const int nl = pass == 0 ? nlo : nho;
    const int32_t* vl = pass == 0 ? vars_lo : vars_ho;
    if (!nl) continue;
    if (!fine->state || !cbuf->state || (int64_t)nl * nelems >= (1ll << 32)) return fail(h, GRB_ERR_INVALID);
    V[pass].n = nl;
    for (int t = 0; t < nl; ++t) {
      if (vl[t] < 0 || vl[t] >= GRB_N_EVOL_VARS) return fail(h, GRB_ERR_INVALID);
      V[pass].v[t] = vl[t];
    }
  }
  const bool faces = fine->bx || fine->by || fine->bz || cbuf->bx || cbuf->by || cbuf->bz;
  if (faces && (!fine->bx || !fine->by || !fine->bz || !cbuf->bx || !cbuf->by || !cbuf->bz || !have_fine))
    return fail(h, GRB_ERR_INVALID);
  cudaStream_t s = (cudaStream_t)stream;
  KScope ks(h, s, GRB_KIND_OTHER);
  if (elem_kind == GRB_ELEM_FACE)
    launch_prolong<GRB_ELEM_FACE>(G, ext, fine, cbuf, nelems, fine_q, cbuf_q, elem_id, have_fine, V, faces, s);
  else if (elem_kind == GRB_ELEM_EDGE)
    launch_prolong<GRB_ELEM_EDGE>(G, ext, fine, cbuf, nelems, fine_q, cbuf_q, elem_id, have_fine, V, faces, s);
  else
    launch_prolong<GRB_ELEM_CORNER>(G, ext, fine, cbuf, nelems, fine_q, cbuf_q, elem_id, have_fine, V, faces, s);
  h->launches += (V[0].n > 0) + (V[1].n > 0) + 2 * faces;
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_accumulate_boundary_outflow(grb_handle* h, const grb_grid* g, int64_t nfaces, const int64_t* quad,
                                    const uint8_t* face, const double* dx, double dt, double dtfact,
                                    double* outflow, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  int rc = check_grid(h, g);
  if (rc) return fail(h, rc);
  if (nfaces < 0 || nfaces > 0x7fffffff || !outflow || (nfaces && (!quad || !face || !dx)))
    return fail(h, GRB_ERR_INVALID);
  if (nfaces == 0) return GRB_OK;
  if (!h->B.flux) return fail(h, GRB_ERR_NOT_RESERVED);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  cudaStream_t s = (cudaStream_t)stream;
  KScope ks(h, s, GRB_KIND_OTHER);
  k_boundary_outflow<<<(unsigned)nfaces, kOutflowThreads, 0, s>>>(G, h->B.flux, quad, face, dx, dt * dtfact, outflow);
  ++h->launches;
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_fill_ghosts_gather(grb_handle* h, const grb_grid* g, const grb_fields* f, const grb_gather* cells,
                           int32_t nvars, const grb_gather* faces, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  if (!g || !f || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->nq < 1 || g->ngz < 1 || nvars < 0 ||
      nvars > GRB_N_EVOL_VARS)
    return fail(h, GRB_ERR_INVALID);
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq);
  cudaStream_t s = (cudaStream_t)stream;
  KScope ks(h, s, GRB_KIND_GHOST);
  auto ok = [](const grb_gather* m) {
    return m->n >= 0 && m->n < (1ll << 40) && (m->n == 0 || (m->cnt && m->dst && m->src && m->w));
  };
  if (cells && nvars > 0 && cells->n > 0) {
    if (!ok(cells) || !f->state) return fail(h, GRB_ERR_INVALID);
    const dim3 gr(nblk(cells->n, 256), (unsigned)nvars);
    k_ghost_gather<<<gr, 256, 0, s>>>(cells->n, G.cells, cells->cnt, cells->dst, cells->src, cells->w, f->state);
    ++h->launches;
  }
  if (faces) {
    double* arr[3] = {f->bx, f->by, f->bz};
    const int64_t per[3] = {(int64_t)(G.NX + 1) * G.NY * G.NZ, (int64_t)G.NX * (G.NY + 1) * G.NZ,
                            (int64_t)G.NX * G.NY * (G.NZ + 1)};  // one variable of a block
    for (int d = 0; d < 3; ++d) {
      const grb_gather& m = faces[d];
      if (m.n <= 0) continue;
      if (!ok(&m) || !arr[d]) return fail(h, GRB_ERR_INVALID);
      k_ghost_gather<<<nblk(m.n, 256), 256, 0, s>>>(m.n, per[d], m.cnt, m.dst, m.src, m.w, arr[d]);
      ++h->launches;
    }
  }
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_set_reflux(grb_handle* h, const grb_reflux* r) {
  if (!h) return GRB_ERR_INVALID;
  if (!r || (r->nfaces == 0 && r->nsame_faces == 0 && r->nedges == 0 && r->nsame_edges == 0)) {
    h->reflux = false;
    h->rf = RefluxDev{};
    return GRB_OK;
  }
  if (!h->reserved) return fail(h, GRB_ERR_NOT_RESERVED);
  const Geo& G = h->geo;
  if (G.nx != G.ny || G.nx != G.nz || G.nx % 2 || r->nfaces < 0 || r->nsame_faces < 0 || r->nedges < 0 ||
      r->nsame_edges < 0)
    return fail(h, GRB_ERR_INVALID);
  if ((r->nfaces && (!r->face_coarse_q || !r->face_coarse_id || !r->face_fine_q)) ||
      (r->nsame_faces && (!r->same_face_q || !r->same_face_id)) ||
      (r->nedges && (!r->edge_nsides || !r->edge_id || !r->edge_is_fine || !r->edge_q || !r->edge_off)) ||
      (r->nsame_edges && (!r->same_edge_nsides || !r->same_edge_id || !r->same_edge_q)))
    return fail(h, GRB_ERR_INVALID);
  const size_t need = sizeof(double) * (size_t)G.nx * (2 * (size_t)r->nedges + (size_t)r->nsame_edges);
  if (need > h->refacc_bytes) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(nullptr, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
      return fail(h, GRB_ERR_INVALID);
    cudaFree(h->d_refacc);
    h->d_refacc = nullptr;
    h->refacc_bytes = 0;
    if (cudaMalloc(&h->d_refacc, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(h, GRB_ERR_NOMEM);
    }
    h->refacc_bytes = need;
  }
  RefluxDev R{};
  R.nfaces = r->nfaces; R.face_cq = r->face_coarse_q; R.face_cid = r->face_coarse_id; R.face_fq = r->face_fine_q;
  R.nsame = r->nsame_faces; R.same_q = r->same_face_q; R.same_id = r->same_face_id;
  R.nedges = r->nedges; R.edge_ns = r->edge_nsides; R.edge_id = r->edge_id; R.edge_fine = r->edge_is_fine;
  R.edge_q = r->edge_q; R.edge_off = r->edge_off;
  R.nsame_edges = r->nsame_edges; R.sedge_ns = r->same_edge_nsides; R.sedge_id = r->same_edge_id;
  R.sedge_q = r->same_edge_q;
  R.acc_edges = h->d_refacc;
  R.acc_same_edges = h->d_refacc + (size_t)G.nx * 2 * (size_t)r->nedges;
  h->rf = R;
  h->reflux_flux_same = r->same_level_flux_average != 0;
  h->reflux = true;
  return GRB_OK;
}

int grb_set_fofc_list_capacity(grb_handle* h, int64_t faces) {
  if (!h || faces < 0) return fail(h, GRB_ERR_INVALID);
  if (!h->reserved) return fail(h, GRB_ERR_NOT_RESERVED);
  h->B.fcap = (uint32_t)std::min<int64_t>(faces, h->fcap_alloc);
  return GRB_OK;
}

int grb_set_mode(grb_handle* h, int32_t mode) {
  if (!h || (mode != GRB_MODE_PLAIN && mode != GRB_MODE_TUNED)) return GRB_ERR_INVALID;
  h->mode = mode;
  return GRB_OK;
}

// Time the register-cap variants of the heavy kernels on device copies of
// the first blocks of the grid (live arrays are only read) and keep the
// fastest per kernel family for the tuned mode.
int grb_autotune(grb_handle* h, const grb_grid* g, const grb_fields* nw, const grb_fields* old,
                 const double* aux, void* stream) {
  if (!h) return GRB_ERR_INVALID;
  int rc = check_grid(h, g);
  if (rc) return fail(h, rc);
  if (!nw || !old || !aux) return fail(h, GRB_ERR_INVALID);
  cudaStream_t s = (cudaStream_t)stream;
  // a sample of nt blocks spread evenly over the grid (block k*nq/nt), so
  // that the candidates see every level of a hierarchy, not only its first
  const int64_t nt = g->nq < 96 ? g->nq : 96;
  const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, nt);
  const size_t c1 = sizeof(double) * G.cells;  // one variable of one block
  const size_t cs = c1 * nt;
  const size_t f1[3] = {sizeof(double) * (size_t)(G.NX + 1) * G.NY * G.NZ,
                        sizeof(double) * (size_t)G.NX * (G.NY + 1) * G.NZ,
                        sizeof(double) * (size_t)G.NX * G.NY * (G.NZ + 1)};
  const size_t fsz[3] = {f1[0] * nt, f1[1] * nt, f1[2] * nt};
  double *ns = nullptr, *os = nullptr, *ax = nullptr, *b3[6] = {nullptr};
  double *pns = nullptr, *pax = nullptr, *pb3[3] = {nullptr}, *sidx = nullptr, *scrd = nullptr;
  bool ok = cudaMalloc(&ns, cs * GRB_N_EVOL_VARS) == cudaSuccess &&
            cudaMalloc(&os, cs * GRB_N_EVOL_VARS) == cudaSuccess &&
            cudaMalloc(&ax, cs * GRB_N_AUX_VARS) == cudaSuccess &&
            cudaMalloc(&pns, cs * GRB_N_EVOL_VARS) == cudaSuccess &&
            cudaMalloc(&pax, cs * GRB_N_AUX_VARS) == cudaSuccess &&
            cudaMalloc(&sidx, sizeof(double) * 3 * nt) == cudaSuccess &&
            (!g->coords || cudaMalloc(&scrd, sizeof(double) * 3 * nt) == cudaSuccess);
  for (int a = 0; a < 6 && ok; ++a) ok = cudaMalloc(&b3[a], fsz[a % 3]) == cudaSuccess;
  for (int a = 0; a < 3 && ok; ++a) ok = cudaMalloc(&pb3[a], fsz[a]) == cudaSuccess;
  auto cleanup = [&]() {
    cudaFree(ns); cudaFree(os); cudaFree(ax); cudaFree(pns); cudaFree(pax); cudaFree(sidx); cudaFree(scrd);
    for (int a = 0; a < 6; ++a) cudaFree(b3[a]);
    for (int a = 0; a < 3; ++a) cudaFree(pb3[a]);
  };
  if (!ok) { cleanup(); cudaGetLastError(); return fail(h, GRB_ERR_NOMEM); }
  const double* srcb[6] = {nw->bx, nw->by, nw->bz, old->bx, old->by, old->bz};
  for (int64_t k = 0; k < nt; ++k) {
    const int64_t q = k * g->nq / nt;
    cudaMemcpyAsync(ns + k * G.cells * GRB_N_EVOL_VARS, nw->state + q * G.cells * GRB_N_EVOL_VARS,
                    c1 * GRB_N_EVOL_VARS, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(os + k * G.cells * GRB_N_EVOL_VARS, old->state + q * G.cells * GRB_N_EVOL_VARS,
                    c1 * GRB_N_EVOL_VARS, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(ax + k * G.cells * GRB_N_AUX_VARS, aux + q * G.cells * GRB_N_AUX_VARS, c1 * GRB_N_AUX_VARS,
                    cudaMemcpyDeviceToDevice, s);
    for (int a = 0; a < 6; ++a) {
      const size_t e = f1[a % 3] / sizeof(double);
      cudaMemcpyAsync(b3[a] + k * e, srcb[a] + q * e, f1[a % 3], cudaMemcpyDeviceToDevice, s);
    }
    cudaMemcpyAsync(sidx + 3 * k, g->idx + 3 * q, 3 * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (scrd) cudaMemcpyAsync(scrd + 3 * k, g->coords + 3 * q, 3 * sizeof(double), cudaMemcpyDeviceToDevice, s);
  }
  // pristine copies of what the candidates modify
  cudaMemcpyAsync(pns, ns, cs * GRB_N_EVOL_VARS, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(pax, ax, cs * GRB_N_AUX_VARS, cudaMemcpyDeviceToDevice, s);
  for (int a = 0; a < 3; ++a) cudaMemcpyAsync(pb3[a], b3[a], fsz[a], cudaMemcpyDeviceToDevice, s);
  grb_fields fn{ns, b3[0], b3[1], b3[2]}, fo{os, b3[3], b3[4], b3[5]};
  grb_grid gs = *g;
  gs.nq = nt;
  gs.idx = sidx;
  gs.coords = scrd;
  // the static-metric cache of the first nt blocks stands in for the
  // sample's (the timing reads it the same way; the values do not matter)
  const double* md = static_metric(h, make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq), g->idx);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const bool timing = h->timing;
  h->timing = false;
  const DevParams& P = h->dp;
  StageBufs B = h->B;
  // restore the copies before every launch so that each candidate sees the
  // same input (the update and aux kernels modify their arrays)
  auto restore = [&]() {
    cudaMemcpyAsync(ns, pns, cs * GRB_N_EVOL_VARS, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(ax, pax, cs * GRB_N_AUX_VARS, cudaMemcpyDeviceToDevice, s);
    for (int a = 0; a < 3; ++a) cudaMemcpyAsync(b3[a], pb3[a], fsz[a], cudaMemcpyDeviceToDevice, s);
  };
  auto time_it = [&](auto&& fn_launch) {
    restore();
    fn_launch();  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
      restore();
      cudaEventRecord(e0, s);
      fn_launch();
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      best = t < best ? t : best;
    }
    return best;
  };
  const int gz = G.g;
  // face fluxes along x with the tuned range
  int lo[3] = {gz - 1, gz - 1, gz - 1}, n[3] = {G.nx + 3, G.ny + 2, G.nz + 2};
  if (P.emf == GRB_EMF_UCT) { lo[1] = lo[2] = gz - 3; n[1] = G.ny + 6; n[2] = G.nz + 6; }
  const Box fbx = box(lo[0], lo[1], lo[2], n[0], n[1], n[2], nt);
  const Box fb = box(gz - 1, gz - 1, gz - 1, G.nx + 2, G.ny + 2, G.nz + 2, nt);
  const Box ub = box(gz, gz, gz, G.nx, G.ny, G.nz, nt);
  Box ab = trimmed(h) ? tuned_aux_box(h, G, s) : box(0, 0, 0, G.NX, G.NY, G.NZ, nt);
  ab.nq = nt;
  int best[4] = {0, 0, 0, 0};
  for (int fam = 0; fam < 4; ++fam) {
    float bt = 1e30f;
    for (int v = 0; v < kNumVar; ++v) {
      float t = 0.f;
      if (fam == 0)
        t = time_it([&] { launch_flux_tuned<0>(v, nblk(fbx.count(), 128), s, P, G, fbx, os, ax, fo.bx, B); });
      else if (fam == 1)
        t = time_it([&] { launch_flag_tuned(v, nblk(fb.count(), 128), s, P, G, fb, 1e-3, 1.0, ns, os, fo.bx,
                                            fo.by, fo.bz, gs.idx, gs.coords, B); });
      else if (fam == 2)
        t = time_it([&] { launch_update_tuned(v, nblk(ub.count(), 128), s, P, G, ub, 1e-12, 1.0, ns, os, ax,
                                              gs.idx, B, md); });
      else
        t = time_it([&] { launch_aux_tuned(v, nblk(ab.count(), 128), s, P, G, ab, ns, fn.bx, fn.by, fn.bz,
                                           ax, gs.idx, gs.coords, B); });
      h->tune_ms[fam][v] = t;
      if (t < bt) { bt = t; best[fam] = v; }
    }
  }
  // the work-queue forms of the chosen candidates of every family
  h->tune_flux_queue_ms = time_it([&] {
    launch_flux_tuned<0>(best[0] + 3, nblk(fbx.count(), 128), s, P, G, fbx, os, ax, fo.bx, B, h->d_queue + 2);
  });
  if (h->tune_flux_queue_ms < h->tune_ms[0][best[0]]) best[0] += 3;
  h->tune_update_queue_ms = time_it([&] {
    launch_update_tuned(best[2] + 3, nblk(ub.count(), 128), s, P, G, ub, 1e-12, 1.0, ns, os, ax, gs.idx, B, md,
                        h->d_queue + 3);
  });
  if (h->tune_update_queue_ms < h->tune_ms[2][best[2]]) best[2] += 3;
  h->tune_flag_queue_ms = time_it([&] {
    launch_flag_tuned(best[1] + 3, nblk(fb.count(), 128), s, P, G, fb, 1e-3, 1.0, ns, os, fo.bx, fo.by, fo.bz,
                      gs.idx, gs.coords, B, h->d_queue + 1);
  });
  if (h->tune_flag_queue_ms < h->tune_ms[1][best[1]]) best[1] += 3;
  h->tune_aux_queue_ms = time_it([&] {
    launch_aux_tuned(best[3] + 3, nblk(ab.count(), 128), s, P, G, ab, ns, fn.bx, fn.by, fn.bz, ax, gs.idx,
                     gs.coords, B, nullptr, h->d_queue);
  });
  // and the deferred-backup form of the same cap (its list allocated for the
  // whole grid's aux cells, and freed again if another form wins)
  const Box abig = trimmed(h) ? tuned_aux_box(h, make_geo(g->nx, g->ny, g->nz, g->ngz, g->nq), s)
                              : box(0, 0, 0, G.NX, G.NY, G.NZ, g->nq);
  float defer_ms = 1e30f;
  if (ensure_aux_defer(h, abig.count())) {
    B = h->B;
    defer_ms = time_it([&] {
      launch_aux_tuned(best[3] + 6, nblk(ab.count(), 128), s, P, G, ab, ns, fn.bx, fn.by, fn.bz, ax, gs.idx,
                       gs.coords, B);
    });
  }
  h->tune_aux_defer_ms = defer_ms;
  if (h->tune_aux_queue_ms < h->tune_ms[3][best[3]] && h->tune_aux_queue_ms <= defer_ms) best[3] += 3;
  else if (defer_ms < h->tune_ms[3][best[3]]) best[3] += 6;
  if (best[3] < 6) free_aux_defer(h);
  h->var_flux = best[0];
  h->var_flag = best[1];
  h->var_update = best[2];
  h->var_aux = best[3];
  h->autotuned = true;
  h->timing = timing;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(s);
  cleanup();
  CK(cudaGetLastError());
  return GRB_OK;
}

int grb_get_tuning(grb_handle* h, int32_t* variant, float* ms) {
  if (!h || !variant) return GRB_ERR_INVALID;
  variant[0] = kFluxMinB[h->var_flux % 3] + (kFluxTma[h->var_flux % 3] ? 100 : 0) + 1000 * (h->var_flux / 3);
  variant[1] = kMinBC2p[h->var_flag % 3] + 100 * (h->var_flag / 3);
  variant[2] = (h->d_metder ? kMinBCached[h->var_update % 3] : kMinB[h->var_update % 3]) + 100 * (h->var_update / 3);
  variant[3] = kMinBC2p[h->var_aux % 3] + 100 * (h->var_aux / 3);
  if (ms)
    for (int f = 0; f < 4; ++f)
      for (int v = 0; v < kNumVar; ++v) ms[f * kNumVar + v] = h->tune_ms[f][v];
  return GRB_OK;
}

int grb_get_tuning_forms(grb_handle* h, float* ms, int32_t n) {
  if (!h || !ms || n < 0) return GRB_ERR_INVALID;
  const float v[5] = {h->tune_flag_queue_ms, h->tune_aux_queue_ms, h->tune_aux_defer_ms, h->tune_flux_queue_ms,
                      h->tune_update_queue_ms};
  for (int i = 0; i < n && i < 5; ++i) ms[i] = v[i];
  return GRB_OK;
}

int grb_set_tuning(grb_handle* h, const int32_t* variant) {
  if (!h || !variant) return GRB_ERR_INVALID;
  for (int f = 0; f < 4; ++f)
    if (variant[f] < 0 || variant[f] >= (f == 3 ? 3 * kNumVar : 2 * kNumVar))
      return fail(h, GRB_ERR_INVALID);
  if (variant[3] >= 2 * kNumVar) {
    // the deferred-backup aux pass: its list, for the reserved grid
    if (!h->reserved) return fail(h, GRB_ERR_NOT_RESERVED);
    const Box ab = h->p.ranges == GRB_RANGES_NEXT_STAGE && h->dp.emf == GRB_EMF_GS
                       ? tuned_aux_box(h, h->geo, nullptr)
                       : box(0, 0, 0, h->geo.NX, h->geo.NY, h->geo.NZ, h->geo.nq);
    if (!ensure_aux_defer(h, ab.count())) return fail(h, GRB_ERR_NOMEM);
  }
  h->var_flux = variant[0];
  h->var_flag = variant[1];
  h->var_update = variant[2];
  h->var_aux = variant[3];
  h->autotuned = true;
  return GRB_OK;
}

// FP64 throughput probe: kFmaChains independent fused multiply-add chains
// per thread, iters steps each; the final values feed a store that never
// happens (their sum is never negative), so nothing is optimised away.
constexpr int kFmaChains = 8;
__global__ void __launch_bounds__(256) k_fp64_peak(int iters, double b, double c, double* __restrict__ sink) {
  double a[kFmaChains];
#pragma unroll
  for (int u = 0; u < kFmaChains; ++u) a[u] = 1.0 + 1e-9 * (threadIdx.x + 37 * u);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kFmaChains; ++u) a[u] = fma(a[u], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int u = 0; u < kFmaChains; ++u) s += a[u];
  if (s < 0.0) sink[blockIdx.x] = s;
}

int grb_measure_fp64_peak(double* tflops, double* ms_out, void* stream) {
  if (!tflops) return GRB_ERR_INVALID;
  grb_handle* h = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const unsigned grid = (unsigned)(sms * 8);
  const int iters = 1 << 14;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  k_fp64_peak<<<grid, 256, 0, s>>>(iters / 16, 0.9999999, 1e-7, nullptr);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0, s);
    k_fp64_peak<<<grid, 256, 0, s>>>(iters, 0.9999999, 1e-7, nullptr);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    best = t < best ? t : best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaGetLastError());
  const double flops = 2.0 * kFmaChains * (double)iters * grid * 256.0;
  *tflops = flops / (best * 1e-3) / 1e12;
  if (ms_out) *ms_out = best;
  return GRB_OK;
}

int grb_set_kernel_timing(grb_handle* h, int32_t enable) {
  if (!h) return GRB_ERR_INVALID;
  h->timing = enable != 0;
  return GRB_OK;
}

int grb_kernel_times(grb_handle* h, double* ms, int64_t* counts, int32_t nkinds) {
  if (!h || nkinds < GRB_KIND_COUNT) return GRB_ERR_INVALID;
  if (!h->marks.empty()) {
    CK(cudaEventSynchronize(h->marks.back().b));
    for (auto& m : h->marks) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, m.a, m.b));
      h->kind_ms[m.kind] += t;
      h->kind_n[m.kind] += 1;
      h->pool.push_back(m.a);
      h->pool.push_back(m.b);
    }
    h->marks.clear();
  }
  for (int k = 0; k < GRB_KIND_COUNT; ++k) {
    if (ms) ms[k] = h->kind_ms[k];
    if (counts) counts[k] = h->kind_n[k];
    h->kind_ms[k] = 0;
    h->kind_n[k] = 0;
  }
  return GRB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Scratch-free stage: grb_advance_substep_static.
//
// For callers that cannot call cudaMalloc: host codes whose device memory is
// entirely reserved up front by a pooling allocator (a Kokkos or RMM arena
// that owns the GPU), and plugin hosts that forbid a library from allocating
// device memory once the run has started.  The face/edge scratch of the
// stage lives in this file-scope device array instead of handle-owned
// memory.  Its size is fixed at GRB_STATIC_SCRATCH_BYTES; the stage runs
// over the blocks in chunks that fit, so the limit is per block: one block's
// scratch (about 30 doubles per face-grid point plus 3 per cell, ~4.2 MB for
// 16^3 blocks with 4 ghosts) must fit in the array.  Every GPU that loads the
// library holds the array until the process exits.
// ---------------------------------------------------------------------------
namespace {
static __device__ __align__(256) unsigned char g_static_scratch[GRB_STATIC_SCRATCH_BYTES];

// cell-centred E = -vtilde x B with B including sqrt(gamma)
// (auxiliaries.cpp:131-162), for the blocks of one chunk
__global__ void __launch_bounds__(128) k_ecenter_static(Geo G, Box box, const double* __restrict__ st,
                                                         const double* __restrict__ bx,
                                                         const double* __restrict__ by,
                                                         const double* __restrict__ bz,
                                                         const double* __restrict__ aux, double* __restrict__ ec) {
  int i, j, k;
  int64_t q;
  if (!decode(box, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k, q)) return;
  const Met m = cell_met(G, st, i, j, k, q);
  const int64_t a0 = cvar(G, i, j, k, 0, GRB_N_AUX_VARS, q);
  const double cbx = 0.5 * (bx[bxi(G, i, j, k, q)] + bx[bxi(G, i + 1, j, k, q)]);
  const double cby = 0.5 * (by[byi(G, i, j, k, q)] + by[byi(G, i, j + 1, k, q)]);
  const double cbz = 0.5 * (bz[bzi(G, i, j, k, q)] + bz[bzi(G, i, j, k + 1, q)]);
  const double z[3] = {aux[a0 + G.cells * GRB_ZVECX], aux[a0 + G.cells * GRB_ZVECY], aux[a0 + G.cells * GRB_ZVECZ]};
  const double W = sqrt(1. + sqs(m.g, z));
  double vt[3];
  for (int a = 0; a < 3; ++a) vt[a] = m.alp * z[a] / W - m.beta[a];
  ec[eci(G, i, j, k, 0, q)] = cby * vt[2] - cbz * vt[1];
  ec[eci(G, i, j, k, 1, q)] = -cbx * vt[2] + cbz * vt[0];
  ec[eci(G, i, j, k, 2, q)] = cbx * vt[1] - cby * vt[0];
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct StaticLayout {
  size_t flux, eface, vbar, ecenter, emf, ftag, etag, per_block;
};
StaticLayout static_layout(const Geo& G1, int emf_kind) {
  StaticLayout L{};
  L.flux = align256(sizeof(double) * G1.fcells * 7 * 3);
  L.eface = emf_kind == GRB_EMF_GS ? align256(sizeof(double) * G1.fcells * 2 * 3) : 0;
  L.vbar = emf_kind == GRB_EMF_UCT ? align256(sizeof(double) * G1.fcells * 4 * 3) : 0;
  L.ecenter = emf_kind == GRB_EMF_GS ? align256(sizeof(double) * G1.cells * 3) : 0;
  L.emf = align256(sizeof(double) * G1.fcells * 3);
  L.ftag = align256((size_t)G1.fcells * 3);
  L.etag = align256((size_t)G1.fcells * 3);
  L.per_block = L.flux + L.eface + L.vbar + L.ecenter + L.emf + L.ftag + L.etag;
  return L;
}
}  // namespace

extern "C" int grb_advance_substep_static(const grb_params* p, const grb_grid* g, double t,
                                          double dt, double dtfact, const grb_fields* nw,
                                          const grb_fields* old, const double* aux,
                                          void* stream) {
  (void)t;
  if (!valid_params(p)) return GRB_ERR_INVALID;
  if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->nq < 1 || g->ngz < 4 || !g->idx) return GRB_ERR_INVALID;
  if (p->excise_by_radius && !g->coords) return GRB_ERR_INVALID;
  if (!nw || !old || !aux || !nw->state || !nw->bx || !nw->by || !nw->bz || !old->state || !old->bx ||
      !old->by || !old->bz)
    return GRB_ERR_INVALID;
  const size_t header = 256;  // [0,16): FOFC counters, [16,20): status flags
  const Geo G1 = make_geo(g->nx, g->ny, g->nz, g->ngz, 1);
  const StaticLayout L = static_layout(G1, p->emf);
  if (L.per_block + header > (size_t)GRB_STATIC_SCRATCH_BYTES) {
    std::fprintf(stderr,
                 "grb_advance_substep_static: one %dx%dx%d block with %d ghosts needs %zu bytes of "
                 "scratch, above the static maximum of %zu bytes\n",
                 g->nx, g->ny, g->nz, g->ngz, L.per_block, (size_t)GRB_STATIC_SCRATCH_BYTES - header);
    return GRB_ERR_INVALID;
  }
  // The host-side name g_static_scratch is only a stand-in: the kernels need
  // the array's device address on the current device.  It is looked up on
  // every call (cheap, allocates nothing), so it stays right after a device
  // reset reloads the module.  On a device's first call this also loads the
  // module there, which is why that first call belongs before any capture.
  void* ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, g_static_scratch) != cudaSuccess || !ptr) return GRB_ERR_CUDA;
  unsigned char* base = static_cast<unsigned char*>(ptr);
  const DevParams P = to_dev(*p);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t chunk = (int64_t)((GRB_STATIC_SCRATCH_BYTES - header) / L.per_block);
  const int gz = G1.g, T = 128;
  StageBufs B{};
  B.counters = reinterpret_cast<unsigned long long*>(base);
  B.flags = reinterpret_cast<uint32_t*>(base + 16);
  if (cudaMemsetAsync(base, 0, header, s) != cudaSuccess) return GRB_ERR_CUDA;
  const int64_t cst = G1.cells, bxs = (int64_t)(G1.NX + 1) * G1.NY * G1.NZ,
                bys = (int64_t)G1.NX * (G1.NY + 1) * G1.NZ, bzs = (int64_t)G1.NX * G1.NY * (G1.NZ + 1);
  for (int64_t q0 = 0; q0 < g->nq; q0 += chunk) {
    const int64_t nq = (g->nq - q0 < chunk) ? g->nq - q0 : chunk;
    const Geo G = make_geo(g->nx, g->ny, g->nz, g->ngz, nq);
    unsigned char* c = base + header;
    B.flux = reinterpret_cast<double*>(c); c += L.flux * nq;
    B.eface = L.eface ? reinterpret_cast<double*>(c) : nullptr; c += L.eface * nq;
    B.vbar = L.vbar ? reinterpret_cast<double*>(c) : nullptr; c += L.vbar * nq;
    B.ecenter = L.ecenter ? reinterpret_cast<double*>(c) : nullptr; c += L.ecenter * nq;
    B.emf = reinterpret_cast<double*>(c); c += L.emf * nq;
    B.ftag = reinterpret_cast<int8_t*>(c); c += L.ftag * nq;
    B.etag = reinterpret_cast<int8_t*>(c); c += L.etag * nq;
    // edge EMFs outside the computed range must read as zero (see grb_reserve)
    if (cudaMemsetAsync(B.emf, 0, L.emf * nq, s) != cudaSuccess) return GRB_ERR_CUDA;
    double* ns = nw->state + q0 * cst * GRB_N_EVOL_VARS;
    double* nbx = nw->bx + q0 * bxs;
    double* nby = nw->by + q0 * bys;
    double* nbz = nw->bz + q0 * bzs;
    const double* os = old->state + q0 * cst * GRB_N_EVOL_VARS;
    const double* obx = old->bx + q0 * bxs;
    const double* oby = old->by + q0 * bys;
    const double* obz = old->bz + q0 * bzs;
    const double* ax = aux + q0 * cst * GRB_N_AUX_VARS;
    const double* idx = g->idx + 3 * q0;
    const double* crd = g->coords ? g->coords + 3 * q0 : nullptr;
    if (P.emf == GRB_EMF_GS) {
      const Box cb = box(0, 0, 0, G.NX, G.NY, G.NZ, nq);
      k_ecenter_static<<<nblk(cb.count(), T), T, 0, s>>>(G, cb, os, obx, oby, obz, ax, B.ecenter);
    }
    const double* bf[3] = {obx, oby, obz};
    for (int dir = 0; dir < 3; ++dir) {
      int lo[3] = {0, 0, 0}, n[3] = {G.NX, G.NY, G.NZ};
      lo[dir] = gz - 1;
      n[dir] = (dir == 0 ? G.nx : dir == 1 ? G.ny : G.nz) + 3;
      const Box b = box(lo[0], lo[1], lo[2], n[0], n[1], n[2], nq);
      if (dir == 0) k_flux<0><<<nblk(b.count(), T), T, 0, s>>>(P, G, b, os, ax, bf[0], B);
      if (dir == 1) k_flux<1><<<nblk(b.count(), T), T, 0, s>>>(P, G, b, os, ax, bf[1], B);
      if (dir == 2) k_flux<2><<<nblk(b.count(), T), T, 0, s>>>(P, G, b, os, ax, bf[2], B);
    }
    const Box eb = box(gz, gz, gz, G.nx + 1, G.ny + 1, G.nz + 1, nq);
    if (P.emf == GRB_EMF_GS)
      k_emf_gs<<<nblk(eb.count(), T), T, 0, s>>>(G, eb, B);
    else
      k_emf_uct<<<nblk(eb.count(), T), T, 0, s>>>(P, G, eb, obx, oby, obz, B);
    if (P.fofc && P.emf == GRB_EMF_GS) {
      if (cudaMemsetAsync(B.ftag, 0, L.ftag * nq, s) != cudaSuccess) return GRB_ERR_CUDA;
      if (cudaMemsetAsync(B.etag, 0, L.etag * nq, s) != cudaSuccess) return GRB_ERR_CUDA;
      const Box fb = box(gz - 1, gz - 1, gz - 1, G.nx + 2, G.ny + 2, G.nz + 2, nq);
      k_fofc_flag<1><<<nblk(fb.count(), T), T, 0, s>>>(P, G, fb, dt, dtfact, ns, os, obx, oby, obz, idx, crd, B);
      k_fofc_faces<false><<<nblk(fb.count(), T), T, 0, s>>>(P, G, fb, os, ax, obx, oby, obz, B);
      k_fofc_edges<<<nblk(fb.count(), T), T, 0, s>>>(G, fb, B);
    }
    const Box ub = box(gz, gz, gz, G.nx, G.ny, G.nz, nq);
    k_update<1><<<nblk(ub.count(), T), T, 0, s>>>(P, G, ub, dt, dtfact, ns, os, ax, idx, B);
    k_ct<<<nblk(eb.count(), T), T, 0, s>>>(G, eb, dt, dtfact, nbx, nby, nbz, idx, B);
    if (cudaGetLastError() != cudaSuccess) return GRB_ERR_CUDA;
  }
  return GRB_OK;
}
