/*
 * grace_b200.h — C ABI of the B200-native Cowling GRMHD stage library.
 *
 * The library replaces GRACE's Cowling-metric GRMHD right-hand-side-and-
 * update path on one GPU.  GRACE's host side (p4est forest, ghost exchange,
 * regrid, I/O) keeps ownership of its Kokkos views and passes their raw
 * device pointers (view.data()) through this interface; the library borrows
 * them for the duration of a call and owns only its own scratch.
 *
 * Array layout contract (GRACE LayoutLeft, i fastest):
 *   state  (nx+2g, ny+2g, nz+2g, GRB_N_EVOL_VARS, nq)    var_array_t
 *   aux    (nx+2g, ny+2g, nz+2g, GRB_N_AUX_VARS,  nq)    var_array_t
 *   bx     (nx+2g+1, ny+2g, nz+2g, 1, nq)                face_staggered_fields_x
 *   by     (nx+2g, ny+2g+1, nz+2g, 1, nq)                face_staggered_fields_y
 *   bz     (nx+2g, ny+2g, nz+2g+1, 1, nq)                face_staggered_fields_z
 *   idx    (3, nq)  inverse cell spacings, idx[d + 3*q]   getinvspacings()
 * Variable indices follow include/grace/data_structures/variable_indices.hh
 * (Cowling build): evolved DENS..ENTROPYSTAR (0-6), GXX..GZZ (7-12), ALP (13),
 * BETAX..BETAZ (14-16), KXX..KZZ (17-22); aux RHO, ZVEC(3), B(3), YE, TEMP,
 * ENTROPY, EPS, PRESS, BDIV, C2P_DENS_ERR, C2P_ERR (0-14).
 *
 * All calls are ordered on the CUDA stream passed in (a cudaStream_t given
 * as void*, NULL = legacy default stream); the caller synchronises.  Every
 * entry point returns GRB_OK (0) or a negative GRB_ERR_* code; device-side
 * fatal conditions (the reference's Kokkos::abort sites) are recorded in a
 * device status word read back by grb_get_status(), never by a trap.
 *
 * A handle belongs to one host thread and one device at a time (GRACE: one
 * rank, one stream): its scratch, work-queue counter, tuned-mode lists and
 * caches are shared by the calls made through it, so two calls on the same
 * handle must not overlap on the GPU (order them on one stream, or use one
 * handle per stream).  The exception is grb_copy_evolved_packed on
 * different arrays, documented there.  First calls that allocate (reserve,
 * the tuned aux list, the copy staging, the static-metric cache) must come
 * before any stream capture that records the handle's work.
 */
#ifndef GRACE_B200_H
#define GRACE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- variable counts and indices (variable_indices.hh:162-287) ---------- */
#define GRB_N_HRSC 7
#define GRB_N_EVOL_VARS 23
#define GRB_N_AUX_VARS 15
enum grb_evol_index {
  GRB_DENS = 0, GRB_SX, GRB_SY, GRB_SZ, GRB_TAU, GRB_YESTAR, GRB_ENTROPYSTAR,
  GRB_GXX, GRB_GXY, GRB_GXZ, GRB_GYY, GRB_GYZ, GRB_GZZ, GRB_ALP,
  GRB_BETAX, GRB_BETAY, GRB_BETAZ,
  GRB_KXX, GRB_KXY, GRB_KXZ, GRB_KYY, GRB_KYZ, GRB_KZZ
};
enum grb_aux_index {
  GRB_RHO = 0, GRB_ZVECX, GRB_ZVECY, GRB_ZVECZ, GRB_BX, GRB_BY, GRB_BZ,
  GRB_YE, GRB_TEMP, GRB_ENTROPY, GRB_EPS, GRB_PRESS, GRB_BDIV,
  GRB_C2P_DENS_ERR, GRB_C2P_ERR
};
/* local cons / prims orderings of one cell (grmhd_helpers.hh:105-149) */
enum grb_cons_local { GRB_C_DENS = 0, GRB_C_STX, GRB_C_STY, GRB_C_STZ, GRB_C_TAU,
                      GRB_C_YES, GRB_C_ENTS, GRB_C_BSX, GRB_C_BSY, GRB_C_BSZ,
                      GRB_NUM_CONS };
enum grb_prims_local { GRB_P_RHO = 0, GRB_P_PRESS, GRB_P_ZX, GRB_P_ZY, GRB_P_ZZ,
                       GRB_P_YE, GRB_P_TEMP, GRB_P_EPS, GRB_P_ENT, GRB_P_BX,
                       GRB_P_BY, GRB_P_BZ, GRB_P_CS2, GRB_NUM_PRIMS };

/* ---- status codes -------------------------------------------------------- */
enum grb_status_code {
  GRB_OK = 0,
  GRB_ERR_INVALID = -1,     /* bad argument / unsupported option */
  GRB_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  GRB_ERR_NOMEM = -3,       /* scratch allocation failed */
  GRB_ERR_NOT_RESERVED = -4, /* grb_reserve was not called for this grid */
  GRB_ERR_NO_MODEL = -5      /* learned c2p requested before a model was trained or set */
};
/* bits of grb_status.device_flags: device-side conditions the reference
 * turns into Kokkos::abort (c2p.hh:167-316); the kernels record and go on
 * with the lenient branch instead. */
enum grb_device_flag {
  GRB_FLAG_C2P_RHO_TOO_HIGH = 1u << 0,
  GRB_FLAG_EOS_RHO_TOO_HIGH = 1u << 1,
  GRB_FLAG_EOS_EPS_TOO_HIGH = 1u << 2,
  GRB_FLAG_EOS_TEMP_TOO_HIGH = 1u << 3,
  GRB_FLAG_EOS_PRESS_TOO_HIGH = 1u << 4,
  GRB_FLAG_BAD_LEARNED_BRACKET = 1u << 8, /* informational: fallback taken */
  GRB_FLAG_WAIT_TIMEOUT = 1u << 9         /* a bounded wait in a kernel gave up
                                             (its results are not valid) */
};

/* ---- scheme selectors (runtime; the reference picks them in CMake) ------- */
enum grb_eos_kind { GRB_EOS_IDEAL_GAS = 0, GRB_EOS_HYBRID_PWPOLY = 1 };
enum grb_recon_kind { GRB_RECON_WENOZ = 0, GRB_RECON_MC2 = 1,
                      GRB_RECON_MINMOD = 2, GRB_RECON_DONOR = 3 };
enum grb_riemann_kind { GRB_RIEMANN_HLL = 0, GRB_RIEMANN_LLF = 1 };
enum grb_emf_kind { GRB_EMF_GS = 0, GRB_EMF_UCT = 1 };
/* What grb_compute_auxiliary_quantities(_dt) and grb_linop_apply write in
 * GRB_MODE_TUNED.  GRB_RANGES_FULL (the default, the drop-in contract):
 * every cell of every block, ghosts included, as compute_auxiliary_quantities
 * (auxiliaries.cpp:111-130) and linop_apply (tstep_utils.hh:54-229) do, so
 * any consumer of aux or of the combined state (regrid, output, diagnostics)
 * sees complete arrays.  GRB_RANGES_NEXT_STAGE: only what the next
 * advance_substep reads before the caller's ghost exchange refills the rest
 * (aux: the cells with at least two indices in [ngz-1, n+ngz+1) and the
 * cells of [ngz-2, n+ngz+2)^3, GS EMF only; linop: the 7 evolved HRSC
 * variables on the cells with y, z in [ngz-2, n+ngz+2) and the faces with
 * interior y, z, the Cowling metric being static); the other aux ghost
 * cells, their c2p rewrites of the state, and the metric and outer planes
 * of a linop target keep their previous values.  GRB_MODE_PLAIN ignores it. */
enum grb_ranges_kind { GRB_RANGES_FULL = 0, GRB_RANGES_NEXT_STAGE = 1 };

#define GRB_MAX_PIECES 8

/* EOS description (eos_storage.cpp:160-190, piecewise_polytropic_eos.hh,
 * hybrid_eos.hh, ideal_gas_eos.hh).  grb_eos_setup_pwpoly() fills the
 * derived pw_* tables from kappa_0 / gammas / rhos exactly as GRACE's
 * setup_cold_polytrope does. */
typedef struct grb_eos_params {
  int32_t kind;          /* grb_eos_kind */
  int32_t n_pieces;      /* hybrid: number of polytropic pieces (<= 8) */
  double gamma;          /* ideal gas adiabatic index */
  double pw_kappa[GRB_MAX_PIECES];
  double pw_gamma[GRB_MAX_PIECES];
  double pw_rho[GRB_MAX_PIECES];   /* segment lower densities, pw_rho[0] = 0 */
  double pw_eps[GRB_MAX_PIECES];
  double pw_press[GRB_MAX_PIECES];
  double gamma_th;       /* hybrid thermal index */
  double eps_max;        /* eos.eps_maximum (c2p eps ceiling) */
  double entropy_min;    /* eos.entropy_minimum */
  double temp_atm;       /* EOS atmosphere temperature = grmhd.atmosphere.temp_fl */
} grb_eos_params;

/* Runtime parameters of the path (grmhd_helpers.hh:41-96 POD structs). */
typedef struct grb_params {
  grb_eos_params eos;
  /* atmosphere: grmhd.atmosphere.* */
  double rho_fl, ye_fl, temp_fl, atmo_tol;
  /* excision: grmhd.excision.* */
  int32_t excise_by_radius;
  double r_ex, alp_ex, rho_ex, temp_ex, ye_ex;
  /* c2p: grmhd.c2p.* */
  double c2p_tol, max_w, max_sigma, beta_fallback, alp_bh_thresh;
  int32_t use_ent_backup;
  /* Riemann: grmhd.riemann.rusanov_use_c_limit */
  double rusanov_use_c_limit;
  /* FOFC: GRACE_ENABLE_FOFC + grmhd.fofc.* */
  int32_t fofc_enable, dmp_enable;
  double dmp_M;
  /* scheme selection */
  int32_t recon, riemann, emf;
  /* cells the aux pass and linop_apply cover in GRB_MODE_TUNED
   * (grb_ranges_kind); the plain mode always covers every cell */
  int32_t ranges;
} grb_params;

/* Block geometry shared by all blocks of a call. */
typedef struct grb_grid {
  int32_t nx, ny, nz, ngz;  /* interior cells per block, ghost width (>= 4) */
  int64_t nq;               /* number of blocks (quadrants) */
  const double* idx;        /* device (3, nq): inverse spacings */
  const double* coords;     /* device (3, nq) or NULL: Cartesian centre of
                               cell (0,0,0) of each block (ghosts included);
                               required only for radius-based excision */
} grb_grid;

/* One evolved state: cell-centred vars + the three face-staggered B arrays. */
typedef struct grb_fields {
  double* state;
  double* bx;
  double* by;
  double* bz;
} grb_fields;

typedef struct grb_status {
  uint32_t device_flags;    /* OR of grb_device_flag since the last clear */
  int32_t last_error;       /* last grb_status_code returned */
  int64_t fofc_faces;       /* faces recomputed by FOFC in the last stage */
  int64_t fofc_edges;       /* edges recomputed by FOFC in the last stage */
  int64_t launches;         /* kernels launched by this handle since creation */
} grb_status;

typedef struct grb_handle grb_handle;

/* ---- parameter helpers (host only) --------------------------------------- */
/* Fill p with GRACE's schema defaults (parameters/grmhd.yaml, eos.yaml) for
 * an EOS of the given kind; EOS-specific numbers still have to be set. */
void grb_params_defaults(grb_params* p, int32_t eos_kind);
/* Derive pw_kappa/pw_eps/pw_press from kappa_0, gammas[n], rhos[n-1]
 * (eos_storage.cpp:53-100, setup_cold_polytrope). */
int grb_eos_setup_pwpoly(grb_eos_params* e, int32_t n_pieces, double kappa_0,
                         const double* gammas, const double* rhos);

/* ---- lifetime ------------------------------------------------------------ */
/* Replaces eos_storage_t construction + the get_*_params() lookups
 * (grmhd_helpers.hh:163-292): validates p and uploads it. */
int grb_create(grb_handle** out, const grb_params* p);
int grb_destroy(grb_handle* h);
/* Size library-owned scratch (fluxes, face/edge EMFs, FOFC tags) for grid g;
 * mirrors resize_aux_staging_and_flux_buffers (variables.cpp:227-).
 * Calls on smaller grids use a prefix of the scratch.  A run of blocks
 * [q0, q1) of the reserved grid — the same block geometry, idx = the
 * reserved idx + 3 q0, every field pointer at block q0, nq = q1 - q0 — is
 * a grid of its own for every stage call; the scratch that outlives a call
 * (the Gardiner-Stone cell-centred E that the aux pass leaves for the next
 * substep) is then addressed from block q0, so runs of blocks may be
 * stepped one after another (each run's ghost zones filled).  With
 * refluxing descriptors set (grb_set_reflux), substeps take the whole
 * reserved grid only (GRB_ERR_INVALID otherwise). */
int grb_reserve(grb_handle* h, const grb_grid* g);
int grb_get_status(grb_handle* h, grb_status* st);
int grb_clear_status(grb_handle* h);

/* ---- the hot path -------------------------------------------------------- */
/* = grace::advance_substep<eos_t>(t, dt, dtfact, new_state, old_state,
 *   new_stag, old_stag) (src/evolution/evolve.cpp:1671-1717): fluxes, EMFs,
 *   FOFC flag + correction, flux divergence + geometric sources, CT update.
 *   aux must hold the primitives of old_state. */
int grb_advance_substep(grb_handle* h, const grb_grid* g, double t, double dt,
                        double dtfact, const grb_fields* new_state,
                        const grb_fields* old_state, const double* aux,
                        void* stream);
/* No counterpart in the reference (it differentiates the metric at every
 * stage).  Cowling: declares the lapse, shift and 3-metric of st->state
 * static and computes, once, the sixth-order derivatives that
 * add_fluxes_and_source_terms (grmhd.hh:232-330) takes of them on every
 * interior cell: 30 doubles per cell in device memory owned by the handle,
 * the same arithmetic as the stage's.  GRB_MODE_TUNED stages on a grid of
 * the same block geometry, the same idx pointer and at most these nq blocks
 * then read them instead of differentiating the metric (identical
 * results); so do stages on a run of these blocks, a grid whose idx points
 * at block q0 of the cached spacings (and whose field pointers start at
 * block q0 alike).  The plain mode ignores them.  Call again after changing the
 * metric or the spacings; st = NULL frees them.  GRB_ERR_NOMEM when the
 * cache cannot be allocated. */
int grb_set_static_metric(grb_handle* h, const grb_grid* g, const grb_fields* st,
                          void* stream);
/* = grace::compute_auxiliary_quantities<eos_t>(state, sstate, aux)
 *   (src/evolution/auxiliaries.cpp:81-180): c2p on every cell including
 *   ghosts, conservative rewrites, C2P_ERR sticky-OR, BDIV, and (GS) the
 *   cell-centred E used by the next stage's EMF.
 *   Only with GRB_MODE_TUNED, the GS EMF and params.ranges =
 *   GRB_RANGES_NEXT_STAGE: just the cells the next advance_substep reads
 *   before the ghost exchange refills the rest, those with at least two
 *   indices in [ngz-1, n+ngz+1), and [ngz-2, n+ngz+2)^3 (14 % fewer cells
 *   for 16^3 blocks with 4 ghosts); aux and the conservative rewrites of the
 *   other 1,936 ghost cells of a 16^3 block are then left as they were.
 *   With the default GRB_RANGES_FULL every cell is written in both modes. */
int grb_compute_auxiliary_quantities(grb_handle* h, const grb_grid* g,
                                     const grb_fields* state, double* aux,
                                     void* stream);
/* compute_auxiliary_quantities fused with the time-step reduction of
 *   find_stable_timestep_impl (src/evolution/find_stable_timestep.cpp:73-125,
 *   compute_max_eigenspeed grmhd.hh:444-519) over the interior cells, from
 *   the primitives this pass computes: *dt_out (device double) becomes
 *   min over interior cells of cfl / cmax * dx(0, q); dx is the (3, nq)
 *   device view of getspacings().  dt_out == NULL: plain aux pass.  The
 *   cross-rank MPI minimum stays with the caller. */
int grb_compute_auxiliary_quantities_dt(grb_handle* h, const grb_grid* g,
                                        const grb_fields* state, double* aux,
                                        const double* dx, double cfl,
                                        double* dt_out, void* stream);
/* = find_stable_timestep_impl on this rank's blocks, as a separate pass over
 *   aux and the metric (same result as the fused form). */
int grb_find_stable_timestep(grb_handle* h, const grb_grid* g,
                             const grb_fields* state, const double* aux,
                             const double* dx, double cfl, double* dt_out,
                             void* stream);
/* = the reset_c2p_diagnostics kernel at the top of evolve_impl
 *   (evolve.cpp:154-161). */
int grb_reset_c2p_diagnostics(grb_handle* h, const grb_grid* g, double* aux,
                              void* stream);
/* = grace::linop_apply (include/grace/utils/tstep_utils.hh:54-229):
 *   A = b*B (C == NULL) or A = b*B + c*C on cells and faces, all 23 vars.
 *   Only with GRB_MODE_TUNED and params.ranges = GRB_RANGES_NEXT_STAGE: just
 *   what the next advance_substep reads before the ghost exchange, the 7
 *   evolved HRSC variables on the cells with y, z in [ngz-2, n+ngz+2) (all
 *   x) and the faces with y, z in the interior (all x) (the metric is static
 *   in Cowling); A's metric, curvature and outer planes keep their previous
 *   values, and the caller's ghost exchange must refill A's ghost zones
 *   before anything else reads them, as evolve_impl does after every stage.
 *   With the default GRB_RANGES_FULL all 23 variables everywhere. */
int grb_linop_apply(grb_handle* h, const grb_grid* g, const grb_fields* A,
                    const grb_fields* B, const grb_fields* C, double b,
                    double c, void* stream);
/* = the three-term grace::linop_apply (include/grace/utils/tstep_utils.hh:
 *   231-311), which the reference's other time integrators use:
 *   A = b*B + c*C + d*D on every cell of all 23 variables and every face,
 *   whatever the mode and params.ranges.  A may be the same arrays as B, C
 *   or D. */
int grb_linop_apply3(grb_handle* h, const grb_grid* g, const grb_fields* A, const grb_fields* B,
                     const grb_fields* C, const grb_fields* D, double b, double c, double d,
                     void* stream);
/* Batched c2p on n independent states (the unit of the c2p micro-benchmark):
 *   cons   [GRB_NUM_CONS][n] densitized conserved incl. cell-centred B*sqrtg
 *   metric [10][n] gxx,gxy,gxz,gyy,gyz,gzz,betax,betay,betaz,alp, or NULL
 *          for the flat metric
 *   prims  [GRB_NUM_PRIMS][n] out; cons_out [GRB_NUM_CONS][n] out or NULL
 *   err    [n] out: c2p_err bits (c2p.hh:98-121); NULL allowed
 *   use_learned: 1 = start the Kastaun root solve from the learned bracket
 *          of the model made by grb_c2p_train or grb_c2p_model_set (per
 *          state, the plain bracket when the learned one misses the root);
 *          GRB_ERR_NO_MODEL without a model.
 * GRB_MODE_TUNED evaluates the c2p with the tuned-mode arithmetic (the same
 * functions up to rounding: fewer divisions, W and b^2 formed once) and
 * defers the entropy-based backup solves to a second pass over the states
 * that need them (compacted, so its warps are uniform; each state's
 * operations and their order unchanged).  The handle keeps one record per
 * state for that pass: the first tuned call with a larger n allocates it
 * (make it before any stream capture). */
int grb_c2p_batch(grb_handle* h, int64_t n, const double* cons,
                  const double* metric, double* prims, double* cons_out,
                  uint32_t* err, int32_t use_learned, void* stream);

/* ---- learned c2p bracket (no counterpart in the reference) --------------
 * A 12-64-64-64-1 ReLU network (BF16 tensor-core hidden layers, FP32
 * accumulation) predicts y = asinh(L / 1e-4), L = log(mu0/mu), for a state:
 * mu is the root of the Kastaun master function (kastaun_c2p.hh:245-290),
 * mu0 the top of the plain bracket (kastaun_c2p.hh:355-369).  Features: D,
 * tau/D, |S|/D, |B|^2/D, cos^2(S,B) (kastaun_c2p.hh:306-337) and log mu0,
 * normalised and split into BF16 high parts and remainders.  The FP64 Brent
 * solve (1e-15 abscissa tolerance, as the plain one) runs on
 * [mu0 e^(-1e-4 sinh(y+delta)), min(mu0 e^(-1e-4 sinh(y-delta)), mu0)] when
 * the master function changes sign there, else on the plain [0, mu0]: the
 * network changes only the starting bracket.
 * Parameters: GRB_MLP_NUM_PARAMS floats, W1[64][16] b1[64] W2[64][64] b2[64]
 * W3[64][64] b3[64] w4[64] b4 (the GRB_MLP_NUM_WEIGHTS trainable ones), then
 * feature means[6], feature sds[6], y mean, y sd, delta. */
#define GRB_MLP_NUM_WEIGHTS 9473
#define GRB_MLP_NUM_PARAMS 9488

typedef struct grb_c2p_diag {
  int32_t* iters;      /* [n] Brent iterations of the Kastaun solve, or NULL */
  int8_t* guess_used;  /* [n] 1 where the learned bracket held the root, or NULL */
  double* mu;          /* [n] Kastaun root (0 where no Kastaun solve ran), or NULL */
  double* bracket;     /* [2][n] learned bracket lo, hi (0 where none), or NULL */
} grb_c2p_diag;
/* grb_c2p_batch with per-state diagnostics (device arrays). */
int grb_c2p_batch_diag(grb_handle* h, int64_t n, const double* cons,
                       const double* metric, double* prims, double* cons_out,
                       uint32_t* err, int32_t use_learned,
                       const grb_c2p_diag* diag, void* stream);

typedef struct grb_train_config {
  int64_t steps;        /* Adam steps (default 8000) */
  int32_t batch;        /* states per step, a multiple of 64 (default 16384) */
  float lr;             /* peak learning rate (default 3e-3) */
  float lr_min;         /* end of the cosine decay (default 3e-5) */
  uint64_t seed;        /* weight initialisation and sampling */
  int64_t calib_states; /* states timed to choose delta (default 2^18) */
} grb_train_config;
typedef struct grb_train_report {
  int64_t states;       /* states given */
  int64_t labelled;     /* states whose plain c2p ran the Kastaun solve */
  float loss_first;     /* batch MSE of normalised y, first step */
  float loss_last;      /* ... last step */
  float err_q50;        /* |y_net - y| quantiles over the states */
  float err_q90;
  float err_q99;
  float err_q999;
  float err_max;
  float delta;          /* chosen bracket half-width (in y) */
  float delta_cand[4];  /* candidates: 1.2 x the q90, q99, q999, q9999 errors */
  float calib_ms[4];    /* learned c2p time on the calibration states */
  double train_ms;      /* device time: labels + statistics + Adam steps */
  float calib_cost[4];  /* the choice's cost: mean over warps of the largest
                           per-state Brent iterations (+1 where the learned
                           bracket missed the root) */
} grb_train_report;
void grb_train_config_defaults(grb_train_config* c);
/* Train the bracket network on the GPU from n states (cons/metric as for
 * grb_c2p_batch): labels are the roots of the plain FP64 c2p of the same
 * states; the tensor-core forward, the FP32 backward and Adam run as this
 * library's kernels; delta is then chosen among four quantiles of the
 * prediction error by the learned c2p's warp-level Brent cost on the
 * calibration states (a count, so the same training gives the same model
 * every run; the times are reported beside it).  Synchronises the stream. */
int grb_c2p_train(grb_handle* h, int64_t n, const double* cons,
                  const double* metric, const grb_train_config* cfg,
                  grb_train_report* report, void* stream);
/* Copy the model to / from a host array of GRB_MLP_NUM_PARAMS floats. */
int grb_c2p_model_get(grb_handle* h, float* params, int64_t nparams);
int grb_c2p_model_set(grb_handle* h, const float* params, int64_t nparams);
/* Features [6][n] (FP32) and target y [n] (NaN where mu <= 0 or mu is NULL)
 * of n states, mu the plain roots; device arrays. */
int grb_c2p_features(grb_handle* h, int64_t n, const double* cons,
                     const double* metric, const double* mu, float* feat,
                     float* target, void* stream);
/* Network output y [n] for raw features [6][n] with the parameter block
 * params (device; NULL = the handle's model). */
int grb_mlp_eval(grb_handle* h, int64_t n, const float* params,
                 const float* feat, float* out, void* stream);
/* Gradient of the mean squared error of normalised y over n samples
 * (targets NaN are skipped but still count in the mean) with respect to the
 * GRB_MLP_NUM_WEIGHTS trainable parameters; grad[GRB_MLP_NUM_WEIGHTS] receives
 * the loss.  All device arrays; synchronises the stream. */
int grb_mlp_grad(grb_handle* h, int64_t n, const float* params,
                 const float* feat, const float* target, float* grad,
                 void* stream);


/* ---- execution mode and autotuning --------------------------------------- */
/* GRB_MODE_PLAIN: one thread per face / edge / cell over the reference's own
 * launch ranges (compute_fluxes computes faces over the full transverse
 * ghost range, evolve.cpp:908-922; linop_apply combines all 23 variables).
 * GRB_MODE_TUNED: only the faces the stage reads (internal scratch), one
 * reciprocal per face for the HLL fluxes, division-free WENO-Z weights, the
 * register-cap variant picked by grb_autotune, fewer divisions in the c2p.
 * Results agree with the plain mode to rounding.  Which cells the aux pass
 * and linop_apply write is chosen separately, by params.ranges
 * (grb_ranges_kind). */
enum grb_mode { GRB_MODE_PLAIN = 0, GRB_MODE_TUNED = 1 };
int grb_set_mode(grb_handle* h, int32_t mode);
/* Times the register-cap variants of the flux, FOFC-flag, update and aux
 * kernels on device copies of up to 96 blocks spread evenly over the grid
 * (block k nq / 96: every level of a hierarchy ordered by level is
 * represented; the arrays passed in are only read) and keeps the fastest
 * for the tuned mode.  Allocates and frees temporary copies; synchronises
 * the stream. */
int grb_autotune(grb_handle* h, const grb_grid* g, const grb_fields* new_state,
                 const grb_fields* old_state, const double* aux, void* stream);
/* variant[4]: chosen minimum-CTAs-per-SM of flux, flag, update, aux (flux:
 * plus 100 when the TMA-staged shared-memory kernel was chosen, plus 1000
 * for its work-queue form; update: of the kernel that reads the
 * static-metric cache when one is set; flag, update and aux: plus 100 for
 * the work-queue form; aux: plus 200 for the deferred-backup form); ms[12]
 * (or NULL): timed milliseconds of the 3 grid-launched candidates per
 * family. */
int grb_get_tuning(grb_handle* h, int32_t* variant, float* ms);
/* ms[n] (n <= 5 written): milliseconds grb_autotune timed for the other
 * launch forms of the candidate it chose in each family: the work-queue
 * FOFC flag, the work-queue aux pass, the deferred-backup aux pass, the
 * work-queue flux (x faces), the work-queue update (0 before autotuning;
 * 1e30 for a form that could not be set up). */
int grb_get_tuning_forms(grb_handle* h, float* ms, int32_t n);
/* Choose the tuned-mode candidates without timing: variant[4] = candidate
 * index of flux, flag, update, aux: 0..2 grid launches (flux: 0 global-load kernel, 1 the
 * TMA-staged kernel with 128-thread tiles at 4 CTAs/SM, 2 with 256-thread
 * tiles (twice the face rows per tile) at 2 CTAs/SM; update: 1, 4, 5
 * CTAs/SM (1, 3, 4 for the kernel that reads the static-metric cache);
 * flag and aux: 3, 4, 5 CTAs/SM); 3..5 the work-queue form of candidate
 * 0..2 — one wave of persistent CTAs pulling tiles (128 items, or the TMA
 * flux kernel's tiles) from a device counter; aux also 6..8: the
 * deferred-backup form — the cells whose Kastaun result is distrusted
 * listed and finished by a second kernel running their entropy backups
 * together — at 3, 4, 5 CTAs/SM, its list allocated here for the reserved
 * grid: call before any stream capture). */
int grb_set_tuning(grb_handle* h, const int32_t* variant);

/* Capacity, in faces, of the compacted list through which GRB_MODE_TUNED
 * stages recompute the FOFC-tagged faces: at most what grb_reserve
 * allocated (min(4 Mi, the grid's faces); the default).  A substep that
 * tags more faces than this recomputes them in a loop over the whole FOFC
 * box instead, with the same results; 0 sends every substep there (so that
 * tests can reach that path).  Calls after it on this handle use the new
 * capacity until the next grb_reserve of another geometry.
 * GRB_ERR_NOT_RESERVED before grb_reserve. */
int grb_set_fofc_list_capacity(grb_handle* h, int64_t faces);

/* ---- measurement helpers -------------------------------------------------- */
/* Kernel kinds for grb_kernel_times. */
enum grb_kernel_kind {
  GRB_KIND_FLUX = 0, GRB_KIND_EMF, GRB_KIND_FOFC_FLAG, GRB_KIND_FOFC_FIX, GRB_KIND_UPDATE,
  GRB_KIND_CT, GRB_KIND_AUX, GRB_KIND_LINOP, GRB_KIND_GHOST, GRB_KIND_C2P, GRB_KIND_OTHER,
  GRB_KIND_COUNT
};
/* When enabled, every launch group is bracketed by CUDA events recorded on
 * the caller's stream.  grb_kernel_times synchronises on the last event,
 * returns the summed milliseconds and launch-group counts per kind
 * (arrays of GRB_KIND_COUNT) and resets the accumulators. */
int grb_set_kernel_timing(grb_handle* h, int32_t enable);
/* No counterpart in the reference: the current device's FP64 throughput,
 * the denominator of the FP64 roofline.  Times (CUDA events, best of 5 on
 * the stream) a kernel of independent fused multiply-add chains, 8 CTAs of
 * 256 threads per SM; *tflops = 2 x FMAs / time in TFLOP/s, *ms (or NULL)
 * the launch time.  Synchronises the stream. */
int grb_measure_fp64_peak(double* tflops, double* ms, void* stream);
int grb_kernel_times(grb_handle* h, double* ms, int64_t* counts, int32_t nkinds);

/* ---- harness-side helper (outside the reference's hot path) -------------- */
/* Ghost fill for a brick of nbx*nby*nbz same-level blocks (block q at
 * (q % nbx, (q / nbx) % nby, q / (nbx*nby))): periodic axes copy from the
 * neighbouring block, the others copy the nearest interior cell / face
 * (zero-gradient outflow, extrap_bc_t<0> of
 * include/grace/amr/ghostzone_kernels/phys_bc_kernels.hh:169).  Stands in for
 * GRACE's amr::apply_boundary_conditions on a unigrid brick; exchanges the
 * 7 evolved HRSC variables and the three face-B arrays. */
int grb_fill_ghosts_brick(grb_handle* h, const grb_grid* g, const grb_fields* f, int32_t nbx,
                          int32_t nby, int32_t nbz, const int32_t* periodic, void* stream);
/* No counterpart in the reference: grb_fill_ghosts_brick restricted to the
 * ghost zones of blocks [q_begin, q_end) of the brick (g and f still
 * describe the whole brick; the sources, interior cells and faces of the
 * neighbouring blocks, may lie anywhere in it).  For pipelines that fill a
 * run of blocks as soon as the blocks it reads from are final. */
int grb_fill_ghosts_brick_range(grb_handle* h, const grb_grid* g, const grb_fields* f, int32_t nbx,
                                int32_t nby, int32_t nbz, const int32_t* periodic, int64_t q_begin,
                                int64_t q_end, void* stream);
/* No counterpart in the reference (its state stays on the device): copies
 * the interior of the evolved variables, i.e. the 7 HRSC variables on the
 * interior cells and the three face-B arrays on the interior faces
 * (staggered index in [ngz, n+ngz]), between host arrays and the device
 * arrays `dev` of the same layout, to_device = 1 host -> device, 0 device ->
 * host.  host_state_nvars: variables per block in host->state, either
 * GRB_N_EVOL_VARS (the device layout) or GRB_N_HRSC (the evolved
 * variables only).  The host arrays must be pinned and mapped (cudaHostAlloc, or any
 * page-locked allocation visible to the device); one kernel per array
 * reads or writes them over the bus in whole rows of the interior (y, z)
 * range.  An upload leaves the device ghost zones as they were (refill them
 * with the ghost exchange); a download also writes the x-ghost cells of the
 * interior rows of the host arrays.  GRB_ERR_INVALID when a host array is
 * not device-accessible. */
int grb_copy_evolved_interior(grb_handle* h, const grb_grid* g, const grb_fields* host,
                              int32_t host_state_nvars, const grb_fields* dev, int32_t to_device,
                              void* stream);
/* No counterpart in the reference: the same interior as
 * grb_copy_evolved_interior, with host arrays in a packed interior layout
 * (no ghosts, LayoutLeft): host->state [nq][GRB_N_HRSC][nz][ny][nx],
 * host->bx [nq][nz][ny][nx+1], host->by [nq][nz][ny+1][nx],
 * host->bz [nq][nz+1][ny][nx].  Each array crosses the bus as one
 * contiguous DMA copy through a device staging buffer owned by the handle
 * (packed or unpacked on the device by one kernel), so the copy engine
 * moves only interior bytes at its full rate; host arrays should be pinned.
 * The first call allocates the staging (make it before any stream
 * capture); an upload leaves the device ghost zones as they were.  An array
 * whose host and device pointers are both NULL is skipped; each array has
 * its own staging region, so calls that move different arrays may run on
 * different streams at the same time. */
int grb_copy_evolved_packed(grb_handle* h, const grb_grid* g, const grb_fields* host,
                            const grb_fields* dev, int32_t to_device, void* stream);

/* ---- FMR: restriction into coarse buffers ---------------------------------- */
/* = the ghost-zone restriction of GRACE's AMR
 *   (include/grace/amr/ghostzone_kernels/restriction_task_factories.hh:64-
 *   200, restrict_kernels.hh:42-165): for each of the nquads fine
 *   quadrants, block src_q[i] of `fine` writes the coarse-resolution image
 *   of its interior into block dst_q[i] of the coarse buffers `cbuf` (same
 *   block geometry; coarse cells (ngz + [0, n/2))^3):
 *     state variables vars_lo[0..nlo) by the 8-cell average
 *       (second_order_restrict_op, pr_helpers.hh:187-213);
 *     state variables vars_ho[0..nho) by the 5-point Lagrange restriction
 *       (lagrange_restrict_op<4>, pr_helpers.hh:216-322, the coefficients of
 *       fill_fifth_order_restriction_coefficients), its interior stencils
 *       mirrored by the quadrant's half of its parent: bits 0, 1, 2 of
 *       child_id[i] (the p4est Morton child id) for x, y, z;
 *     face B (the arrays not NULL in both `fine` and `cbuf`) by the average
 *       of the 4 fine faces in each coarse face (div_free_restrict_op),
 *       which keeps div B of the coarse image at round-off.
 *   src_q, dst_q (int64) and child_id (uint8) are device arrays of nquads;
 *   the dst_q must be distinct.  Results are those of the reference's
 *   operators bit for bit (each product and sum rounded on its own). */
int grb_restrict_to_coarse(grb_handle* h, const grb_grid* g, const grb_fields* fine,
                           const grb_fields* cbuf, int64_t nquads, const int64_t* src_q,
                           const int64_t* dst_q, const uint8_t* child_id,
                           const int32_t* vars_lo, int32_t nlo, const int32_t* vars_ho,
                           int32_t nho, void* stream);

/* ---- boundary mass outflux ------------------------------------------------ */
/* = boundary_outflow_t::accumulate (include/grace/evolution/
 *   boundary_outflow.hh:79-180, called from evolve.cpp:1704): for each of
 *   the nfaces (quad[i], face[i]) on a non-periodic outer boundary (face =
 *   2 axis + side, side 1 the upper face), adds
 *     sign * dt * dtfact * dA * sum over the face's interior cells of the
 *     DENS flux through the block's boundary face plane
 *   to the device scalar *outflow (sign +1 on upper faces, -1 on lower;
 *   dA the product of the two tangential spacings from dx, the (3, nq)
 *   device array dx[d + 3 q] of getspacings()).  It reads the face fluxes
 *   the last grb_advance_substep on this handle computed (after the FOFC
 *   correction), so call it after each substep with that substep's dt and
 *   dtfact.  quad (int64), face (uint8) are device arrays; one CTA per face,
 *   summed into *outflow by one atomic add each, as the reference does.
 *   Reading back, the MPI sum over ranks, the symmetry multiplier and the
 *   reset (flush_to_host) stay with the caller. */
int grb_accumulate_boundary_outflow(grb_handle* h, const grb_grid* g, int64_t nfaces,
                                    const int64_t* quad, const uint8_t* face, const double* dx,
                                    double dt, double dtfact, double* outflow, void* stream);

/* ---- FMR: prolongation into ghost zones --------------------------------- */
#define GRB_ELEM_FACE 0
#define GRB_ELEM_EDGE 1
#define GRB_ELEM_CORNER 2
/* = the ghost-zone prolongation of GRACE's AMR, one task per element kind
 *   (include/grace/amr/ghostzone_kernels/prolongation_task_factories.hh:
 *   70-230, prolongation_kernels.hh:46-399): for each of the nelems ghost
 *   elements of kind elem_kind (GRB_ELEM_FACE: face elem_id[i] in 0..5 =
 *   2 axis + side; GRB_ELEM_EDGE: edge 0..11, 4 x its axis + the sides of
 *   the two other axes in bits 0, 1; GRB_ELEM_CORNER: corner 0..7, bit d the
 *   side along axis d), the ghost cells of block fine_q[i] of `fine` in that
 *   element are filled from block cbuf_q[i] of the coarse buffers `cbuf`
 *   (same block geometry; coarse cell ngz + t covers fine cells ngz + 2t,
 *   ngz + 2t + 1, the low coarse ghosts start at ngz/2):
 *     state variables vars_lo[0..nlo) by the minmod slope-limited operator
 *       (slope_limited_prolong_op<minmod>, pr_helpers.hh:73-103);
 *     state variables vars_ho[0..nho) by the 5-point Lagrange operator
 *       (lagrange_prolong_op<4>, pr_helpers.hh:105-185, the coefficients of
 *       fill_fifth_order_prolongation_coefficients);
 *     face B (when the face arrays are given, all six) by the Toth-Roe
 *       divergence-preserving prolongation (div_free_prolong_op): the fine
 *       faces on coarse faces from the coarse face and its minmod slopes,
 *       except the first face of an axis where have_fine[6 i + 2 axis + 0]
 *       is set and with the last one where have_fine[6 i + 2 axis + 1] is
 *       not (the neighbour on that side holds fine data), then the faces
 *       inside coarse cells from those around them.
 *   Blocks are cubic (nx = ny = nz, even, >= 4) with an even ngz >= 4.
 *   fine_q, cbuf_q (int64), elem_id (uint8) and have_fine (int8, 6 per
 *   element) are device arrays.  Results are those of the reference's
 *   functors bit for bit (each product and sum rounded on its own); one
 *   launch per variable list and two for face B. */
int grb_prolong_to_ghosts(grb_handle* h, const grb_grid* g, const grb_fields* fine,
                          const grb_fields* cbuf, int32_t elem_kind, int64_t nelems,
                          const int64_t* fine_q, const int64_t* cbuf_q, const uint8_t* elem_id,
                          const int8_t* have_fine, const int32_t* vars_lo, int32_t nlo,
                          const int32_t* vars_ho, int32_t nho, void* stream);

/* ---- ghost fill by gather maps (harness-side helper) --------------------- */
/* One gather map: entry e sets, for each variable v, a[dst[e] + v vs] =
 * the sum over its cnt[e] (1..8) slots k of w[k n + e] * a[src[k n + e] +
 * v vs] (accumulated in slot order, each product and sum rounded on its
 * own); dst and src are element offsets of variable 0 in the array, vs the
 * cells of one variable of a block. */
typedef struct grb_gather {
  int64_t n;
  const int8_t* cnt;   /* [n] device */
  const int64_t* dst;  /* [n] device */
  const int64_t* src;  /* [8][n] device, slot-major */
  const double* w;     /* [8][n] device, slot-major */
} grb_gather;
/* No counterpart in the reference (its ghost exchange is the host's): fills
 * the ghost zones of f by precomputed gather maps, cells for the first nvars
 * state variables and faces[0..2] for the face-B arrays staggered along x, y,
 * z (NULL entries skipped).  Stands in, for multi-level block lists on one
 * rank, for the host's same-level copies, restriction and prolongation: the
 * maps encode where each ghost value comes from (grace_b200.fmr builds them
 * for a static hierarchy).  The sources must be interior cells and faces. */
int grb_fill_ghosts_gather(grb_handle* h, const grb_grid* g, const grb_fields* f, const grb_gather* cells,
                           int32_t nvars, const grb_gather* faces, void* stream);

/* ---- reflux at coarse-fine interfaces ------------------------------------ */
/* The reflux descriptors of the caller's AMR hierarchy on this rank: what
 * GRACE's ghost layer builds from the p4est face and edge iterators
 * (include/grace/amr/amr_ghosts.hh:190-330, src/amr/ghost_helpers/
 * iterate_faces.cpp:150-280, iterate_edges.cpp:330-407), here as device
 * arrays of block indices.  Blocks are cubic.  Face ids are 2 axis + side
 * (side 1 the upper face); edge ids are p4est's (4 axis + s_a + 2 s_b, with
 * s_a, s_b the sides along the edge's two other axes in x, y, z order). */
typedef struct grb_reflux {
  /* hanging faces: face face_coarse_id[i] of block face_coarse_q[i] is
   * covered by the four blocks face_fine_q[4 i + c] of the next finer level,
   * c = a + 2 b with a, b the halves along the face's other two axes (x
   * before y before z); each touches it with its opposite face */
  int64_t nfaces;
  const int64_t* face_coarse_q;
  const uint8_t* face_coarse_id;
  const int64_t* face_fine_q;
  /* faces between blocks of the same level: blocks same_face_q[2 i + s]
   * meet with their faces same_face_id[2 i + s], s = 0, 1 */
  int64_t nsame_faces;
  const int64_t* same_face_q;
  const uint8_t* same_face_id;
  /* average the fluxes of same-level faces too (the reference's
   * GRACE_SAME_LEVEL_FACE_AVERAGE build option); EMFs always are */
  int32_t same_level_flux_average;
  /* hanging edges (blocks of two levels along one edge, and the two middle
   * lines of each hanging face): edge_nsides[i] <= 4 sides; side s has the
   * edge id edge_id[4 i + s] in its block(s), edge_is_fine[4 i + s] set
   * when it holds the two finer blocks edge_q[8 i + 2 s + c] (c the lower,
   * upper half along the edge), else one coarser block edge_q[8 i + 2 s]
   * whose edge cell other axes move to the block's middle where
   * edge_off[8 i + 2 s + 0 / 1] is set (middle lines of a hanging face) */
  int64_t nedges;
  const uint8_t* edge_nsides;
  const uint8_t* edge_id;
  const uint8_t* edge_is_fine;
  const int64_t* edge_q;
  const uint8_t* edge_off;
  /* edges between blocks of one level: same_edge_nsides[i] <= 4 sides, side
   * s is edge same_edge_id[4 i + s] of block same_edge_q[4 i + s] */
  int64_t nsame_edges;
  const uint8_t* same_edge_nsides;
  const uint8_t* same_edge_id;
  const int64_t* same_edge_q;
} grb_reflux;
/* = the refluxing of advance_substep (src/evolution/evolve.cpp:1690-1705,
 *   src/evolution/refluxing.cpp:528-1170, the local branches): from now on
 *   every grb_advance_substep on this handle, after FOFC and before the flux
 *   divergence, replaces the coarse flux on each hanging face by the area
 *   average of the fine fluxes (and averages same-level faces' fluxes if
 *   asked), and after the update, before the CT update, makes the edge EMFs
 *   of every interface agree (hanging faces' inner lines from the fine
 *   EMFs, same-level faces' inner lines by the mean of both sides, hanging
 *   and same-level edges by the rule of the reference: the fine, or the
 *   first, side in edge-id order).  The arrays are the caller's and are read
 *   by every later substep (keep them alive and unchanged, or set again);
 *   the handle allocates its edge accumulation buffers here (call before any
 *   stream capture).  r = NULL, or all counts 0, turns refluxing off.
 *   Requires grb_reserve and cubic blocks.  The MPI exchange of remote
 *   sides stays with the caller. */
int grb_set_reflux(grb_handle* h, const grb_reflux* r);

/* ---- scratch-free stage -------------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a host code whose GPU memory is owned up front by a pooling allocator, or
 * a plugin host that forbids libraries to allocate device memory after
 * start-up): the same stage as grb_advance_substep, with the library's
 * face/edge scratch in a file-scope device array of GRB_STATIC_SCRATCH_BYTES
 * instead of handle-owned memory.  No handle is needed (creating one
 * allocates); the call allocates and frees nothing.  Blocks are processed in
 * chunks that fit the array, so any nq works; a single block whose scratch
 * (~30 doubles per face-grid point + 3 per cell) exceeds the array is
 * rejected with GRB_ERR_INVALID and a message on stderr.  Every GPU that
 * loads the library holds the array until exit.  Each call looks up the
 * array's device address on the current device (cudaGetSymbolAddress, no
 * allocation), so the address stays right after a device reset; the first
 * call on a device also loads the library's kernels there, so make that
 * first call before any stream capture.  All calls share
 * the one array, which keeps the last call's contents (what must start at
 * zero is cleared by each call), so calls that overlap on the GPU — from
 * two streams or two threads — race and corrupt each other's results.
 * FOFC counts and status flags are not reported by this entry point. */
#define GRB_STATIC_SCRATCH_BYTES (64u << 20)
int grb_advance_substep_static(const grb_params* p, const grb_grid* g, double t, double dt,
                               double dtfact, const grb_fields* new_state,
                               const grb_fields* old_state, const double* aux, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GRACE_B200_H */
