"""ctypes mirror of include/grace_b200.h (the library's C ABI).

The structures here are byte-for-byte the C structs of the header; the
layout test in tests/ checks their sizes and offsets against the compiled
library's exported helpers.
"""
import ctypes as C

N_HRSC = 7
N_EVOL_VARS = 23
N_AUX_VARS = 15
MAX_PIECES = 8

# evolved variable indices (variable_indices.hh:162-241, Cowling build)
(DENS, SX, SY, SZ, TAU, YESTAR, ENTROPYSTAR, GXX, GXY, GXZ, GYY, GYZ, GZZ, ALP,
 BETAX, BETAY, BETAZ, KXX, KXY, KXZ, KYY, KYZ, KZZ) = range(23)
# aux variable indices (variable_indices.hh:243-287)
(RHO, ZVECX, ZVECY, ZVECZ, BX, BY, BZ, YE, TEMP, ENTROPY, EPS, PRESS, BDIV,
 C2P_DENS_ERR, C2P_ERR) = range(15)
# local cons / prims of one cell (grmhd_helpers.hh:105-149)
(C_DENS, C_STX, C_STY, C_STZ, C_TAU, C_YES, C_ENTS, C_BSX, C_BSY, C_BSZ) = range(10)
(P_RHO, P_PRESS, P_ZX, P_ZY, P_ZZ, P_YE, P_TEMP, P_EPS, P_ENT, P_BX, P_BY, P_BZ,
 P_CS2) = range(13)

EOS_IDEAL_GAS, EOS_HYBRID_PWPOLY = 0, 1
RECON_WENOZ, RECON_MC2, RECON_MINMOD, RECON_DONOR = 0, 1, 2, 3
RIEMANN_HLL, RIEMANN_LLF = 0, 1
EMF_GS, EMF_UCT = 0, 1
RANGES_FULL, RANGES_NEXT_STAGE = 0, 1

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_NOT_RESERVED, ERR_NO_MODEL = 0, -1, -2, -3, -4, -5
STATIC_SCRATCH_BYTES = 64 << 20
MODE_PLAIN, MODE_TUNED = 0, 1
MLP_NUM_WEIGHTS, MLP_NUM_PARAMS = 9473, 9488
MLP_IN = 6
KIND_NAMES = ["flux", "emf", "fofc_flag", "fofc_fix", "update", "ct", "aux", "linop", "ghost",
              "c2p", "other"]


class EosParams(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("n_pieces", C.c_int32),
        ("gamma", C.c_double),
        ("pw_kappa", C.c_double * MAX_PIECES),
        ("pw_gamma", C.c_double * MAX_PIECES),
        ("pw_rho", C.c_double * MAX_PIECES),
        ("pw_eps", C.c_double * MAX_PIECES),
        ("pw_press", C.c_double * MAX_PIECES),
        ("gamma_th", C.c_double),
        ("eps_max", C.c_double),
        ("entropy_min", C.c_double),
        ("temp_atm", C.c_double),
    ]


class Params(C.Structure):
    _fields_ = [
        ("eos", EosParams),
        ("rho_fl", C.c_double), ("ye_fl", C.c_double), ("temp_fl", C.c_double),
        ("atmo_tol", C.c_double),
        ("excise_by_radius", C.c_int32),
        ("r_ex", C.c_double), ("alp_ex", C.c_double), ("rho_ex", C.c_double),
        ("temp_ex", C.c_double), ("ye_ex", C.c_double),
        ("c2p_tol", C.c_double), ("max_w", C.c_double), ("max_sigma", C.c_double),
        ("beta_fallback", C.c_double), ("alp_bh_thresh", C.c_double),
        ("use_ent_backup", C.c_int32),
        ("rusanov_use_c_limit", C.c_double),
        ("fofc_enable", C.c_int32), ("dmp_enable", C.c_int32),
        ("dmp_M", C.c_double),
        ("recon", C.c_int32), ("riemann", C.c_int32), ("emf", C.c_int32),
        ("ranges", C.c_int32),
    ]


class Grid(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("ngz", C.c_int32),
        ("nq", C.c_int64),
        ("idx", C.c_void_p),
        ("coords", C.c_void_p),
    ]


class Fields(C.Structure):
    _fields_ = [("state", C.c_void_p), ("bx", C.c_void_p), ("by", C.c_void_p),
                ("bz", C.c_void_p)]


class Status(C.Structure):
    _fields_ = [("device_flags", C.c_uint32), ("last_error", C.c_int32),
                ("fofc_faces", C.c_int64), ("fofc_edges", C.c_int64),
                ("launches", C.c_int64)]


class Reflux(C.Structure):
    _fields_ = [("nfaces", C.c_int64), ("face_coarse_q", C.c_void_p), ("face_coarse_id", C.c_void_p),
                ("face_fine_q", C.c_void_p),
                ("nsame_faces", C.c_int64), ("same_face_q", C.c_void_p), ("same_face_id", C.c_void_p),
                ("same_level_flux_average", C.c_int32),
                ("nedges", C.c_int64), ("edge_nsides", C.c_void_p), ("edge_id", C.c_void_p),
                ("edge_is_fine", C.c_void_p), ("edge_q", C.c_void_p), ("edge_off", C.c_void_p),
                ("nsame_edges", C.c_int64), ("same_edge_nsides", C.c_void_p), ("same_edge_id", C.c_void_p),
                ("same_edge_q", C.c_void_p)]


class Gather(C.Structure):
    _fields_ = [("n", C.c_int64), ("cnt", C.c_void_p), ("dst", C.c_void_p), ("src", C.c_void_p),
                ("w", C.c_void_p)]


class C2PDiag(C.Structure):
    _fields_ = [("iters", C.c_void_p), ("guess_used", C.c_void_p), ("mu", C.c_void_p),
                ("bracket", C.c_void_p)]


class TrainConfig(C.Structure):
    _fields_ = [("steps", C.c_int64), ("batch", C.c_int32), ("lr", C.c_float), ("lr_min", C.c_float),
                ("seed", C.c_uint64), ("calib_states", C.c_int64)]


class TrainReport(C.Structure):
    _fields_ = [("states", C.c_int64), ("labelled", C.c_int64), ("loss_first", C.c_float),
                ("loss_last", C.c_float), ("err_q50", C.c_float), ("err_q90", C.c_float),
                ("err_q99", C.c_float), ("err_q999", C.c_float),
                ("err_max", C.c_float), ("delta", C.c_float), ("delta_cand", C.c_float * 4),
                ("calib_ms", C.c_float * 4), ("train_ms", C.c_double), ("calib_cost", C.c_float * 4)]


# Every extern "C" symbol declared in include/grace_b200.h, with its
# (restype, argtypes).  The loader binds exactly these.
PROTOTYPES = {
    "grb_params_defaults": (None, [C.POINTER(Params), C.c_int32]),
    "grb_eos_setup_pwpoly": (C.c_int, [C.POINTER(EosParams), C.c_int32, C.c_double,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "grb_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(Params)]),
    "grb_destroy": (C.c_int, [C.c_void_p]),
    "grb_reserve": (C.c_int, [C.c_void_p, C.POINTER(Grid)]),
    "grb_get_status": (C.c_int, [C.c_void_p, C.POINTER(Status)]),
    "grb_clear_status": (C.c_int, [C.c_void_p]),
    "grb_advance_substep": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.c_double, C.c_double,
                                      C.c_double, C.POINTER(Fields), C.POINTER(Fields),
                                      C.c_void_p, C.c_void_p]),
    "grb_compute_auxiliary_quantities": (C.c_int, [C.c_void_p, C.POINTER(Grid),
                                                   C.POINTER(Fields), C.c_void_p,
                                                   C.c_void_p]),
    "grb_compute_auxiliary_quantities_dt": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields),
                                                      C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                                      C.c_void_p]),
    "grb_find_stable_timestep": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields), C.c_void_p,
                                           C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]),
    "grb_reset_c2p_diagnostics": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.c_void_p,
                                            C.c_void_p]),
    "grb_linop_apply": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields),
                                  C.POINTER(Fields), C.POINTER(Fields), C.c_double,
                                  C.c_double, C.c_void_p]),
    "grb_linop_apply3": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields),
                                   C.POINTER(Fields), C.POINTER(Fields), C.POINTER(Fields),
                                   C.c_double, C.c_double, C.c_double, C.c_void_p]),
    "grb_c2p_batch": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "grb_c2p_batch_diag": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C2PDiag),
                                     C.c_void_p]),
    "grb_train_config_defaults": (None, [C.POINTER(TrainConfig)]),
    "grb_c2p_train": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                C.POINTER(TrainConfig), C.POINTER(TrainReport), C.c_void_p]),
    "grb_c2p_model_get": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "grb_c2p_model_set": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int64]),
    "grb_c2p_features": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
    "grb_mlp_eval": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p]),
    "grb_mlp_grad": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "grb_set_mode": (C.c_int, [C.c_void_p, C.c_int32]),
    "grb_autotune": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields), C.POINTER(Fields),
                               C.c_void_p, C.c_void_p]),
    "grb_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "grb_get_tuning_forms": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int32]),
    "grb_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "grb_set_fofc_list_capacity": (C.c_int, [C.c_void_p, C.c_int64]),
    "grb_set_reflux": (C.c_int, [C.c_void_p, C.POINTER(Reflux)]),
    "grb_fill_ghosts_gather": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields), C.POINTER(Gather),
                                         C.c_int32, C.POINTER(Gather), C.c_void_p]),
    "grb_set_kernel_timing": (C.c_int, [C.c_void_p, C.c_int32]),
    "grb_measure_fp64_peak": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]),
    "grb_kernel_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                   C.c_int32]),
    "grb_advance_substep_static": (C.c_int, [C.POINTER(Params), C.POINTER(Grid), C.c_double,
                                             C.c_double, C.c_double, C.POINTER(Fields),
                                             C.POINTER(Fields), C.c_void_p, C.c_void_p]),
    "grb_fill_ghosts_brick": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields),
                                        C.c_int32, C.c_int32, C.c_int32,
                                        C.POINTER(C.c_int32), C.c_void_p]),
    "grb_fill_ghosts_brick_range": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields),
                                              C.c_int32, C.c_int32, C.c_int32,
                                              C.POINTER(C.c_int32), C.c_int64, C.c_int64, C.c_void_p]),
    "grb_restrict_to_coarse": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields), C.POINTER(Fields),
                                         C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32),
                                         C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_void_p]),
    "grb_accumulate_boundary_outflow": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.c_int64, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p]),
    "grb_prolong_to_ghosts": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields), C.POINTER(Fields),
                                        C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32), C.c_int32,
                                        C.c_void_p]),
    "grb_set_static_metric": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields), C.c_void_p]),
    "grb_copy_evolved_packed": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields), C.POINTER(Fields),
                                          C.c_int32, C.c_void_p]),
    "grb_copy_evolved_interior": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Fields), C.c_int32,
                                            C.POINTER(Fields), C.c_int32, C.c_void_p]),
}
