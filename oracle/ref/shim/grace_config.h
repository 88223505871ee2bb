// Build configuration used when compiling the reference's numerics in place
// for the CPU checker: 3-D, Cowling metric, Gardiner-Stone EMF, HLLE,
// WENO-Z, temperature reconstruction, FOFC on, 6th-order metric derivatives.
#pragma once
#include <stdlib.h>
#define GRACE_NSPACEDIM 3
#define GRACE_3D
#define GRACE_CARTESIAN_COORDINATES
#define GRACE_ENABLE_OMP
#define GRACE_ENABLE_FOFC
#define GRACE_METRIC_EVOL_COWLING 0
#define GRACE_METRIC_EVOL_Z4 1
#define GRACE_METRIC_EVOL GRACE_METRIC_EVOL_COWLING
#define GRACE_EMF_SCHEME_GS 0
#define GRACE_EMF_SCHEME_UCT 1
#define GRACE_EMF_SCHEME GRACE_EMF_SCHEME_GS
#define GRACE_RIEMANN_SOLVER_HLL 0
#define GRACE_RIEMANN_SOLVER_ADV 1
#define GRACE_RIEMANN_SOLVER_LLF 2
#define GRACE_RIEMANN_SOLVER GRACE_RIEMANN_SOLVER_HLL
#define GRACE_RECON_THERMO_TEMP
#define MATTER_METRIC_DER_ORDER 6
#define Z4C_DER_ORDER 4
#define VEC(X,Y,Z) X,Y,Z
#define EXPR(X,Y,Z) X Y Z
#define SQR(a) ((a)*(a))
#define GRACE_USE_ALWAYS_INLINE 0
#define GRACE_FORCE_INLINE inline
