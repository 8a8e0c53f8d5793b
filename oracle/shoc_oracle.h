/*
 * shoc_oracle.h -- CPU restatement of SHOC's 3D tracer step (TEST
 * INFRASTRUCTURE ONLY: the checker for the CUDA path, never linked into it).
 *
 * oracle_step() performs, on one window, the sequence the reference runs per
 * tracer step for a closed z-coordinate window:
 *   set_lateral_BC_tr  model/hd/tracers/tracers.c:5574
 *   set_dz             model/hd/tracers/tracers.c:5682 (z branch :5731-5848)
 *   advect_diffuse     model/hd/tracers/tracers.c:401-1054
 *   vert_diffuse_3d    model/hd/tracers/tracers.c:3782-3957
 *     implicit_vdiff_tr model/hd/tracers/tracers.c:4067-4214
 * with QUICKEST (non-uniform, :1819-1931) or Van Leer (:2037-2119) face
 * values, the ULTIMATE limiter (:3501-3557), horizontal diffusion
 * (:3595-3668), surf_conc (:3047-3207) and tr_bounds (:3217-3324).
 * Compile with -ffp-contract=off so every product and sum is rounded the way
 * the reference's are.
 */
#ifndef SHOC_ORACLE_H
#define SHOC_ORACLE_H

#include "shoc_tr.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

/* Work arrays persist across steps the way wincon's do (vcs1 / vc1 and the
 * work array shared by w9 and dzcell keep their values between calls). */
oracle_ctx *oracle_create(const shoc_tr_geom *g, int ntr);
void oracle_destroy(oracle_ctx *o);

/* One tracer step; tracers and sur_t/nsur_t in st are updated in place. */
int oracle_step(oracle_ctx *o, const shoc_tr_geom *g, shoc_tr_state *st,
                const shoc_tr_opts *op, shoc_tr_diag *diag);

/* Strips of a decomposed basin: only columns with owned2d[c2] != 0 count in
 * the sub-step minimum (NULL: all; the array must outlive the steps), and a
 * given basin-wide minimum replaces the window's own (0: none). */
void oracle_set_owned(const int *owned2d);
void oracle_set_substep_min(double dmin);

/* nsteps steps; stops at the first non-zero status. */
int oracle_run(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op,
               int nsteps, shoc_tr_diag *diag);

#ifdef __cplusplus
}
#endif
#endif
