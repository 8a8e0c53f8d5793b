/*
 * shoc_tr_gpu.h -- C-ABI of the B200 tracer-transport step for SHOC.
 *
 * Replaces, for one window, the calls tracer_step_3d makes between
 * set_lateral_BC_tr and the auxiliary routines:
 *
 *   set_lateral_BC_tr  model/hd/tracers/tracers.c:5574 (called from :159)
 *   set_dz             model/hd/tracers/tracers.c:5682 (called from
 *                      model/hd/tracers/transport.c:457 / the 3D mode)
 *   advect_diffuse     model/hd/tracers/tracers.c:401  (called from :265)
 *   vert_diffuse_3d    model/hd/tracers/tracers.c:3782 (called from :279)
 *
 * with the same inputs (shoc_tr.h mirrors the window structs), the same
 * results, and the same failures reported as status codes instead of
 * hd_quit_and_dump: SHOC_TR_ESUBSTEP where tracers.c:664-668 quits,
 * SHOC_TR_EPIVOT where tracers.c:4190-4193 quits.  There is no CPU path:
 * without a usable CUDA device every entry point returns SHOC_TR_ECUDA.
 *
 * Typical use from the driver (one handle per window, created once):
 *
 *   shoc_tr_gpu_create(&geom, &opts, ntr, SHOC_TR_FP64, device, &h);
 *   each step:  shoc_tr_gpu_step(h, &state, &diag);      // host arrays in/out
 *
 * or, keeping tracers resident on the GPU between steps:
 *
 *   shoc_tr_gpu_upload_tracers(h, tr_wc);
 *   shoc_tr_gpu_set_flow(h, &state);       // whenever u/w/Kz/eta change
 *   shoc_tr_gpu_run(h, nsteps);            // asynchronous on the stream
 *   shoc_tr_gpu_sync(h, &diag);
 *   shoc_tr_gpu_download_tracers(h, tr_wc);
 *
 * A handle is not thread-safe; each window uses its own handle and stream,
 * as each dp worker thread owns its window in the reference
 * (model/hd/control/dp.c:351-359).
 */
#ifndef SHOC_TR_GPU_H
#define SHOC_TR_GPU_H

#include <stddef.h>

#include "shoc_tr.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Arithmetic of the step. */
#define SHOC_TR_FP64 0        /* plain: FP64 everywhere, matches tracers.c */
#define SHOC_TR_FP32_MIXED 1  /* FP32 tracers/fluxes/Thomas, FP64 mass sums
                                 and one FP64-residual refinement per solve */
#define SHOC_TR_FP32_COMP 2   /* FP32_MIXED with a 16-bit compensation stored
                                 beside every FP32 value (6 bytes a value): a
                                 value changing by less than half an FP32 ulp
                                 per step keeps its changes.  Two-kernel
                                 sub-step only (no fused k_step32); a
                                 decomposed basin's halo exchange answers
                                 SHOC_TR_EUNSUPPORTED; columns the general
                                 path steps (surface crossing a layer face)
                                 keep their FP32 values and restart their
                                 compensation at 0 */

typedef struct shoc_tr_gpu shoc_tr_gpu;

/* Builds the device copy of the window (maps, lists, metrics) and the
 * tracer / work buffers.  The geometry arrays are copied; the caller may free
 * them afterwards.  Replaces the per-window set-up the reference does in
 * win_consts_init / dp_init (model/hd/master/hd_init.c:244-256). */
int shoc_tr_gpu_create(const shoc_tr_geom *geom, const shoc_tr_opts *opts,
                       int ntr, int precision, int device, shoc_tr_gpu **out);
void shoc_tr_gpu_destroy(shoc_tr_gpu *h);

/* One step on host arrays: copies st's tracers, surface vectors and flow
 * fields to the device, runs the step, copies tracers and surface vectors
 * back into st, and waits.  Drop-in for set_lateral_BC_tr + set_dz +
 * advect_diffuse + vert_diffuse_3d on one window.  The tracers travel in
 * chunks, so the copies back of the first chunks overlap the copies up of
 * the later ones and the step of every chunk; the results are those of
 * shoc_tr_gpu_upload_tracers + shoc_tr_gpu_run(h, 1) +
 * shoc_tr_gpu_download_tracers, bit for bit.  Copies reach the host link's
 * speed only from page-locked memory: see shoc_tr_gpu_host_register.  With
 * SHOC_TR_FP32_MIXED the handle keeps its per-column mass carry (the FP64
 * mass the FP32-stored values owe each column) from one call to the next:
 * the values it belongs to come back unchanged through the FP64 host arrays,
 * so a run of drop-in steps equals the same steps on resident tracers. */
int shoc_tr_gpu_step(shoc_tr_gpu *h, shoc_tr_state *st, shoc_tr_diag *diag);

/* Page-locks (cudaHostRegister) / releases a host array the caller passes to
 * shoc_tr_gpu_step every step (tracers, flow fields), so its copies run at
 * the host link's full speed without a staging copy.  No counterpart in the
 * reference: an addition of this library for a host model that keeps its
 * window arrays for the whole run.  Register once after allocating the
 * array and unregister before freeing it. */
int shoc_tr_gpu_host_register(void *ptr, size_t bytes);
int shoc_tr_gpu_host_unregister(void *ptr);

/* Device-resident use.  Uploading tracers starts from new values: the
 * FP32-mixed path's mass carry is cleared. */
int shoc_tr_gpu_upload_tracers(shoc_tr_gpu *h, double *const *tr_wc);
int shoc_tr_gpu_download_tracers(shoc_tr_gpu *h, double **tr_wc);
/* Copies flow fields (u1, u2, w, fluxes, Kz, dzu1/dzu2/u1kh/u2kh when any
 * tracer diffuses horizontally, eta, oldeta, dt) and the surface vectors
 * sur_t / nsur_t. */
int shoc_tr_gpu_set_flow(shoc_tr_gpu *h, const shoc_tr_state *st);
int shoc_tr_gpu_get_surface(shoc_tr_gpu *h, int *sur_t, int *nsur_t);
/* Transport-mode flow preamble.  With on != 0, every step (shoc_tr_gpu_run
 * and shoc_tr_gpu_step) first computes on the device what SHOC's transport
 * mode computes before the tracer step (transport_step, model/hd/tracers/
 * transport.c:436-462): dzu1 / dzu2 (set_dz_at_u1 / set_dz_at_u2, model/hd/
 * momentum/vel3d.c:720, :2718), u1flux3d / u2flux3d (set_flux_3d,
 * vel3d.c:4041, VEL3D) from the state's u1, u2 and eta, and w from
 * continuity (vel_w_update, vel3d.c:4609, CONS_W) with wtop = detadt.  Then
 * the state's w, u1flux3d, u2flux3d, dzu1 and dzu2 are neither read nor
 * needed (they may be NULL).  Covers z-level windows without open
 * boundaries, a linear free surface, no point sources of water and
 * mdx = mdy = 1; SHOC_TR_EUNSUPPORTED where the window's w3_e1 / w3_e2 are
 * not one run of faces from the surface layer down per face column.
 * set_detadt copies the surface velocity detadt [sgsizS] (used by every
 * following step; call it after set_preamble(h, 1)); get_flow copies the
 * device's current fields back (any pointer may be NULL). */
int shoc_tr_gpu_set_preamble(shoc_tr_gpu *h, int on);
int shoc_tr_gpu_set_detadt(shoc_tr_gpu *h, const double *detadt);
int shoc_tr_gpu_get_flow(shoc_tr_gpu *h, double *u1flux3d, double *u2flux3d, double *w,
                         double *dzu1, double *dzu2);
/* Enqueues nsteps steps on the handle's stream (CUDA-graph replays once the
 * sub-step schedule is known).  May synchronise once after set_flow to learn
 * the sub-step count. */
int shoc_tr_gpu_run(shoc_tr_gpu *h, int nsteps);
/* Waits for the stream and returns the first error status raised on the
 * device since the last sync (and clears it). */
int shoc_tr_gpu_sync(shoc_tr_gpu *h, shoc_tr_diag *diag);

/* Checkpoint and resume of the device-resident state: the tracers in the
 * handle's own precision, the FP32-mixed path's per-column mass carry and
 * the surface vectors, as one versioned raw image (header: magic, version,
 * precision, ntr, sgsiz, columns, carry flag).  state_size gives the image's
 * bytes; save copies it into buf (host memory), load puts it back into a
 * handle of the same window and precision (else SHOC_TR_EARG).  A resumed
 * run (load + set_flow + run) continues bit for bit where the saved one
 * left off.  The reference restarts from the NetCDF state it dumps
 * (restart_name / restart_dt, model/hd/inputs/readparam.c:1143-1145); this
 * image is the library's own device state, with no counterpart there. */
int shoc_tr_gpu_state_size(shoc_tr_gpu *h, size_t *bytes);
int shoc_tr_gpu_save_state(shoc_tr_gpu *h, void *buf, size_t bytes);
int shoc_tr_gpu_load_state(shoc_tr_gpu *h, const void *buf, size_t bytes);

/* Total tracer mass of every tracer: sum of tr * dz * cellarea over each
 * column from its current surface cell (top at eta) to the bottom (botz),
 * accumulated in FP64 with compensated (Neumaier) summation.  mass[ntr]. */
int shoc_tr_gpu_mass(shoc_tr_gpu *h, double *mass);

/* The same mass reduction, allocating nothing (no counterpart in the
 * reference: an addition of this library).  For host frameworks that hand
 * out all device memory from a pool they reserved at start-up and forbid
 * any other cudaMalloc once the run is going (a coupled model sharing the
 * GPU with other components, say): shoc_tr_gpu_mass allocates a small
 * stream-ordered buffer on every call, this entry point does not.  The
 * per-block partial sums go to a fixed device array of about 152 KB (room
 * for 64 tracers) that every device loading the library holds until the
 * process exits; with more tracers it returns SHOC_TR_ESCRATCH.  The first
 * call on a device looks the array's device address up once
 * (cudaGetSymbolAddress) and keeps it, so do not keep using the library
 * across a reset of the device (cudaDeviceReset).  All calls share the one array: calls whose GPU
 * work overlaps in time (two handles on different streams, say) race and
 * must be serialised by the caller.  mass[ntr] is host memory; the call
 * copies the sums into it and waits for its stream before returning. */
int shoc_tr_gpu_mass_noalloc(shoc_tr_gpu *h, double *mass);

/* Differences between the current tracers of two handles of the same window
 * on the same device, in either precision (the FP32-mixed path against the
 * plain FP64 one, say), computed on the device.  Over the wet cells of every
 * column that carries the tracer in both handles: the largest |a - b|, the
 * largest |b|, sum (a - b)^2 and sum b^2 per tracer -- per region when
 * region[sgsizS] (SHOC 2D cell -> region 0..nregion-1, < 0: left out) is
 * given, else over the whole window (nregion 1).  Outputs [nregion][ntr].
 * Waits for both handles' streams.  No reference counterpart: the accuracy
 * measurement of this library. */
int shoc_tr_gpu_compare(shoc_tr_gpu *a, shoc_tr_gpu *b, const int *region, int nregion,
                        double *maxabs, double *maxref, double *sumsq_diff, double *sumsq_ref);

/* The other per-column tridiagonal solves of SHOC, batched over every water
 * column of the window (from its bottom cell to its current surface cell,
 * nsur_t of the last step or of set_flow; dry columns are left alone), in
 * FP64 with the reference's arithmetic (bitwise its results).  Arrays are
 * host arrays indexed by SHOC cell, [sgsiz] (a cell carries the row of its
 * layer; the reference gathers the rows into layer vectors first), or by 2D
 * cell, [sgsizS].  A zero divisor returns SHOC_TR_EPIVOT where the
 * reference quits.
 *
 * shoc_tr_gpu_tridiag replaces the closures' tridiagonal
 * (model/hd/closure/MY2-5.c:499-536, called by the MY2-5, k-e and k-w
 * closures): C (main diagonal), Cm1 (lower), Cp1 (upper), rhs; var receives
 * max(solution, minvar).
 *
 * shoc_tr_gpu_vdiff_cols replaces implicit_vdiff_at_cc
 * (model/hd/tracers/tracers.c:7407-7545) for every column at once: var is
 * diffused in place with the coefficients C, Cm1, Cp1, the cell thicknesses
 * dzcell, the fluxes out of the bottom and the top fb, ft [sgsizS], the
 * source parts Splus, Sminus (NULL: none) and the scale [sgsizS]; a column
 * whose surface lies in its bottom layer takes the reference's one-layer
 * update with the window's dt (set_flow) and hmin.  No thin layers. */
int shoc_tr_gpu_tridiag(shoc_tr_gpu *h, const double *C, const double *Cm1, const double *Cp1,
                        const double *rhs, double *var, double minvar);
int shoc_tr_gpu_vdiff_cols(shoc_tr_gpu *h, double *var, const double *dzcell, const double *C,
                           const double *Cm1, const double *Cp1, const double *fb,
                           const double *ft, const double *Splus, const double *Sminus,
                           const double *scale, double dt);

/* One basin decomposed over several GPUs: each GPU steps one strip of
 * columns as its own window, widened by halo columns that are copies of its
 * neighbours' columns.  QUICKEST and ULTIMATE reach two cells across a face
 * (tracers.c:1854-1855, :3528-3530), so with halos 2 x (sub-steps per step)
 * columns wide, exchanged once per step, every owned column steps exactly as
 * in the undivided basin (the halos' outer columns go wrong and are
 * overwritten at the next exchange).  This replaces, for this path, SHOC's
 * window transfers (win_data_fill_3d / win_data_empty_3d,
 * model/hd/slaves/transfers.c:349,769, over the MPI buffers of
 * model/hd/slaves/TransferBuffer.cpp:282-443); the caller moves the buffers
 * between GPUs (NCCL send/recv, or a peer copy into a local buffer).
 *   halo_plan    the cells this window sends and receives (SHOC cell
 *                numbers, host arrays; copied to the device).
 *   halo_pack    writes every tracer's send-cell values into buf (device
 *                memory, [ntr][nsend] values of the handle's precision) and
 *                waits for its stream, so buf is ready for the transfer.
 *   halo_unpack  enqueues on the handle's stream the copy of buf ([ntr][nrecv]
 *                values, device memory) into the receive cells of both
 *                tracer buffers; the next run sees it.
 *   mass_region  shoc_tr_gpu_mass over the columns whose 2D cell has
 *                region[c2] == reg (a strip's own columns). */
int shoc_tr_gpu_halo_plan(shoc_tr_gpu *h, int nsend, const int *send_cells, int nrecv,
                          const int *recv_cells);
int shoc_tr_gpu_halo_pack(shoc_tr_gpu *h, void *buf);
int shoc_tr_gpu_halo_unpack(shoc_tr_gpu *h, const void *buf);
int shoc_tr_gpu_mass_region(shoc_tr_gpu *h, const int *region, int reg, double *mass);
/* The sub-step length of a step is the basin-wide minimum of the stability
 * criterion (tracers.c:591-668): a strip must take the basin's, not its own.
 *   set_owned        owned2d[sgsizS] (1: the strip's own column, 0: halo;
 *                    NULL: every column) -- only owned columns count below.
 *   substep_min      the criterion's minimum over the owned columns for the
 *                    current flow and surface (+inf: no sub-stepping
 *                    needed); changes no state.
 *   set_substep_min  the basin-wide minimum (the smallest substep_min of
 *                    all strips) the window's steps then use; 0 goes back to
 *                    the window's own.  Call after set_flow, before run. */
int shoc_tr_gpu_set_owned(shoc_tr_gpu *h, const int *owned2d);
int shoc_tr_gpu_substep_min(shoc_tr_gpu *h, double *dmin);
int shoc_tr_gpu_set_substep_min(shoc_tr_gpu *h, double dmin);

/* cudaStream_t of the handle, for event timing by the caller. */
void *shoc_tr_gpu_stream(shoc_tr_gpu *h);

/* Launch tuning: columns per block (32; 0 keeps it) and tracers per block
 * of the column kernel (0 keeps it).  Takes effect at the next step. */
int shoc_tr_gpu_set_tiling(shoc_tr_gpu *h, int cols_per_block, int tracers_per_block);

/* The transport kernels' launch configuration.  No reference counterpart
 * (launch tuning of this library). */
typedef struct {
  int fused;             /* FP32-mixed: 1 one fused launch per sub-step (k_step32),
                            0 the advection + column kernel pair */
  int tracers_per_block; /* column kernel: tracers per k_vd64 block (1..8), or warps per
                            k_vd32 block, each stepping its share of the tracers (1..16) */
  int tile_x;            /* k_step32: tile width along i (8, 16, 32; 32 / tile_x
                            columns along j) */
  int phase_b_warps;     /* k_step32: warps of its column phase */
  int prefetch;          /* k_vd32: 1 stages the next tracer's column while the
                            current one is solved (twice the per-warp shared memory) */
} shoc_tr_tuning;
/* set_tuning validates (SHOC_TR_EUNSUPPORTED for a configuration the window
 * or the shared memory does not allow) and takes effect at the next step.
 * Results are bitwise independent of tracers_per_block, tile_x and
 * phase_b_warps; the FP32-mixed fused and two-kernel sub-steps agree to FP32
 * rounding. */
int shoc_tr_gpu_get_tuning(shoc_tr_gpu *h, shoc_tr_tuning *t);
int shoc_tr_gpu_set_tuning(shoc_tr_gpu *h, const shoc_tr_tuning *t);

/* Autotuner: from the current state, runs `steps` trial steps with each
 * candidate configuration, times the transport kernels with CUDA events,
 * puts the state back (a device copy taken before the trials: the tracers,
 * surface vectors and mass carry are as they were) and keeps the fastest.
 * Candidates: 2..8 tracers per k_vd64 block, or 2..16 warps per k_vd32
 * block with and without its prefetch; for FP32-mixed also the fused sub-step with tile widths 8, 16, 32 and the most and half
 * the most phase-B warps its shared memory allows.  With use_cache != 0 the
 * choice is looked up in and saved to a file keyed by the GPU model and the
 * window's configuration (sizes, tracers, precision, scheme, diffusion),
 * named by the environment variable SHOC_TR_TUNE_CACHE (default
 * $HOME/.cache/shoc_tr_gpu/tuning.txt, "off" for none): a cached choice is
 * applied without trial steps and *from_cache set to 1.  best / from_cache
 * may be NULL.  Call after the flow is set and any earlier step synced.
 * The device copy holds one tracer buffer (ntr x S values, plus their
 * compensations with SHOC_TR_FP32_COMP); without room for it the call
 * returns SHOC_TR_ENOMEM and changes nothing.
 * shoc_tr_gpu_autotune is autotune_ex without the cache, returning the
 * tracers per block. */
int shoc_tr_gpu_autotune_ex(shoc_tr_gpu *h, int steps, int use_cache, shoc_tr_tuning *best,
                            int *from_cache);
int shoc_tr_gpu_autotune(shoc_tr_gpu *h, int steps, int *tracers_per_block);

/* Time of the transport of a step's last sub-step (the transport kernels
 * of the precision: one launch for SHOC_TR_FP64, the advection and the column
 * kernel for SHOC_TR_FP32_MIXED), averaged over the steps since the last call
 * (CUDA events on the handle's stream; enabled by shoc_tr_gpu_profile(h, 1)).
 * No reference counterpart: measurement hooks of this library. */
int shoc_tr_gpu_profile(shoc_tr_gpu *h, int enable);
int shoc_tr_gpu_kernel_time(shoc_tr_gpu *h, double *ms_per_launch, int *launches);
/* The same for one part: 0 the whole transport (as above), 1 the advection
 * kernel, 2 the column kernel (tr_bounds, surf_conc, vertical diffusion) of
 * SHOC_TR_FP32_MIXED. */
int shoc_tr_gpu_kernel_time_part(shoc_tr_gpu *h, int part, double *ms_per_launch,
                                 int *launches);

/* Counts of kernels this library launched since creation. */
long long shoc_tr_gpu_launch_count(shoc_tr_gpu *h);

const char *shoc_tr_gpu_strerror(int status);

#ifdef __cplusplus
}
#endif
#endif
