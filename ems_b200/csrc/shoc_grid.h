/*
 * shoc_grid.h -- builds a SHOC-style sparse window for a closed rectangular
 * (or curvilinear) basin: the layout model/hd/master/preprocess.c:108
 * (build_sparse_map) produces, restricted to what the tracer step reads.
 *
 * Numbering: wet cells layer by layer from the surface layer (k = nz-1)
 * down, i fastest then j (preprocess.c:355-370); each layer's lateral ghost
 * cells follow its wet cells (preprocess.c:532-563); one sediment cell per
 * column comes last with a self-mapping zm1.  Slot 0 is unused.
 */
#ifndef SHOC_GRID_H
#define SHOC_GRID_H

#include "shoc_tr.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct shoc_grid_spec {
  int nx, ny, nz;              /* nce1, nce2, layers */
  const double *layers;        /* [nz+1] layer faces, layers[0] deepest */
  const double *bathy;         /* [ny*nx] bottom z (negative down) */
  const unsigned char *land;   /* [ny*nx] nonzero = land column */
  /* metrics at cell centres and faces, all [(ny+1)*(nx+1)] with row
   * stride nx+1 so faces on the i = nx / j = ny edges have values */
  const double *h1acell, *h2acell, *h1au1, *h2au1, *h1au2, *h2au2;
} shoc_grid_spec;

/* A built window.  Owns every array; geom points into them. */
typedef struct shoc_grid {
  shoc_tr_geom geom;
  int nx, ny, nz;
  int nwet;                    /* wet 3D cells (== a3_t) */
  int ncol;                    /* wet columns (== b2_t) */
  int nghost;                  /* lateral ghost cells */
  int *kbot;                   /* [ny*nx] bottom layer, -1 for land */
  int *map_top;                /* [ny*nx] surface-layer cell, 0 for land */
  int *is_wet;                 /* [sgsiz] 1 for wet cells */
  /* owned storage */
  int *w3_t, *w2_t, *bot_t, *w3_e1, *w3_e2;
  int *xp1, *xm1, *yp1, *ym1, *zp1, *zm1, *m2d, *s2i, *s2j, *s2k;
  int *bpt, *bin;
  double *h1au1, *h2au2, *h1au2, *h2au1, *h1acell, *h2acell, *cellarea, *botz;
  double *gridz;
} shoc_grid;

/* Returns 0 on success, SHOC_TR_EGEOM on an inconsistent spec,
 * SHOC_TR_ENOMEM on allocation failure. */
int shoc_grid_build(const shoc_grid_spec *spec, shoc_grid *out);
void shoc_grid_free(shoc_grid *g);

/* Surface vectors for a free surface at eta: nsur_t[cc] is the cell holding
 * the surface (the walk of tracers.c:5756-5769); sur_t is set equal. */
void shoc_grid_init_surface(const shoc_grid *g, const double *eta,
                            int *sur_t, int *nsur_t);

/* Vertical velocity from continuity, bottom up (the z-model branch of
 * model/hd/momentum/vel3d.c:4609 vel_w_update, no sources): w at the bottom
 * face of each column's bottom cell is 0 and w[zp1] = (flux into cell c
 * from below and the sides) / cellarea, up to the cell below the surface
 * cell sur_t.  w is zeroed first. */
void shoc_grid_w_from_continuity(const shoc_grid *g, const int *sur_t,
                                 const double *u1flux3d,
                                 const double *u2flux3d, double *w);

#ifdef __cplusplus
}
#endif
#endif

/* ---- seeded synthetic fields (loops over every wet cell / face) ---- */
#ifdef __cplusplus
extern "C" {
#endif
/* Face volume fluxes of a closed basin from a corner transport
 * streamfunction psi [(ny+1)*(nx+1)] (barotropic, spread over each face's
 * wet layers by thickness) plus a baroclinic part amp [ny*nx] * |U| / D *
 * dz * (q - qbar) whose depth integral is zero on every face; scaled so the
 * largest face velocity is umax.  Fills u1, u2, u1flux3d, u2flux3d, dzu1,
 * dzu2 [sgsiz] (zero elsewhere).  eta: free surface [sgsizS]. */
int shoc_synth_flow(const shoc_grid *g, const double *psi, const double *amp,
                    const double *eta, double umax, double *u1, double *u2,
                    double *u1flux3d, double *u2flux3d, double *dzu1, double *dzu2);
/* Kz at bottom faces: k0 * (k1/k0)^(depth of the face / column depth). */
void shoc_synth_kz_exp(const shoc_grid *g, double k0, double k1, double *Kz);
/* Kz log-uniform in [lo, hi], independent per cell (counter-based RNG). */
void shoc_synth_kz_logu(const shoc_grid *g, unsigned long long seed, double lo,
                        double hi, double *Kz);
/* Tracer n: mag_n * exp(1.5 (sm_n - 0.5) + 0.25 N + 0.3 cos(pi k / nz + n)), N a
 * unit-variance Irwin-Hall (four-uniform) deviate from a counter-based hash,
 * mag_n log-spaced in [lo_mag, hi_mag]; sm [ntr*ny*nx] smooth fields. */
void shoc_synth_tracers_logn(const shoc_grid *g, unsigned long long seed, int ntr,
                             double lo_mag, double hi_mag, const double *sm,
                             double *tr);
#ifdef __cplusplus
}
#endif
