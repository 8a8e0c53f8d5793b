/*
 * shoc_tr.h -- plain-C description of one SHOC window for the 3D tracer
 * transport step (advection + implicit vertical diffusion).
 *
 * Every array here is a SHOC sparse array with SHOC's own numbering: index 0
 * is the unused slot, wet cells are numbered layer by layer from the surface
 * layer down, lateral ghost cells follow each layer's wet cells and the
 * sediment (bottom ghost) cells come last.  Lists such as w3_t are 1-based,
 * exactly as in the reference.  The fields are the ones the reference hot
 * path reads from its window structs:
 *
 *   geometry_t  model/hd/include/sparse.h:660-1004
 *   window_t    model/hd/include/sparse.h:2393-2790
 *   win_priv_t  model/hd/include/sparse.h:246-654
 *
 * A SHOC maintainer fills these structs from window/windat/wincon with plain
 * pointer assignments (no copies); nothing here owns memory.
 */
#ifndef SHOC_TR_H
#define SHOC_TR_H

#ifdef __cplusplus
extern "C" {
#endif

/* Advection scheme flags: same values as model/hd/include/hd_params.h:331-344 */
#define SHOC_TR_ORDER1 0x000002      /* first-order upwind (order1) */
#define SHOC_TR_ORDER2 0x000004      /* second-order centred (order2) */
#define SHOC_TR_ORDER4 0x000010      /* fourth-order centred, uniform grid (order4) */
#define SHOC_TR_QUICKEST 0x000020    /* QUICKEST, non-uniform grid (quickest) */
#define SHOC_TR_QUICKEST_CO 0x000040 /* QUICKEST, uniform grid (quickest_uniform) */
#define SHOC_TR_VANLEER 0x000080     /* Van Leer (van_leer) */
#define SHOC_TR_ORDER2_UW 0x002000   /* second-order upwind (order2_upwind) */

/* Stability flags: same values as model/hd/include/hd_params.h:237-242 */
#define SHOC_TR_ORIGINAL 1
#define SHOC_TR_SUB_STEP 2
#define SHOC_TR_SUB_STEP_NOSURF 4
#define SHOC_TR_SUB_STEP_TRACER 16

/* DRY_FRAC of model/hd/include/hd_params.h:42 */
#define SHOC_TR_DRY_FRAC 0.05

/* Status codes.  0 = success.  The reference maps the first two onto
 * hd_quit_and_dump (tracers.c:664-668 and tracers.c:4190-4193). */
#define SHOC_TR_OK 0
#define SHOC_TR_ESUBSTEP 1      /* more than itermax tracer sub-steps needed */
#define SHOC_TR_EPIVOT 2        /* zero pivot in the tridiagonal solve */
#define SHOC_TR_ENAN 3          /* NaN in a tracer after the step */
#define SHOC_TR_EGEOM 4         /* geometry fails the layout checks */
#define SHOC_TR_EUNSUPPORTED 5  /* option outside the supported set */
#define SHOC_TR_ECUDA 6         /* CUDA runtime error */
#define SHOC_TR_EARG 7          /* bad argument (NULL pointer, size) */
#define SHOC_TR_ENOMEM 8        /* device or host allocation failed */
#define SHOC_TR_ESCRATCH 9      /* problem larger than a fixed scratch area */

/* Static geometry of one window (geometry_t). */
typedef struct shoc_tr_geom {
  int nz;          /* number of layers */
  int sgsiz;       /* 3D sparse size (sgnum + 1) */
  int sgsizS;      /* 2D sparse size (sgnumS + 1) */

  /* 3D cell-centred lists: w3_t[1..v3_t] wet, ..b3_t +OBC, ..a3_t +aux,
   * ..n3_t +ghost (sparse.h geometry_t).  Closed single windows have
   * v3_t == b3_t == a3_t. */
  int n3_t, a3_t, b3_t, v3_t;
  const int *w3_t;
  /* 2D lists and the bottom cell of each column (bot_t[1..b2_t]) */
  int n2_t, a2_t, b2_t, v2_t;
  const int *w2_t;
  const int *bot_t;
  /* interior e1 / e2 faces (w3_e1[1..v3_e1], w3_e2[1..v3_e2]) */
  int v3_e1, v3_e2;
  const int *w3_e1, *w3_e2;

  /* spatial maps [sgsiz]; the 2D maps are the same arrays restricted to
   * 2D indices (1..sgsizS-1), as in SHOC */
  const int *xp1, *xm1, *yp1, *ym1, *zp1, *zm1;
  const int *m2d;                 /* 3D cell -> surface-layer (2D) cell */
  const int *s2i, *s2j, *s2k;     /* sparse -> Cartesian indices */

  /* lateral ghost cells: tr[bpt[i]] = tr[bin[i]], i = 1..nbpt */
  int nbpt;
  const int *bpt, *bin;

  /* 2D metrics [sgsizS] */
  const double *h1au1, *h2au2, *h1au2, *h2au1;
  const double *h1acell, *h2acell, *cellarea, *botz;
  /* 3D: z of the bottom face of each cell [sgsiz] */
  const double *gridz;
} shoc_tr_geom;

/* Per-window state read and written by one tracer step (window_t plus the
 * surface vectors of geometry_t that set_dz updates). */
typedef struct shoc_tr_state {
  int ntr;
  double **tr_wc;                 /* [ntr][sgsiz], updated in place */
  int *sur_t;                     /* [b2_t+1] old surface cell, set_dz output */
  int *nsur_t;                    /* [a2_t+1] new surface cell, set_dz in/out */
  const double *u1, *u2, *w;      /* face velocities [sgsiz] */
  const double *u1flux3d, *u2flux3d; /* face volume fluxes [sgsiz] */
  const double *Kz;               /* vertical diffusivity at bottom faces */
  const double *dzu1, *dzu2;      /* face thickness (horizontal diffusion) */
  const double *u1kh, *u2kh;      /* horizontal diffusivity (may be NULL) */
  const double *eta, *oldeta;     /* [sgsizS] */
  double dt;                      /* windat->dt (== windat->dttr here) */
} shoc_tr_state;

/* Options (win_priv_t flags and per-tracer attributes). */
typedef struct shoc_tr_opts {
  int trasc;                      /* SHOC_TR_QUICKEST or SHOC_TR_VANLEER */
  int ultimate;                   /* ULTIMATE limiter on/off */
  int stab;                       /* stability bits; SUB_STEP* enable sub-steps */
  double hmin;                    /* minimum cell thickness (m) */
  int ntbdy;                      /* advected tracers: tbdy[0..ntbdy-1] */
  const int *tbdy;
  int ntdif_v;                    /* vertically diffused: tdif_v[0..ntdif_v-1] */
  const int *tdif_v;
  const int *advect;              /* [ntr] per-tracer advect flag */
  const int *diffuse;             /* [ntr] per-tracer horizontal diffusion flag */
  const double *mintr, *maxtr;    /* [ntr] valid range */
  /* Optional (NULL: every tracer in every column).  Per 2D cell (SHOC 2D
   * index, [sgsizS]): the number of leading tracers, tracer numbers
   * 0..ntr2d[c2]-1, that the step updates in that water column; the others
   * keep their values.  No reference counterpart: it lets one window hold
   * several independent basins that carry different numbers of tracers, so
   * that they step in one launch (the tbdy list must be ascending when it is
   * given). */
  const int *ntr2d;
} shoc_tr_opts;

/* What one step reports besides the status code. */
typedef struct shoc_tr_diag {
  int nsub;                       /* number of advection sub-steps taken */
  double dtm;                     /* sub-step length (== dt when none) */
  long long nwarn;                /* range violations tr_bounds would warn on */
  int vc, vcs;                    /* cells / surface cells processed */
} shoc_tr_diag;

#ifdef __cplusplus
}
#endif
#endif
