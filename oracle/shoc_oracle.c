/*
 * shoc_oracle.c -- CPU restatement of SHOC's 3D tracer step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is
 * compared against; nothing in the product links or calls it.  It restates,
 * in its own code, the algorithm of model/hd/tracers/tracers.c (citations
 * per function below) for closed z-coordinate windows: no OBCs, no sigma, no
 * thin-layer merging, no point sources, passive tracers (zero surface and
 * bottom fluxes).  Built with -O2 -ffp-contract=off.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "shoc_oracle.h"

#define SF 0.8          /* fraction of the Courant limit, tracers.c:427 */

/* Strips of a decomposed basin (tests of ems_b200.decomp): the columns whose
 * cells count in the sub-step minimum (owned2d[c2] != 0; NULL: all), and a
 * basin-wide minimum imposed on the schedule (0: the window's own). */
static const int *oracle_owned = NULL;
static double oracle_dmin_given = 0.0;
void oracle_set_owned(const int *owned2d) { oracle_owned = owned2d; }
void oracle_set_substep_min(double dmin) { oracle_dmin_given = dmin; }
#define MINVAL 1e-10    /* minimum velocity, tracers.c:428 */
#define ITERMAX 20      /* maximum sub-steps, tracers.c:430 */
#define CLIP_EPS 1e-5   /* tr_bounds clipping threshold, tracers.c:3230 */

struct oracle_ctx {
  int sgsiz, sgsizS, ntr, nz;
  /* cells to process (set_dz outputs, wincon->s1/i1/i2/i3/vc..) */
  int *s1, *i1, *i2, *i3, *cbt;
  int vc, vcs, vc1, vcs1;
  /* wincon work arrays */
  double *dz, *w5, *w6, *w7, *w8, *w9, *d1, *d2, *d3, *d4;
  double *Fx, *Fy, *Fz, *dtracer;
  double *dzface, *Kzw, *Cm1, *C, *Cp1;
  /* implicit_vdiff_tr column vectors */
  double *rhs, *sol, *ud, *B, *Bm1, *Bp1, *vdz;
};

static double *dz_(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }
static int *iz_(size_t n) { return (int *)calloc(n ? n : 1, sizeof(int)); }

oracle_ctx *oracle_create(const shoc_tr_geom *g, int ntr) {
  oracle_ctx *o = (oracle_ctx *)calloc(1, sizeof(oracle_ctx));
  if (!o) return NULL;
  size_t S = (size_t)g->sgsiz, S2 = (size_t)g->sgsizS;
  o->sgsiz = g->sgsiz; o->sgsizS = g->sgsizS; o->ntr = ntr; o->nz = g->nz;
  o->s1 = iz_(S); o->i1 = iz_(S2); o->i2 = iz_(S2); o->i3 = iz_(S2); o->cbt = iz_(S2);
  o->dz = dz_(S); o->w5 = dz_(S); o->w6 = dz_(S); o->w7 = dz_(S); o->w8 = dz_(S);
  o->w9 = dz_(S); o->d1 = dz_(S2); o->d2 = dz_(S2); o->d3 = dz_(S2); o->d4 = dz_(S2);
  o->Fx = dz_(S); o->Fy = dz_(S); o->Fz = dz_(S); o->dtracer = dz_(S);
  o->dzface = dz_(S); o->Kzw = dz_(S); o->Cm1 = dz_(S); o->C = dz_(S); o->Cp1 = dz_(S);
  size_t nzp = (size_t)g->nz + 1;
  o->rhs = dz_(nzp); o->sol = dz_(nzp); o->ud = dz_(nzp); o->B = dz_(nzp);
  o->Bm1 = dz_(nzp); o->Bp1 = dz_(nzp); o->vdz = dz_(nzp);
  return o;
}

void oracle_destroy(oracle_ctx *o) {
  if (!o) return;
  void *p[] = {o->s1, o->i1, o->i2, o->i3, o->cbt, o->dz, o->w5, o->w6, o->w7,
               o->w8, o->w9, o->d1, o->d2, o->d3, o->d4, o->Fx, o->Fy, o->Fz,
               o->dtracer, o->dzface, o->Kzw, o->Cm1, o->C, o->Cp1, o->rhs,
               o->sol, o->ud, o->B, o->Bm1, o->Bp1, o->vdz};
  for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++) free(p[i]);
  free(o);
}

/* No-flux lateral boundary: each ghost takes its interior value
 * (set_lateral_BC_tr, tracers.c:5574-5592). */
static void lateral_bc(const shoc_tr_geom *g, shoc_tr_state *st) {
  for (int cc = 1; cc <= g->nbpt; cc++)
    for (int n = 0; n < st->ntr; n++) st->tr_wc[n][g->bpt[cc]] = st->tr_wc[n][g->bin[cc]];
}

/* Cells to process and layer thicknesses, z-coordinates
 * (set_dz, tracers.c:5731-5848). */
static void set_dz(oracle_ctx *o, const shoc_tr_geom *g, shoc_tr_state *st,
                   const shoc_tr_opts *op) {
  const int *zm1 = g->zm1, *zp1 = g->zp1;
  /* new surface cell of every column: walk down from the surface layer
   * until the cell's bottom face is below eta (:5739-5755) */
  for (int cc = 1; cc <= g->a2_t; cc++) {
    int c = g->w2_t[cc], cs = c;
    if (cc <= g->b2_t) st->sur_t[cc] = st->nsur_t[cc];
    int m = zm1[c];
    while (c != m && g->gridz[c] >= st->eta[cs]) {
      c = m;
      m = zm1[c];
    }
    st->nsur_t[cc] = c;
  }
  /* surface cells first: the lower of the old / new surface (:5778-5800) */
  int vc = 1;
  for (int cc = 1; cc <= g->b2_t; cc++) {
    int c = st->sur_t[cc] > st->nsur_t[cc] ? st->sur_t[cc] : st->nsur_t[cc];
    int cs = g->m2d[c];
    double top = st->eta[cs] < st->oldeta[cs] ? st->eta[cs] : st->oldeta[cs];
    double bot = SHOC_TR_DRY_FRAC * op->hmin + g->botz[cs];
    if (top > bot && c != zm1[c]) {
      o->s1[vc] = c;
      o->i1[vc] = g->bot_t[cc];
      o->i2[vc] = st->nsur_t[cc];
      o->i3[vc] = st->sur_t[cc];
      if (cc == g->v2_t) o->vcs1 = vc;
      vc++;
    }
  }
  o->vcs = vc - 1;
  /* then each column's sub-surface cells down to the bottom (:5804-5817) */
  for (int cc = 1; cc <= o->vcs; cc++) {
    int c = zm1[o->s1[cc]];
    int m = zm1[c];
    while (c != m) {
      o->s1[vc++] = c;
      c = m;
      m = zm1[c];
    }
    if (cc == o->vcs1) o->vc1 = vc - 1;
  }
  o->vc = vc - 1;
  /* thicknesses: old surface cell from oldeta, the rest from gridz, the
   * bottom cell from botz; cells above the old surface copy the surface
   * thickness (:5824-5846) */
  for (int cc = 1; cc <= g->b2_t; cc++) {
    int c = st->sur_t[cc], c3 = c;
    int c2 = g->m2d[c3];
    int cbot = g->bot_t[cc];
    double top = st->oldeta[c2];
    while (c3 < cbot) {
      double bot = g->gridz[c3];
      o->dz[c3] = top - bot;
      top = bot;
      c3 = zm1[c3];
    }
    o->dz[cbot] = top - g->botz[c2];
    c3 = c;
    while (c > c2) {
      c = zp1[c];
      o->dz[c] = o->dz[c3];
    }
  }
}

/* QUICKEST face values on a non-uniform grid (quickest, tracers.c:1819-1931).
 * Fx/Fy over w3_t[1..a3_t], Fz over s1[1..vc]. */
static void quickest(oracle_ctx *o, const shoc_tr_geom *g, const double *tr) {
  double *Fx = o->Fx, *Fy = o->Fy, *Fz = o->Fz;
  memset(Fx, 0, (size_t)g->n3_t * sizeof(double));
  memset(Fy, 0, (size_t)g->n3_t * sizeof(double));
  memset(Fz, 0, (size_t)g->n3_t * sizeof(double));
  for (int cc = 1; cc <= g->a3_t; cc++) {
    int c = g->w3_t[cc], c2 = g->m2d[c];
    int xp1 = g->xp1[c], yp1 = g->yp1[c], xm1 = g->xm1[c], ym1 = g->ym1[c];
    int xm2 = g->xm1[xm1], ym2 = g->ym1[ym1];
    int xm1s = g->xm1[c2], xp1s = g->xp1[c2], ym1s = g->ym1[c2], yp1s = g->yp1[c2];
    double cx = o->w6[c];
    double db = 2.0 / (g->h1au1[xm1s] + g->h1au1[c2]);
    double df = 2.0 / (g->h1au1[c2] + g->h1au1[xp1s]);
    double face = o->d3[c2] * (tr[c] - tr[xm1]) + tr[xm1];
    double grad = tr[c] - tr[xm1];
    double curv = 0.0;
    if (cx > 0.0)
      curv = db * (g->h1au1[xm1s] * tr[c] + g->h1au1[c2] * tr[xm2]) - 2.0 * tr[xm1];
    else if (cx < 0.0)
      curv = df * (g->h1au1[c2] * tr[xp1] + g->h1au1[xp1s] * tr[xm1]) - 2.0 * tr[c];
    Fx[c] = face - 0.5 * cx * grad - (1.0 - cx * cx) * curv / 6.0;

    double cy = o->w7[c];
    db = 2.0 / (g->h2au2[ym1s] + g->h2au2[c2]);
    df = 2.0 / (g->h2au2[c2] + g->h2au2[yp1s]);
    face = o->d4[c2] * (tr[c] - tr[ym1]) + tr[ym1];
    grad = tr[c] - tr[ym1];
    curv = 0.0;
    if (cy > 0.0)
      curv = db * (g->h2au2[ym1s] * tr[c] + g->h2au2[c2] * tr[ym2]) - 2.0 * tr[ym1];
    else if (cy < 0.0)
      curv = df * (g->h2au2[c2] * tr[yp1] + g->h2au2[yp1s] * tr[ym1]) - 2.0 * tr[c];
    Fy[c] = face - 0.5 * cy * grad - (1.0 - cy * cy) * curv / 6.0;
  }
  for (int cc = 1; cc <= o->vc; cc++) {
    int c = o->s1[cc];
    int zp1 = g->zp1[c], zm1 = g->zm1[c], zm2 = g->zm1[zm1];
    double cz = o->w8[c];
    double db = 2.0 / (o->w9[zm1] + o->w9[c]);
    double df = 2.0 / (o->w9[c] + o->w9[zp1]);
    double face = o->w5[c] * (tr[c] - tr[zm1]) + tr[zm1];
    double grad = tr[c] - tr[zm1];
    double curv = 0.0;
    if (cz > 0.0)
      curv = db * (o->w9[zm1] * tr[c] + o->w9[c] * tr[zm2]) - 2.0 * tr[zm1];
    else if (cz < 0.0)
      curv = df * (o->w9[c] * tr[zp1] + o->w9[zp1] * tr[zm1]) - 2.0 * tr[c];
    Fz[c] = face - 0.5 * cz * grad - (1.0 - cz * cz) * curv / 6.0;
  }
}

/* Van Leer limited upwind face value (van_leer_do, tracers.c:2087-2119). */
static void van_leer_do(double *F, const double *tr, const double *vel,
                        const double *cn, int ss, int se, const int *sdo,
                        const int *fmap, const int *bmap) {
  for (int cc = ss; cc <= se; cc++) {
    int c = sdo[cc], bm1 = bmap[c], bm2 = bmap[bm1];
    double df;
    if (vel[c] > 0.0) {
      df = (tr[bm1] - tr[bm2]) * (tr[c] - tr[bm1]);
      if (df > 0.0)
        df = 2.0 * df / (tr[c] - tr[bm2]);
      else
        df = 0.0;
      F[c] = tr[bm1] + 0.5 * (1.0 - cn[c]) * df;
    } else if (vel[c] < 0.0) {
      df = (tr[c] - tr[bm1]) * (tr[fmap[c]] - tr[c]);
      if (df > 0.0)
        df = 2.0 * df / (tr[fmap[c]] - tr[bm1]);
      else
        df = 0.0;
      F[c] = tr[c] - 0.5 * (1.0 + cn[c]) * df;
    }
  }
}

/* van_leer, tracers.c:2037-2075 */
static void van_leer(oracle_ctx *o, const shoc_tr_geom *g, const shoc_tr_state *st,
                     const double *tr) {
  memset(o->Fx, 0, (size_t)g->n3_t * sizeof(double));
  van_leer_do(o->Fx, tr, st->u1, o->w6, 1, g->v3_e1, g->w3_e1, g->xp1, g->xm1);
  van_leer_do(o->Fx, tr, st->u1, o->w6, g->v3_t + 1, g->a3_t, g->w3_t, g->xp1, g->xm1);
  memset(o->Fy, 0, (size_t)g->n3_t * sizeof(double));
  van_leer_do(o->Fy, tr, st->u2, o->w7, 1, g->v3_e2, g->w3_e2, g->yp1, g->ym1);
  van_leer_do(o->Fy, tr, st->u2, o->w7, g->v3_t + 1, g->a3_t, g->w3_t, g->yp1, g->ym1);
  memset(o->Fz, 0, (size_t)g->n3_t * sizeof(double));
  van_leer_do(o->Fz, tr, st->w, o->w8, 1, o->vc, o->s1, g->zp1, g->zm1);
}

/* ULTIMATE universal limiter (ulimate_filter, tracers.c:3501-3557). */
static void ultimate(const double *cr, double *Fx, const double *F, const int *ctp,
                     int vs, int ve, const int *mapm, const int *mapp) {
  for (int cc = vs; cc <= ve; cc++) {
    int c = ctp[cc];
    if (cr[c] == 0.0) continue;
    double tc, tu, td;
    if (cr[c] > 0.0) {
      int m1 = mapm[c];
      tc = F[m1];
      tu = F[mapm[m1]];
      td = F[c];
    } else {
      tc = F[c];
      tu = F[mapp[c]];
      td = F[mapm[c]];
    }
    double diff = td - tu;
    double nc = 0.0, nu = 0.0;
    if (diff != 0.0) {
      nc = (tc - tu) / diff;
      nu = (Fx[c] - tu) / diff;
    }
    if (nc >= 0.0 && nc <= 1.0) {
      if (nu > 1.0)
        Fx[c] = td;
      else if (nu < nc)
        Fx[c] = tu + nc * (td - tu);
      else if (nu > nc / fabs(cr[c]))
        Fx[c] = tu + nc * (td - tu) / fabs(cr[c]);
    } else
      Fx[c] = tu + nc * (td - tu);
  }
}

/* Face fluxes: scheme, limiter, times volume flux (advect, tracers.c:1487-1576) */
static void advect(oracle_ctx *o, const shoc_tr_geom *g, const shoc_tr_state *st,
                   const shoc_tr_opts *op, const double *tr, double dtu) {
  if (op->trasc == SHOC_TR_QUICKEST)
    quickest(o, g, tr);
  else
    van_leer(o, g, st, tr);
  if (op->ultimate) {
    ultimate(o->w6, o->Fx, tr, g->w3_e1, 1, g->v3_e1, g->xm1, g->xp1);
    ultimate(o->w6, o->Fx, tr, g->w3_t, g->v3_t + 1, g->a3_t, g->xm1, g->xp1);
    ultimate(o->w7, o->Fy, tr, g->w3_e2, 1, g->v3_e2, g->ym1, g->yp1);
    ultimate(o->w7, o->Fy, tr, g->w3_t, g->v3_t + 1, g->a3_t, g->ym1, g->yp1);
    ultimate(o->w8, o->Fz, tr, o->s1, 1, o->vc, g->zm1, g->zp1);
  }
  for (int cc = 1; cc <= g->a3_t; cc++) {
    int c = g->w3_t[cc];
    o->Fx[c] *= st->u1flux3d[c];
    o->Fy[c] *= st->u2flux3d[c];
  }
  for (int cc = 1; cc <= o->vc; cc++) {
    int c = o->s1[cc];
    o->Fz[c] *= (st->w[c] * dtu);
  }
}

/* Horizontal diffusive fluxes, z-model branch (hor_diffuse, tracers.c:3652-3667);
 * mdx = mdy = 1 for the z-model. */
static void hor_diffuse(oracle_ctx *o, const shoc_tr_geom *g, const shoc_tr_state *st,
                        const double *tr) {
  for (int cc = 1; cc <= g->a3_t; cc++) {
    int c = g->w3_t[cc], c2 = g->m2d[c];
    int xm1 = g->xm1[c], ym1 = g->ym1[c];
    double csx = st->dzu1[c] * g->h2au1[c2] * 1.0;
    double csy = st->dzu2[c] * g->h1au2[c2] * 1.0;
    o->Fx[c] -= (csx * st->u1kh[c] * (tr[c] - tr[xm1]) / g->h1au1[c2]);
    o->Fy[c] -= (csy * st->u2kh[c] * (tr[c] - tr[ym1]) / g->h2au2[c2]);
  }
}

/* Mass-conserving surface concentration (surf_conc, tracers.c:3047-3207). */
static double surf_conc(oracle_ctx *o, const shoc_tr_geom *g, const double *tr,
                        double subeta, int c, int c2, int cc, double fcbot,
                        const shoc_tr_opts *op) {
  int cb = o->i1[cc], co = o->i3[cc];
  double osubeta = o->d1[c2];
  double waterbot = (c == cb) ? g->botz[c2] : g->gridz[c];
  double dz = subeta - waterbot;
  double svol = dz * g->cellarea[c2];
  double surftr = -fcbot;
  while (c != co) {
    int zp1 = g->zp1[c];
    double watertop = g->gridz[zp1];
    surftr += (tr[c] * g->cellarea[c2] * (watertop - waterbot) - o->dtracer[c]);
    c = zp1;
    waterbot = g->gridz[c];
  }
  double watertop = osubeta;
  waterbot = (c == cb) ? g->botz[c2] : g->gridz[c];
  surftr += (tr[c] * g->cellarea[c2] * (watertop - waterbot) - o->dtracer[c]);
  if (c != c2) {
    do {
      c = g->zp1[c];
      surftr -= (o->dtracer[c]);
    } while (c != c2);
  }
  if (svol == 0.0 || (surftr < 0.0 && dz <= op->hmin))
    surftr = 0.0;
  else
    surftr /= svol;
  return surftr;
}

/* Range handling after each sub-step (tr_bounds, tracers.c:3217-3324). */
static long long tr_bounds(oracle_ctx *o, const shoc_tr_geom *g, shoc_tr_state *st,
                           const shoc_tr_opts *op) {
  long long nwarn = 0;
  const double *mn = op->mintr, *mx = op->maxtr;
  for (int cc = 1; cc <= o->vcs1; cc++) {
    int c = o->s1[cc], c3 = c;
    int co = o->i3[cc], cb = o->i1[cc];
    if (c < cb && o->dz[co] < op->hmin) {
      for (int nn = 0; nn < op->ntbdy; nn++) {
        int n = op->tbdy[nn];
        double *tr = st->tr_wc[n];
        if (tr[c] < mn[n] || tr[c] > mx[n]) {
          /* c3 is not reset between tracers (tracers.c:3253-3270): after
           * the first replaced tracer it stays at the top of the column */
          double surftr = tr[g->zm1[c]];
          tr[c3] = surftr;
          while (c3 != g->zp1[c3]) {
            c3 = g->zp1[c3];
            tr[c3] = surftr;
          }
        }
      }
    }
  }
  for (int cc = 1; cc <= o->vc1; cc++) {
    int c = o->s1[cc];
    for (int nn = 0; nn < op->ntbdy; nn++) {
      int n = op->tbdy[nn];
      double *tr = st->tr_wc[n];
      if (mn[n] <= CLIP_EPS && tr[c] < mn[n]) tr[c] = mn[n];
      if (tr[c] < mn[n] || tr[c] > mx[n]) nwarn++;
    }
  }
  for (int cc = 1; cc <= o->vcs; cc++) {
    int c = o->s1[cc], cs = c;
    while (c != g->zp1[c]) {
      c = g->zp1[c];
      for (int nn = 0; nn < op->ntbdy; nn++) {
        int n = op->tbdy[nn];
        st->tr_wc[n][c] = st->tr_wc[n][cs];
      }
    }
  }
  return nwarn;
}

/* Advection + horizontal diffusion with sub-stepping
 * (advect_diffuse, tracers.c:401-1054; QUICKEST/VANLEER branches). */
static int advect_diffuse(oracle_ctx *o, const shoc_tr_geom *g, shoc_tr_state *st,
                          const shoc_tr_opts *op, shoc_tr_diag *diag) {
  const int *zm1m = g->zm1;
  double *osubeta = o->d1, *subeta = o->d2;
  const double *u1 = st->u1, *u2 = st->u2, *w = st->w;
  int vc = o->vc, vcs = o->vcs;

  /* scheme work arrays (:561-577 QUICKEST, :530-535 Van Leer) */
  if (op->trasc == SHOC_TR_VANLEER) {
    for (int cc = 1; cc <= g->b3_t; cc++) {
      int c = g->w3_t[cc];
      o->w9[c] = 0.5 * (o->dz[c] + o->dz[zm1m[c]]);
    }
  } else {
    for (int cc = 1; cc <= g->b3_t; cc++) {
      int c = g->w3_t[cc], zm1 = zm1m[c];
      o->w5[c] = o->dz[zm1] / (o->dz[zm1] + o->dz[c]);
      o->w9[c] = 0.5 * (o->dz[c] + o->dz[zm1]);
    }
    for (int cc = 1; cc <= g->n2_t; cc++) {
      int c = g->w2_t[cc], c2 = g->m2d[c];
      int xm1 = g->xm1[c2], ym1 = g->ym1[c2];
      o->d3[c2] = g->h1acell[xm1] / (g->h1acell[xm1] + g->h1acell[c2]);
      o->d4[c2] = g->h2acell[ym1] / (g->h2acell[ym1] + g->h2acell[c2]);
    }
  }

  /* minimum sub-step (:591-668) */
  double dtu = st->dt, dtm = st->dt;
  if (op->stab & (SHOC_TR_SUB_STEP | SHOC_TR_SUB_STEP_NOSURF | SHOC_TR_SUB_STEP_TRACER)) {
    for (int cc = 1; cc <= vc; cc++) {
      int c = o->s1[cc], c2 = g->m2d[c];
      if (oracle_owned && !oracle_owned[c2]) continue;
      int xp1 = g->xp1[c], yp1 = g->yp1[c], zp1 = g->zp1[c];
      double d4 = 0.5 * (u1[c] + u1[xp1]);
      if (fabs(d4) < MINVAL) d4 = MINVAL;
      double d1 = SF * fabs(g->h1acell[c2] / d4);
      if (d1 < dtm) dtm = d1;
      d4 = 0.5 * (u2[c] + u2[yp1]);
      if (fabs(d4) < MINVAL) d4 = MINVAL;
      double d2 = SF * fabs(g->h2acell[c2] / d4);
      if (d2 < dtm) dtm = d2;
      d4 = (cc <= vcs) ? 0.0 : 0.5 * (w[c] + w[zp1]);
      if (fabs(d4) < MINVAL) d4 = MINVAL;
      double d3 = (cc <= vcs) ? dtu : SF * fabs(o->dz[c] * 1.0 / d4);
      if (d3 > 0.0 && d3 < dtm) dtm = d3;
    }
    if (dtm != dtu) dtm = floor(dtm);
    if (oracle_dmin_given > 0.0) {  /* a decomposed basin's minimum */
      dtm = dtu;
      if (oracle_dmin_given < dtm) dtm = oracle_dmin_given;
      if (dtm != dtu) dtm = floor(dtm);
    }
  }
  if (diag) diag->dtm = dtm;
  if (dtm == 0.0 || (int)(dtu / dtm) > ITERMAX) return SHOC_TR_ESUBSTEP;

  for (int cc = 1; cc <= vcs; cc++) {
    int c2 = g->m2d[o->s1[cc]];
    osubeta[c2] = st->oldeta[c2];
  }

  int nsub = 0;
  long long nwarn = 0;
  double trem = dtu;
  while (trem > 0) {
    dtu = dtm;
    if (trem < dtu) dtu = trem;
    if (dtu > 0.0) {
      nsub++;
      /* Courant numbers (:726-737) */
      for (int cc = 1; cc <= g->n3_t; cc++) {
        int c = g->w3_t[cc], c2 = g->m2d[c];
        o->w6[c] = u1[c] * dtu / g->h1au1[c2];
        o->w7[c] = u2[c] * dtu / g->h2au2[c2];
        o->w8[c] = w[c] * dtu / (o->w9[c] * 1.0);
      }
      /* sub-step surface elevation (:746-756) */
      for (int cc = 1; cc <= vcs; cc++) {
        int c2 = g->m2d[o->s1[cc]];
        subeta[c2] = st->oldeta[c2] +
                     (1.0 + (dtu - trem) / st->dt) * (st->eta[c2] - st->oldeta[c2]);
      }
      /* tracer loop (:773-988) */
      for (int nn = 0; nn < op->ntbdy; nn++) {
        int n = op->tbdy[nn];
        double *tr = st->tr_wc[n];
        tr[0] = (double)n;
        memset(o->Fx, 0, (size_t)g->sgsiz * sizeof(double));
        memset(o->Fy, 0, (size_t)g->sgsiz * sizeof(double));
        memset(o->Fz, 0, (size_t)g->sgsiz * sizeof(double));
        memset(o->dtracer, 0, (size_t)g->sgsiz * sizeof(double));
        /* no-gradient bottom ghost (:827-830) */
        for (int cc = 1; cc <= g->b2_t; cc++) {
          int cb = g->bot_t[cc];
          tr[zm1m[cb]] = tr[cb];
        }
        if (op->advect[n]) advect(o, g, st, op, tr, dtu);
        if (op->diffuse[n]) hor_diffuse(o, g, st, tr);
        for (int cc = 1; cc <= g->b3_t; cc++) {
          int c = g->w3_t[cc];
          o->dtracer[c] = (o->Fx[g->xp1[c]] - o->Fx[c] + o->Fy[g->yp1[c]] - o->Fy[c]) * dtu;
        }
        /* interior cells (:912-925); Ds = Hn1 = 1 for the z-model */
        for (int cc = vcs + 1; cc <= o->vc1; cc++) {
          int c = o->s1[cc], c2 = g->m2d[c], zp1 = g->zp1[c];
          tr[c] *= 1.0;
          tr[c] -= ((o->dtracer[c] / g->cellarea[c2] + (o->Fz[zp1] - o->Fz[c])) / o->dz[c]);
          tr[c] /= 1.0;
        }
        /* surface cells (:944-961) */
        if (op->advect[n]) {
          for (int cc = 1; cc <= o->vcs1; cc++) {
            int c = o->s1[cc], c2 = g->m2d[c];
            double top = -o->Fz[c] * g->cellarea[c2];
            double surftr = surf_conc(o, g, tr, subeta[c2], c, c2, cc, top, op);
            tr[c] = (g->botz[c2] > 0.0 && o->dz[c] < op->hmin) ? tr[c] : surftr;
          }
        }
      }
      nwarn += tr_bounds(o, g, st, op);
      for (int cc = 1; cc <= vcs; cc++) {
        int c2 = g->m2d[o->s1[cc]];
        osubeta[c2] = subeta[c2];
      }
    }
    trem -= dtu;
  }
  if (diag) {
    diag->nsub = nsub;
    diag->nwarn += nwarn;
  }
  return SHOC_TR_OK;
}

/* Implicit vertical diffusion (vert_diffuse_3d, tracers.c:3782-3957, and
 * implicit_vdiff_tr, tracers.c:4067-4214) with zero surface and bottom
 * fluxes, no sources, scale = 1, no thin-layer merging. */
static int vert_diffuse_3d(oracle_ctx *o, const shoc_tr_geom *g, shoc_tr_state *st,
                           const shoc_tr_opts *op) {
  const int *zm1m = g->zm1, *zp1m = g->zp1;
  double dt = st->dt;
  int *ctp = o->i2, *cbt = o->cbt;
  double *dzface = o->w7, *dzcell = o->w9, *Kz = o->Kzw;
  double *Cm1 = o->Cm1, *C = o->C, *Cp1 = o->Cp1;
  memset(o->d1, 0, (size_t)g->sgsizS * sizeof(double));
  memset(o->d2, 0, (size_t)g->sgsizS * sizeof(double));
  memcpy(dzcell, o->dz, (size_t)g->sgsiz * sizeof(double));
  memcpy(Kz, st->Kz, (size_t)g->sgsiz * sizeof(double));

  /* tracer-independent tridiagonal coefficients (:3841-3889) */
  for (int cc = 1; cc <= o->vcs; cc++) {
    int c = ctp[cc], cs = c;
    int zm1 = zm1m[c];
    if (zm1 == zm1m[zm1] || !dzcell[zm1]) continue;
    while (c != zm1 && dzcell[c]) {
      dzface[c] = 0.5 * (dzcell[zm1] + dzcell[c]);
      dzcell[c] *= 1.0;
      Kz[c] /= 1.0;
      c = zm1;
      zm1 = zm1m[c];
    }
    int cb = c = zp1m[c];
    int zp1 = zp1m[c];
    cbt[cc] = cb;
    double dzdt = dzcell[c] / dt;
    Cm1[c] = 0.0;
    Cp1[c] = -Kz[zp1] / dzface[zp1];
    C[c] = dzdt - Cp1[c];
    while (zp1 != cs) {
      c = zp1;
      zp1 = zp1m[c];
      dzdt = dzcell[c] / dt;
      Cm1[c] = -Kz[c] / dzface[c];
      Cp1[c] = -Kz[zp1] / dzface[zp1];
      C[c] = dzdt - Cm1[c] - Cp1[c];
    }
    c = cs;
    dzdt = dzcell[c] / dt;
    Cm1[c] = -Kz[c] / dzface[c];
    Cp1[c] = 0.0;
    C[c] = dzdt - Cm1[c];
  }

  double *fb = o->d1, *ft = o->d2;
  double *rhs = o->rhs, *sol = o->sol, *ud = o->ud, *B = o->B, *Bm1 = o->Bm1,
         *Bp1 = o->Bp1, *vdz = o->vdz;
  for (int nn = 0; nn < op->ntdif_v; nn++) {
    int n = op->tdif_v[nn];
    double *var = st->tr_wc[n];
    for (int cc = 1; cc <= o->vcs; cc++) {
      int c = ctp[cc], cs = c;
      int cb = cbt[cc];
      int c2 = g->m2d[c];
      int zm1 = zm1m[c];
      /* single layer (:4125-4132); cth is all zero without thin merging */
      if (zm1 == zm1m[zm1] || !dzcell[zm1]) {
        double h = dzcell[cs] > op->hmin ? dzcell[cs] : op->hmin;
        var[cs] += dt * (fb[c2] - ft[c2]) / h;
        if (c != 0) var[0] = var[cs];
        continue;
      }
      int ks = g->s2k[cs], kb = g->s2k[cb];
      c = cs;
      for (int k = ks; k >= kb; k--) {
        B[k] = C[c];
        Bm1[k] = Cm1[c];
        Bp1[k] = Cp1[c];
        vdz[k] = dzcell[c];
        c = zm1m[c];
      }
      double dzdt = vdz[kb] / dt;
      rhs[kb] = dzdt * var[cb] + fb[c2];
      c = zp1m[cb];
      for (int k = kb + 1; k < ks; k++) {
        dzdt = vdz[k] / dt;
        rhs[k] = dzdt * var[c];
        c = zp1m[c];
      }
      dzdt = vdz[ks] / dt;
      rhs[ks] = dzdt * var[cs] - ft[c2];
      double div = B[kb];
      sol[kb] = rhs[kb] / div;
      for (int k = kb + 1; k <= ks; k++) {
        ud[k] = Bp1[k - 1] / div;
        div = B[k] - Bm1[k] * ud[k];
        if (div == 0.0) return SHOC_TR_EPIVOT;
        sol[k] = (rhs[k] - Bm1[k] * sol[k - 1]) / div;
      }
      c = cs;
      var[cs] += (sol[ks] - var[cs]) * 1.0;
      for (int k = ks - 1; k >= kb; k--) {
        c = zm1m[c];
        sol[k] -= ud[k + 1] * sol[k + 1];
        var[c] += (sol[k] - var[c]) * 1.0;
      }
      /* thin-layer slot: cth[cc] == 0 here, so slot 0 absorbs the update */
      if (cs != 0) var[0] += (sol[ks] - var[cs]) * 1.0;
    }
  }
  return SHOC_TR_OK;
}

int oracle_step(oracle_ctx *o, const shoc_tr_geom *g, shoc_tr_state *st,
                const shoc_tr_opts *op, shoc_tr_diag *diag) {
  if (!o || !g || !st || !op) return SHOC_TR_EARG;
  if (op->trasc != SHOC_TR_QUICKEST && op->trasc != SHOC_TR_VANLEER)
    return SHOC_TR_EUNSUPPORTED;
  if (diag) memset(diag, 0, sizeof(*diag));
  lateral_bc(g, st);
  set_dz(o, g, st, op);
  if (diag) {
    diag->vc = o->vc;
    diag->vcs = o->vcs;
  }
  int rc = advect_diffuse(o, g, st, op, diag);
  if (rc) return rc;
  rc = vert_diffuse_3d(o, g, st, op);
  if (rc) return rc;
  for (int n = 0; n < st->ntr; n++)
    for (int cc = 1; cc <= g->a3_t; cc++)
      if (isnan(st->tr_wc[n][g->w3_t[cc]])) return SHOC_TR_ENAN;
  return SHOC_TR_OK;
}

int oracle_run(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op,
               int nsteps, shoc_tr_diag *diag) {
  oracle_ctx *o = oracle_create(g, st->ntr);
  if (!o) return SHOC_TR_ENOMEM;
  int rc = SHOC_TR_OK;
  shoc_tr_diag d, acc;
  memset(&acc, 0, sizeof(acc));
  for (int s = 0; s < nsteps && rc == SHOC_TR_OK; s++) {
    rc = oracle_step(o, g, st, op, &d);
    acc.nsub = d.nsub;
    acc.dtm = d.dtm;
    acc.nwarn += d.nwarn;
    acc.vc = d.vc;
    acc.vcs = d.vcs;
  }
  if (diag) *diag = acc;
  oracle_destroy(o);
  return rc;
}
