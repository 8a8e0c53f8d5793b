/*
 * shoc_grid.c -- SHOC-style sparse window builder for closed basins.
 *
 * Restates the parts of model/hd/master/preprocess.c:108 build_sparse_map
 * that the tracer transport step depends on:
 *   - wet cells numbered surface layer first, i fastest then j
 *     (preprocess.c:355-370, :549-563);
 *   - one lateral ghost cell per (wet cell, side facing a dry cell), placed
 *     after that layer's wet cells, with wet->ghost and ghost->wet maps and a
 *     bpt/bin entry so set_lateral_BC_tr copies the wet value into it
 *     (preprocess.c:700-820);
 *   - one sediment cell per column at the end of the array: zm1 of the
 *     bottom cell points to it, its own zm1 is self-mapping
 *     (preprocess.c:589-592, :660-680);
 *   - surface-layer cells double as the 2D index (m2d), as in SHOC.
 * Diagonal / inside-corner ghost cells are not generated: they are used only
 * by the semi-Lagrangian schemes (comment at preprocess.c:1180-1186), and the
 * QUICKEST / Van Leer stencils never step diagonally.
 */
#include <stdlib.h>
#include <string.h>
#include "shoc_grid.h"

#define G3(k, j, i) (((size_t)(k) * ny + (j)) * nx + (i))

enum { DW = 0, DE = 1, DS = 2, DN = 3 };

static void *xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

int shoc_grid_build(const shoc_grid_spec *sp, shoc_grid *g) {
  const int nx = sp->nx, ny = sp->ny, nz = sp->nz;
  const int mx = nx + 1; /* metric row stride */
  memset(g, 0, sizeof(*g));
  if (nx < 1 || ny < 1 || nz < 1) return SHOC_TR_EGEOM;
  g->nx = nx; g->ny = ny; g->nz = nz;

  int *kbot = (int *)xcalloc((size_t)nx * ny, sizeof(int));
  if (!kbot) return SHOC_TR_ENOMEM;
  g->kbot = kbot;
  /* Bottom layer: layers[k] <= bathy < layers[k+1] (preprocess.c:253-258) */
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int idx = j * nx + i;
      kbot[idx] = -1;
      if (sp->land[idx]) continue;
      double b = sp->bathy[idx];
      for (int k = 0; k < nz; k++)
        if (b >= sp->layers[k] && b < sp->layers[k + 1]) kbot[idx] = k;
      if (kbot[idx] < 0) return SHOC_TR_EGEOM;
    }
#define WET(k, j, i)                                                        \
  ((i) >= 0 && (i) < nx && (j) >= 0 && (j) < ny && kbot[(j) * nx + (i)] >= 0 && \
   (k) >= kbot[(j) * nx + (i)])

  /* Count cells per layer */
  size_t n3 = (size_t)nz * ny * nx;
  int *map = (int *)xcalloc(n3, sizeof(int));
  if (!map) return SHOC_TR_ENOMEM;
  long nwet = 0, ngh = 0, ncol = 0;
  for (int k = nz - 1; k >= 0; k--)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        if (WET(k, j, i)) {
          nwet++;
          ngh += !WET(k, j, i - 1) + !WET(k, j, i + 1) + !WET(k, j - 1, i) +
                 !WET(k, j + 1, i);
          if (k == nz - 1) ncol++;
        }
  long sgnum = nwet + ngh + ncol;
  if (sgnum + 1 > 0x7fffffffL) { free(map); return SHOC_TR_EGEOM; }
  int sgsiz = (int)sgnum + 1;
  g->nwet = (int)nwet;
  g->ncol = (int)ncol;
  g->nghost = (int)ngh;

#define IA(p, n) if (!((p) = (int *)xcalloc((size_t)(n), sizeof(int)))) goto oom
#define DA(p, n) if (!((p) = (double *)xcalloc((size_t)(n), sizeof(double)))) goto oom
  IA(g->xp1, sgsiz); IA(g->xm1, sgsiz); IA(g->yp1, sgsiz); IA(g->ym1, sgsiz);
  IA(g->zp1, sgsiz); IA(g->zm1, sgsiz); IA(g->m2d, sgsiz);
  IA(g->s2i, sgsiz); IA(g->s2j, sgsiz); IA(g->s2k, sgsiz);
  IA(g->is_wet, sgsiz); DA(g->gridz, sgsiz);
  IA(g->w3_t, nwet + ngh + 1); IA(g->w3_e1, nwet + 1); IA(g->w3_e2, nwet + 1);
  IA(g->bpt, ngh + 1); IA(g->bin, ngh + 1);
  IA(g->map_top, (size_t)nx * ny);

  /* Number wet cells and ghosts layer by layer.  ghost[c*4+d] is the ghost
   * on side d of wet cell c. */
  int *ghost = (int *)xcalloc((size_t)sgsiz * 4, sizeof(int));
  if (!ghost) goto oom;
  int c = 1, nb = 0;
  int top_end = 0; /* last index of the surface layer (wet + ghosts) */
  for (int k = nz - 1; k >= 0; k--) {
    int first = c;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        if (WET(k, j, i)) {
          map[G3(k, j, i)] = c;
          g->is_wet[c] = 1;
          g->s2i[c] = i; g->s2j[c] = j; g->s2k[c] = k;
          g->gridz[c] = sp->layers[k];
          c++;
        }
    int last = c;
    for (int cw = first; cw < last; cw++) {
      int i = g->s2i[cw], j = g->s2j[cw];
      const int di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
      for (int d = 0; d < 4; d++) {
        if (WET(k, j + dj[d], i + di[d])) continue;
        ghost[(size_t)cw * 4 + d] = c;
        g->s2i[c] = i + di[d]; g->s2j[c] = j + dj[d]; g->s2k[c] = k;
        g->gridz[c] = sp->layers[k];
        nb++;
        g->bpt[nb] = c;
        g->bin[nb] = cw;
        c++;
      }
    }
    if (k == nz - 1) top_end = c - 1;
  }
  int sed0 = c;
  (void)sed0;
  /* Self-mapping everywhere first (preprocess.c:611-618) */
  for (int s = 0; s < sgsiz; s++) {
    g->xp1[s] = g->xm1[s] = g->yp1[s] = g->ym1[s] = g->zp1[s] = g->zm1[s] = s;
  }
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++)
      if (kbot[j * nx + i] >= 0) g->map_top[j * nx + i] = map[G3(nz - 1, j, i)];

  /* Sediment cells, one per column in 2D order */
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int kb = kbot[j * nx + i];
      if (kb < 0) continue;
      int cb = map[G3(kb, j, i)];
      g->zm1[cb] = c;
      g->zp1[c] = cb;
      g->s2i[c] = i; g->s2j[c] = j; g->s2k[c] = kb - 1;
      g->gridz[c] = sp->bathy[j * nx + i];
      g->m2d[c] = g->map_top[j * nx + i];
      c++;
    }
  if (c != sgsiz) { free(ghost); goto geom_err; }

  /* Maps of wet cells and their ghosts */
  for (int s = 1; s < sgsiz; s++) {
    if (!g->is_wet[s]) continue;
    int i = g->s2i[s], j = g->s2j[s], k = g->s2k[s];
    g->m2d[s] = g->map_top[j * nx + i];
    g->xm1[s] = WET(k, j, i - 1) ? map[G3(k, j, i - 1)] : ghost[(size_t)s * 4 + DW];
    g->xp1[s] = WET(k, j, i + 1) ? map[G3(k, j, i + 1)] : ghost[(size_t)s * 4 + DE];
    g->ym1[s] = WET(k, j - 1, i) ? map[G3(k, j - 1, i)] : ghost[(size_t)s * 4 + DS];
    g->yp1[s] = WET(k, j + 1, i) ? map[G3(k, j + 1, i)] : ghost[(size_t)s * 4 + DN];
    if (k > kbot[j * nx + i]) g->zm1[s] = map[G3(k - 1, j, i)];
    if (k < nz - 1) g->zp1[s] = map[G3(k + 1, j, i)];
    /* ghost -> wet maps */
    int gw = ghost[(size_t)s * 4 + DW], ge = ghost[(size_t)s * 4 + DE];
    int gs = ghost[(size_t)s * 4 + DS], gn = ghost[(size_t)s * 4 + DN];
    if (gw) { g->xp1[gw] = s; g->m2d[gw] = g->m2d[s]; }
    if (ge) { g->xm1[ge] = s; g->m2d[ge] = g->m2d[s]; }
    if (gs) { g->yp1[gs] = s; g->m2d[gs] = g->m2d[s]; }
    if (gn) { g->ym1[gn] = s; g->m2d[gn] = g->m2d[s]; }
  }
  free(ghost);
  free(map);
  map = NULL;

  /* Lists */
  int n = 0, ne1 = 0, ne2 = 0;
  for (int s = 1; s < sgsiz; s++)
    if (g->is_wet[s]) {
      g->w3_t[++n] = s;
      if (g->is_wet[g->xm1[s]]) g->w3_e1[++ne1] = s;
      if (g->is_wet[g->ym1[s]]) g->w3_e2[++ne2] = s;
    }
  for (int b = 1; b <= nb; b++) g->w3_t[++n] = g->bpt[b];
  int sgsizS = top_end + 1;
  IA(g->w2_t, sgsizS + 1); IA(g->bot_t, ncol + 1);
  int n2 = 0;
  for (int s = 1; s <= top_end; s++)
    if (g->is_wet[s]) {
      g->w2_t[++n2] = s;
      int i = g->s2i[s], j = g->s2j[s];
      int cb = s;
      while (g->zm1[cb] != cb && g->is_wet[g->zm1[cb]]) cb = g->zm1[cb];
      (void)i; (void)j;
      g->bot_t[n2] = cb;
    }
  int nwet2 = n2;
  for (int s = 1; s <= top_end; s++)
    if (!g->is_wet[s]) g->w2_t[++n2] = s;

  /* 2D metrics at every surface-layer cell (wet and ghost), read at the
   * cell's own (i, j) position; positions off the grid edge are clamped. */
  DA(g->h1au1, sgsizS); DA(g->h2au2, sgsizS); DA(g->h1au2, sgsizS);
  DA(g->h2au1, sgsizS); DA(g->h1acell, sgsizS); DA(g->h2acell, sgsizS);
  DA(g->cellarea, sgsizS); DA(g->botz, sgsizS);
  for (int s = 1; s < sgsizS; s++) {
    int i = g->s2i[s], j = g->s2j[s];
    if (i < 0) i = 0;
    if (j < 0) j = 0;
    if (i > nx) i = nx;
    if (j > ny) j = ny;
    size_t m = (size_t)j * mx + i;
    g->h1au1[s] = sp->h1au1[m];
    g->h2au1[s] = sp->h2au1[m];
    g->h1au2[s] = sp->h1au2[m];
    g->h2au2[s] = sp->h2au2[m];
    g->h1acell[s] = sp->h1acell[m];
    g->h2acell[s] = sp->h2acell[m];
    g->cellarea[s] = g->h1acell[s] * g->h2acell[s];
    int ii = i < nx ? i : nx - 1, jj = j < ny ? j : ny - 1;
    g->botz[s] = g->is_wet[s] ? sp->bathy[jj * nx + ii] : sp->layers[nz];
  }

  shoc_tr_geom *G = &g->geom;
  G->nz = nz;
  G->sgsiz = sgsiz;
  G->sgsizS = sgsizS;
  G->v3_t = G->b3_t = G->a3_t = (int)nwet;
  G->n3_t = n;
  G->v2_t = G->b2_t = G->a2_t = nwet2;
  G->n2_t = n2;
  G->w3_t = g->w3_t; G->w2_t = g->w2_t; G->bot_t = g->bot_t;
  G->v3_e1 = ne1; G->v3_e2 = ne2; G->w3_e1 = g->w3_e1; G->w3_e2 = g->w3_e2;
  G->xp1 = g->xp1; G->xm1 = g->xm1; G->yp1 = g->yp1; G->ym1 = g->ym1;
  G->zp1 = g->zp1; G->zm1 = g->zm1; G->m2d = g->m2d;
  G->s2i = g->s2i; G->s2j = g->s2j; G->s2k = g->s2k;
  G->nbpt = nb; G->bpt = g->bpt; G->bin = g->bin;
  G->h1au1 = g->h1au1; G->h2au2 = g->h2au2; G->h1au2 = g->h1au2;
  G->h2au1 = g->h2au1; G->h1acell = g->h1acell; G->h2acell = g->h2acell;
  G->cellarea = g->cellarea; G->botz = g->botz; G->gridz = g->gridz;
  return SHOC_TR_OK;

geom_err:
  free(map);
  shoc_grid_free(g);
  return SHOC_TR_EGEOM;
oom:
  free(map);
  shoc_grid_free(g);
  return SHOC_TR_ENOMEM;
#undef IA
#undef DA
#undef WET
}

void shoc_grid_free(shoc_grid *g) {
  void *p[] = {g->kbot, g->map_top, g->is_wet, g->w3_t, g->w2_t, g->bot_t,
               g->w3_e1, g->w3_e2, g->xp1, g->xm1, g->yp1, g->ym1, g->zp1,
               g->zm1, g->m2d, g->s2i, g->s2j, g->s2k, g->bpt, g->bin,
               g->h1au1, g->h2au2, g->h1au2, g->h2au1, g->h1acell,
               g->h2acell, g->cellarea, g->botz, g->gridz};
  for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++) free(p[i]);
  memset(g, 0, sizeof(*g));
}

void shoc_grid_init_surface(const shoc_grid *g, const double *eta, int *sur_t,
                            int *nsur_t) {
  const shoc_tr_geom *G = &g->geom;
  for (int cc = 1; cc <= G->a2_t; cc++) {
    int c = G->w2_t[cc], cs = c;
    int zm1 = G->zm1[c];
    while (c != zm1 && G->gridz[c] >= eta[cs]) {
      c = zm1;
      zm1 = G->zm1[c];
    }
    nsur_t[cc] = c;
    if (cc <= G->b2_t) sur_t[cc] = c;
  }
}

void shoc_grid_w_from_continuity(const shoc_grid *g, const int *sur_t,
                                 const double *u1flux3d,
                                 const double *u2flux3d, double *w) {
  const shoc_tr_geom *G = &g->geom;
  memset(w, 0, (size_t)G->sgsiz * sizeof(double));
  for (int cc = 1; cc <= G->b2_t; cc++) {
    int c = G->bot_t[cc];
    int cs = G->m2d[c];
    double fcbot = 0.0;
    w[c] = 0.0;
    while (c > sur_t[cc]) {
      int xp1 = G->xp1[c], yp1 = G->yp1[c], zp1 = G->zp1[c];
      double fctop =
          fcbot + u1flux3d[c] - u1flux3d[xp1] + u2flux3d[c] - u2flux3d[yp1];
      w[zp1] = fctop / G->cellarea[cs];
      fcbot = fctop;
      c = zp1;
    }
  }
}

/* ---------------------------------------------------------------------- */
/* seeded synthetic fields                                                 */

#include <math.h>

static unsigned long long mix64(unsigned long long x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
static double u01(unsigned long long seed, unsigned long long a, unsigned long long b) {
  unsigned long long h = mix64(seed ^ mix64(a * 0x100000001b3ull + mix64(b)));
  return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

/* z of the top / bottom face of wet cell c */
static double cell_top(const shoc_grid *g, const double *eta, int c) {
  const shoc_tr_geom *G = &g->geom;
  double e = eta[G->m2d[c]];
  double t = (G->zp1[c] == c) ? e : G->gridz[G->zp1[c]];
  return t < e ? t : e;
}
static double cell_bot(const shoc_grid *g, int c) {
  const shoc_tr_geom *G = &g->geom;
  int zm = G->zm1[c];
  return g->is_wet[zm] ? G->gridz[c] : G->botz[G->m2d[c]];
}

int shoc_synth_flow(const shoc_grid *g, const double *psi, const double *amp, const double *eta,
                    double umax, double *u1, double *u2, double *u1flux3d, double *u2flux3d,
                    double *dzu1, double *dzu2) {
  const shoc_tr_geom *G = &g->geom;
  const int nx = g->nx, ny = g->ny, S = G->sgsiz;
  const size_t nf = (size_t)(nx + 1) * (ny + 1);
  double *D = (double *)calloc(nf, sizeof(double));
  double *Q = (double *)calloc(nf, sizeof(double));
  if (!D || !Q) { free(D); free(Q); return SHOC_TR_ENOMEM; }
  memset(u1, 0, S * sizeof(double)); memset(u2, 0, S * sizeof(double));
  memset(u1flux3d, 0, S * sizeof(double)); memset(u2flux3d, 0, S * sizeof(double));
  memset(dzu1, 0, S * sizeof(double)); memset(dzu2, 0, S * sizeof(double));
  double vmax = 0.0;
  for (int axis = 0; axis < 2; axis++) {
    const int *nbm = axis == 0 ? G->xm1 : G->ym1;
    double *flux = axis == 0 ? u1flux3d : u2flux3d;
    double *vel = axis == 0 ? u1 : u2;
    double *dzf = axis == 0 ? dzu1 : dzu2;
    memset(D, 0, nf * sizeof(double));
    memset(Q, 0, nf * sizeof(double));
    for (int pass = 0; pass < 3; pass++) {
      for (int cc = 1; cc <= G->a3_t; cc++) {
        int c = G->w3_t[cc], nb = nbm[c];
        if (!g->is_wet[nb]) continue;
        int i = G->s2i[c], j = G->s2j[c];
        size_t f = (size_t)j * (nx + 1) + i;
        double tp = fmin(cell_top(g, eta, c), cell_top(g, eta, nb));
        double bt = fmax(cell_bot(g, c), cell_bot(g, nb));
        double dz = tp - bt > 0.0 ? tp - bt : 0.0;
        double zmid = 0.5 * (tp + bt);
        if (pass == 0) {
          D[f] += dz;
        } else {
          double q = cos(3.141592653589793 * zmid / fmax(D[f], 1e-9));
          if (pass == 1) {
            Q[f] += dz * q;
          } else {
            double U = axis == 0 ? psi[(size_t)(j + 1) * (nx + 1) + i] - psi[f]
                                 : -(psi[(size_t)j * (nx + 1) + i + 1] - psi[f]);
            double qbar = Q[f] / D[f];
            int jj = j < ny ? j : ny - 1, ii = i < nx ? i : nx - 1;
            double a = amp[(size_t)jj * nx + ii];
            double fl = U * dz / D[f] + a * fabs(U) / D[f] * dz * (q - qbar);
            int c2 = G->m2d[c];
            double h2 = axis == 0 ? G->h2au1[c2] : G->h1au2[c2];
            double v = dz > 0.0 ? fl / (dz * h2) : 0.0;
            flux[c] = fl;
            vel[c] = v;
            dzf[c] = dz;
            if (fabs(v) > vmax) vmax = fabs(v);
          }
        }
      }
    }
  }
  double s = vmax > 0.0 ? umax / vmax : 0.0;
  for (int c = 0; c < S; c++) {
    u1[c] *= s; u2[c] *= s; u1flux3d[c] *= s; u2flux3d[c] *= s;
  }
  free(D);
  free(Q);
  return SHOC_TR_OK;
}

void shoc_synth_kz_exp(const shoc_grid *g, double k0, double k1, double *Kz) {
  const shoc_tr_geom *G = &g->geom;
  memset(Kz, 0, (size_t)G->sgsiz * sizeof(double));
  double r = log(k1 / k0);
  for (int cc = 1; cc <= G->a3_t; cc++) {
    int c = G->w3_t[cc];
    double H = -G->botz[G->m2d[c]];
    double fr = -G->gridz[c] / H;
    fr = fr < 0.0 ? 0.0 : (fr > 1.0 ? 1.0 : fr);
    Kz[c] = k0 * exp(r * fr);
  }
}

void shoc_synth_kz_logu(const shoc_grid *g, unsigned long long seed, double lo, double hi,
                        double *Kz) {
  const shoc_tr_geom *G = &g->geom;
  memset(Kz, 0, (size_t)G->sgsiz * sizeof(double));
  double a = log(lo), b = log(hi);
#pragma omp parallel for schedule(static)
  for (int cc = 1; cc <= G->a3_t; cc++) {
    int c = G->w3_t[cc];
    Kz[c] = exp(a + (b - a) * u01(seed, 0x4b7a, (unsigned long long)c));
  }
}

void shoc_synth_tracers_logn(const shoc_grid *g, unsigned long long seed, int ntr, double lo_mag,
                             double hi_mag, const double *sm, double *tr) {
  const shoc_tr_geom *G = &g->geom;
  const size_t S = (size_t)G->sgsiz, n2 = (size_t)g->nx * g->ny;
  memset(tr, 0, S * ntr * sizeof(double));
  for (int n = 0; n < ntr; n++) {
    double mag = lo_mag * pow(hi_mag / lo_mag, ntr > 1 ? (double)n / (ntr - 1) : 0.0);
    double *t = tr + (size_t)n * S;
    const double *f = sm + (size_t)n * n2;
    double cosk[4096];
    for (int k = 0; k < G->nz && k < 4096; k++)
      cosk[k] = 0.3 * cos(3.141592653589793 * k / G->nz + n);
#pragma omp parallel for schedule(static)
    for (int cc = 1; cc <= G->a3_t; cc++) {
      int c = G->w3_t[cc];
      int i = G->s2i[c], j = G->s2j[c], k = G->s2k[c];
      /* approximately normal noise: Irwin-Hall sum of four uniforms */
      unsigned long long hh = mix64(seed ^ mix64(((unsigned long long)n << 40) ^ (unsigned long long)c));
      double nz4 = ((double)(hh & 0xffff) + (double)((hh >> 16) & 0xffff) +
                    (double)((hh >> 32) & 0xffff) + (double)(hh >> 48)) / 65536.0 - 2.0;
      double lg = 1.5 * (f[(size_t)j * g->nx + i] - 0.5) + 0.25 * 1.7320508075688772 * nz4 +
                  cosk[k];
      t[c] = mag * exp(lg);
    }
  }
}
