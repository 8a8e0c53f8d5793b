/*
 * ref_preamble.c -- runs the REFERENCE's transport-mode preamble (what
 * transport_step does before the tracer step, model/hd/tracers/
 * transport.c:436-462): set_dz_at_u1 / set_dz_at_u2 (model/hd/momentum/
 * vel3d.c:720), set_flux_3d (vel3d.c:4041, VEL3D), set_dz (tracers.c:5682)
 * and vel_w_update (vel3d.c:4609, the CONS_W branch), compiled unmodified,
 * on a window described by shoc_tr.h.  TEST INFRASTRUCTURE ONLY.
 *
 * The e1 / e2 face columns the reference keeps in geometry_t (w2_e1, bot_e1,
 * botzu1) are built from the window's w3_e1 / w3_e2 the way SHOC's
 * preprocessor lists them: one per surface-layer cell of w3_e1, its bottom
 * cell the deepest cell of the run of w3_e1 cells below it, and botzu1 the
 * higher of the two floors (hd_init.c:1443).  Linear free surface, no
 * sources: wtop = detadt, wbot = 0.
 */
#include <stdlib.h>
#include <string.h>
#include "hd.h"
#include "shoc_tr.h"

void *ref_window_new(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op);
geometry_t *ref_window_geom(void *r);
window_t *ref_window_data(void *r);
win_priv_t *ref_window_con(void *r);
void ref_window_delete(void *r);
void set_dz_at_u1(geometry_t *window, window_t *windat, win_priv_t *wincon);
void set_dz_at_u2(geometry_t *window, window_t *windat, win_priv_t *wincon);
void set_flux_3d(geometry_t *window, window_t *windat, win_priv_t *wincon, int mode);
void set_dz(geometry_t *window, window_t *windat, win_priv_t *wincon);
void vel_w_update(geometry_t *window, window_t *windat, win_priv_t *wincon);

/* face columns of one direction: w3 / ne = the window's w3_e1 (w3_e2), bm =
 * the backward map (xm1 or ym1), e3 = membership flags of w3.  A face column
 * starts at each surface-layer cell of w3 (SHOC's w2_e1), its bottom cell is
 * the deepest cell of the run of w3 cells below it (bot_e1) and its floor the
 * higher of the two sides' (botzu1). */
static int faces(const shoc_tr_geom *g, int ne, const int *w3, const int *bm, const char *e3,
                 int **w2, int **bot, double **botzu) {
  const int S2 = g->sgsizS;
  int n = 0;
  *w2 = (int *)calloc((size_t)ne + 1, sizeof(int));
  *bot = (int *)calloc((size_t)ne + 1, sizeof(int));
  *botzu = (double *)calloc((size_t)S2, sizeof(double));
  for (int i = 1; i <= ne; i++) {
    const int c2 = w3[i];
    if (g->zp1[c2] != c2) continue;
    int c = c2, cb = c2;
    while (g->zm1[c] != c && e3[c]) {
      cb = c;
      c = g->zm1[c];
    }
    n++;
    (*w2)[n] = c2;
    (*bot)[n] = cb;
    const double a = g->botz[bm[c2]], b = g->botz[c2];
    (*botzu)[c2] = a > b ? a : b;
  }
  return n;
}

int ref_preamble(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op,
                 const double *detadt, double *dzu1, double *dzu2, double *u1flux3d,
                 double *u2flux3d, double *wv) {
  void *r = ref_window_new(g, st, op);
  geometry_t *w = ref_window_geom(r);
  window_t *d = ref_window_data(r);
  win_priv_t *c = ref_window_con(r);
  const int S = g->sgsiz, S2 = g->sgsizS;
  char *e1 = (char *)calloc((size_t)S, 1), *e2 = (char *)calloc((size_t)S, 1);
  for (int i = 1; i <= g->v3_e1; i++) e1[g->w3_e1[i]] = 1;
  for (int i = 1; i <= g->v3_e2; i++) e2[g->w3_e2[i]] = 1;
  w->b2_e1 = faces(g, g->v3_e1, g->w3_e1, g->xm1, e1, &w->w2_e1, &w->bot_e1, &w->botzu1);
  w->b2_e2 = faces(g, g->v3_e2, g->w3_e2, g->ym1, e2, &w->w2_e2, &w->bot_e2, &w->botzu2);
  w->sur_e1 = (int *)calloc((size_t)w->b2_e1 + 1, sizeof(int));
  w->sur_e2 = (int *)calloc((size_t)w->b2_e2 + 1, sizeof(int));
  w->b3_e1 = g->v3_e1;
  w->b3_e2 = g->v3_e2;
  d->sur_e1 = (int *)calloc((size_t)S2, sizeof(int));
  d->sur_e2 = (int *)calloc((size_t)S2, sizeof(int));
  d->dzu1 = dzu1;
  d->dzu2 = dzu2;
  d->u1flux3d = u1flux3d;
  d->u2flux3d = u2flux3d;
  d->w = wv;
  d->wtop = (double *)calloc((size_t)S2, sizeof(double));
  d->wbot = (double *)calloc((size_t)S2, sizeof(double));
  d->detadt = (double *)detadt;
  d->waterss = (double *)calloc((size_t)S, sizeof(double));
  c->d5 = (double *)calloc((size_t)S2, sizeof(double));  /* maxeta at e1 faces */
  c->d6 = (double *)calloc((size_t)S2, sizeof(double));  /* maxeta at e2 faces */
  c->cdry_e1 = (int *)calloc((size_t)S2, sizeof(int));
  c->cdry_e2 = (int *)calloc((size_t)S2, sizeof(int));
  c->cbot_e1 = (int *)calloc((size_t)S2, sizeof(int));
  c->cbot_e2 = (int *)calloc((size_t)S2, sizeof(int));
  c->ncbot_e1 = c->ncbot_e2 = 0;  /* built by the momentum step only */
  c->etarlx = NONE;
  c->means = 0;
  c->nonlinear = 0;
  c->momsc = 0;
  c->sigma = 0;
  c->conserve = CONS_W;
  w->wincon = c;

  set_dz_at_u1(w, d, c);
  set_dz_at_u2(w, d, c);
  set_flux_3d(w, d, c, VEL3D);
  set_dz(w, d, c);
  vel_w_update(w, d, c);

  free(e1); free(e2);
  free(w->w2_e1); free(w->bot_e1); free(w->botzu1);
  free(w->w2_e2); free(w->bot_e2); free(w->botzu2);
  free(w->sur_e1); free(w->sur_e2); free(d->sur_e1); free(d->sur_e2);
  free(d->wtop); free(d->wbot); free(d->waterss);
  free(c->d5); free(c->d6); free(c->cdry_e1); free(c->cdry_e2); free(c->cbot_e1); free(c->cbot_e2);
  ref_window_delete(r);
  return 0;
}
