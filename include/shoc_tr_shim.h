/*
 * shoc_tr_shim.h -- the SHOC-side binding of the B200 tracer step.
 *
 * SHOC is C, so the "binding" of this library is this header, included by
 * model/hd/tracers/tracers.c under a build flag after SHOC's own headers
 * (hd.h: geometry_t, window_t and win_priv_t of model/hd/include/sparse.h).
 * It fills the library's window description (shoc_tr.h) from SHOC's window
 * structs with pointer assignments, keeps one handle per window, and maps the
 * library's status codes onto SHOC's failure paths:
 *
 *   #ifdef HAVE_B200_TRACERS
 *   #include "shoc_tr_shim.h"
 *   #endif
 *   ...
 *   in tracer_step_3d (tracers.c:258-280), instead of advect_diffuse and
 *   vert_diffuse_3d:   if (b200_tracer_step(window, windat, wincon)) return;
 *
 * (set_dz is then skipped in transport_step, model/hd/tracers/transport.c:457:
 * the step computes it on the device.)  Link with -lshoc_tr_gpu.
 */
#ifndef SHOC_TR_SHIM_H
#define SHOC_TR_SHIM_H

#include "shoc_tr_gpu.h"

#ifndef B200_MAX_WINDOWS
#define B200_MAX_WINDOWS 64
#endif
#ifndef B200_PRECISION
#define B200_PRECISION SHOC_TR_FP64
#endif

/* one handle per window, created on first use (dp worker threads each own
 * their window, model/hd/control/dp.c:351-359); index = window->wn */
static shoc_tr_gpu *b200[B200_MAX_WINDOWS];

static void b200_geom(geometry_t *w, shoc_tr_geom *g) {
  g->nz = w->nz; g->sgsiz = w->sgsiz; g->sgsizS = w->sgsizS;
  g->n3_t = w->n3_t; g->a3_t = w->a3_t; g->b3_t = w->b3_t; g->v3_t = w->v3_t;
  g->w3_t = w->w3_t;
  g->n2_t = w->n2_t; g->a2_t = w->a2_t; g->b2_t = w->b2_t; g->v2_t = w->v2_t;
  g->w2_t = w->w2_t; g->bot_t = w->bot_t;
  g->v3_e1 = w->v3_e1; g->v3_e2 = w->v3_e2; g->w3_e1 = w->w3_e1; g->w3_e2 = w->w3_e2;
  g->xp1 = w->xp1; g->xm1 = w->xm1; g->yp1 = w->yp1; g->ym1 = w->ym1;
  g->zp1 = w->zp1; g->zm1 = w->zm1; g->m2d = w->m2d;
  g->s2i = w->s2i; g->s2j = w->s2j; g->s2k = w->s2k;
  g->nbpt = w->nbpt; g->bpt = w->bpt; g->bin = w->bin;
  g->h1au1 = w->h1au1; g->h2au2 = w->h2au2; g->h1au2 = w->h1au2; g->h2au1 = w->h2au1;
  g->h1acell = w->h1acell; g->h2acell = w->h2acell; g->cellarea = w->cellarea;
  g->botz = w->botz; g->gridz = w->gridz;
}

static void b200_opts(win_priv_t *c, shoc_tr_opts *o) {
  o->trasc = c->trasc; o->ultimate = c->ultimate; o->stab = c->stab; o->hmin = c->hmin;
  o->ntbdy = c->ntbdy; o->tbdy = c->tbdy; o->ntdif_v = c->ntdif_v; o->tdif_v = c->tdif_v;
  o->advect = c->advect; o->diffuse = c->diffuse; o->mintr = c->mintr; o->maxtr = c->maxtr;
  o->ntr2d = 0;
}

static void b200_state(geometry_t *w, window_t *d, win_priv_t *c, shoc_tr_state *st) {
  st->ntr = d->ntr; st->tr_wc = d->tr_wc; st->sur_t = w->sur_t; st->nsur_t = w->nsur_t;
  st->u1 = d->u1; st->u2 = d->u2; st->w = d->w;
  st->u1flux3d = d->u1flux3d; st->u2flux3d = d->u2flux3d; st->Kz = d->Kz;
  st->dzu1 = d->dzu1; st->dzu2 = d->dzu2; st->u1kh = c->u1kh; st->u2kh = c->u2kh;
  st->eta = d->eta; st->oldeta = c->oldeta; st->dt = d->dt;
}

/* replaces set_dz + advect_diffuse + vert_diffuse_3d in tracer_step_3d;
 * returns 1 where the reference's advect_diffuse would (after quitting) */
static int b200_tracer_step(geometry_t *w, window_t *d, win_priv_t *c) {
  shoc_tr_state st;
  shoc_tr_diag diag;
  if (w->wn < 0 || w->wn >= B200_MAX_WINDOWS) {
    hd_quit("b200: window %d beyond B200_MAX_WINDOWS (%d)\n", w->wn, B200_MAX_WINDOWS);
    return 1;
  }
  if (!b200[w->wn]) {
    shoc_tr_geom g;
    shoc_tr_opts o;
    b200_geom(w, &g);
    b200_opts(c, &o);
    if (shoc_tr_gpu_create(&g, &o, d->ntr, B200_PRECISION, 0, &b200[w->wn])) {
      hd_quit("b200: window %d not supported\n", w->wn);
      return 1;
    }
  }
  b200_state(w, d, c, &st);
  int rc = shoc_tr_gpu_step(b200[w->wn], &st, &diag);
  if (rc == SHOC_TR_ESUBSTEP)
    hd_quit_and_dump("tracer_step_3d: maximum number of sub-steps (%d) exceeded\n", 20);
  else if (rc == SHOC_TR_EPIVOT)
    hd_quit_and_dump("Tracer diffusion;implicit_vdiff_tr: zero divisor\n");
  else if (rc)
    hd_quit("b200 tracer step: %s\n", shoc_tr_gpu_strerror(rc));
  return rc ? 1 : 0;
}

/* at the end of the run, per window */
static void b200_release(geometry_t *w) {
  if (w->wn >= 0 && w->wn < B200_MAX_WINDOWS && b200[w->wn]) {
    shoc_tr_gpu_destroy(b200[w->wn]);
    b200[w->wn] = 0;
  }
}

#endif
