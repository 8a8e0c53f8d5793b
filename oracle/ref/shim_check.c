/*
 * shim_check.c -- compiles include/shoc_tr_shim.h (the SHOC-side binding of
 * the library) against the reference's own headers (model/hd/include/
 * sparse.h through hd.h, with the stub headers of oracle/ref/stub), as a
 * SHOC build with HAVE_B200_TRACERS would.  TEST INFRASTRUCTURE ONLY.
 *
 *   shim_fields  the shim's window description of a window built by the
 *                harness equals the description the window was built from,
 *                field by field (returns the number of fields that differ)
 *   shim_step    nsteps tracer steps through b200_tracer_step, the call
 *                tracer_step_3d makes in a HAVE_B200_TRACERS build
 */
#include <string.h>
#include "hd.h"
#include "shoc_tr_shim.h"

void *ref_window_new(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op);
geometry_t *ref_window_geom(void *r);
window_t *ref_window_data(void *r);
win_priv_t *ref_window_con(void *r);
void ref_window_delete(void *r);

#define SAME(a, b) (n += ((a) != (b)))

int shim_fields(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op) {
  void *r = ref_window_new(g, st, op);
  geometry_t *w = ref_window_geom(r);
  window_t *d = ref_window_data(r);
  win_priv_t *c = ref_window_con(r);
  shoc_tr_geom g2;
  shoc_tr_opts o2;
  shoc_tr_state s2;
  memset(&g2, 0, sizeof(g2));
  memset(&o2, 0, sizeof(o2));
  memset(&s2, 0, sizeof(s2));
  b200_geom(w, &g2);
  b200_opts(c, &o2);
  b200_state(w, d, c, &s2);
  int n = 0;
  SAME(g2.nz, g->nz); SAME(g2.sgsiz, g->sgsiz); SAME(g2.sgsizS, g->sgsizS);
  SAME(g2.n3_t, g->n3_t); SAME(g2.a3_t, g->a3_t); SAME(g2.b3_t, g->b3_t);
  SAME(g2.v3_t, g->v3_t); SAME(g2.w3_t, g->w3_t);
  SAME(g2.n2_t, g->n2_t); SAME(g2.a2_t, g->a2_t); SAME(g2.b2_t, g->b2_t);
  SAME(g2.v2_t, g->v2_t); SAME(g2.w2_t, g->w2_t); SAME(g2.bot_t, g->bot_t);
  SAME(g2.v3_e1, g->v3_e1); SAME(g2.v3_e2, g->v3_e2); SAME(g2.w3_e1, g->w3_e1);
  SAME(g2.w3_e2, g->w3_e2); SAME(g2.xp1, g->xp1); SAME(g2.xm1, g->xm1);
  SAME(g2.yp1, g->yp1); SAME(g2.ym1, g->ym1); SAME(g2.zp1, g->zp1); SAME(g2.zm1, g->zm1);
  SAME(g2.m2d, g->m2d); SAME(g2.s2i, g->s2i); SAME(g2.s2j, g->s2j); SAME(g2.s2k, g->s2k);
  SAME(g2.nbpt, g->nbpt); SAME(g2.bpt, g->bpt); SAME(g2.bin, g->bin);
  SAME(g2.h1au1, g->h1au1); SAME(g2.h2au2, g->h2au2); SAME(g2.h1au2, g->h1au2);
  SAME(g2.h2au1, g->h2au1); SAME(g2.h1acell, g->h1acell); SAME(g2.h2acell, g->h2acell);
  SAME(g2.cellarea, g->cellarea); SAME(g2.botz, g->botz); SAME(g2.gridz, g->gridz);
  SAME(o2.trasc, op->trasc); SAME(o2.ultimate, op->ultimate); SAME(o2.stab, op->stab);
  SAME(o2.hmin, op->hmin); SAME(o2.ntbdy, op->ntbdy); SAME(o2.ntdif_v, op->ntdif_v);
  SAME(o2.advect, op->advect); SAME(o2.diffuse, op->diffuse);
  SAME(o2.mintr, op->mintr); SAME(o2.maxtr, op->maxtr);
  for (int i = 0; i < op->ntbdy; i++) SAME(o2.tbdy[i], op->tbdy[i]);
  for (int i = 0; i < op->ntdif_v; i++) SAME(o2.tdif_v[i], op->tdif_v[i]);
  SAME(s2.ntr, st->ntr); SAME(s2.tr_wc, st->tr_wc); SAME(s2.sur_t, st->sur_t);
  SAME(s2.nsur_t, st->nsur_t); SAME(s2.u1, st->u1); SAME(s2.u2, st->u2); SAME(s2.w, st->w);
  SAME(s2.u1flux3d, st->u1flux3d); SAME(s2.u2flux3d, st->u2flux3d); SAME(s2.Kz, st->Kz);
  SAME(s2.dzu1, st->dzu1); SAME(s2.dzu2, st->dzu2); SAME(s2.eta, st->eta);
  SAME(s2.oldeta, st->oldeta); SAME(s2.dt, st->dt);
  if (st->u1kh) SAME(s2.u1kh, st->u1kh);
  if (st->u2kh) SAME(s2.u2kh, st->u2kh);
  ref_window_delete(r);
  return n;
}

int shim_step(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op, int nsteps) {
  void *r = ref_window_new(g, st, op);
  geometry_t *w = ref_window_geom(r);
  window_t *d = ref_window_data(r);
  win_priv_t *c = ref_window_con(r);
  int rc = 0;
  for (int s = 0; s < nsteps && !rc; s++) rc = b200_tracer_step(w, d, c);
  b200_release(w);
  ref_window_delete(r);
  return rc;
}
