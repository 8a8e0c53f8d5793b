/*
 * ref_harness.c -- runs the REFERENCE's own tracer-step code (compiled
 * unmodified from model/hd/tracers/tracers.c) on a window described by
 * shoc_tr.h.  TEST INFRASTRUCTURE ONLY: it pins the oracle and provides the
 * CPU baseline; the product never links it.
 *
 * It fills SHOC's geometry_t / window_t / win_priv_t (sparse.h:660-1004,
 * :2393-2790, :246-654) with the caller's arrays and, per step, calls what
 * tracer_step (tracers.c:142) and tracer_step_3d (tracers.c:239) call for a
 * closed passive-tracer window:
 *   set_lateral_BC_tr (tracers.c:5574), set_dz (tracers.c:5682),
 *   advect_diffuse (tracers.c:401), vert_diffuse_3d (tracers.c:3782).
 * Everything else the file references is stubbed below: region budgets,
 * sources/sinks, OBCs, means, debugging and diagnostics have nothing to do
 * in a closed window with passive tracers.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "hd.h"
#if defined(HAVE_OMP)
#include <omp.h>
#endif
#include "shoc_tr.h"

/* ---- globals the reference file expects (globals.h:71-76) ---- */
master_t *master = NULL;
geometry_t *geom = NULL;

/* ---- error trapping: hd_quit_and_dump / exit paths come back here ---- */
static jmp_buf ref_jmp;
static int ref_jmp_armed = 0;
static int ref_err = 0;
static long long ref_nwarn = 0;
static char ref_msg[512];

void hd_quit_and_dump(const char *s, ...) {
  va_list ap;
  va_start(ap, s);
  vsnprintf(ref_msg, sizeof(ref_msg), s, ap);
  va_end(ap);
  ref_err = strstr(s, "zero divisor") ? SHOC_TR_EPIVOT : SHOC_TR_ESUBSTEP;
  if (ref_jmp_armed && ref_err == SHOC_TR_EPIVOT) longjmp(ref_jmp, 1);
}
void hd_quit(const char *s, ...) {
  va_list ap;
  va_start(ap, s);
  vsnprintf(ref_msg, sizeof(ref_msg), s, ap);
  va_end(ap);
  ref_err = SHOC_TR_EUNSUPPORTED;
  if (ref_jmp_armed) longjmp(ref_jmp, 1);
}
void hd_warn(const char *s, ...) {
  if (strncmp(s, "Tracer %s outside range", 23) == 0) {
#if defined(HAVE_OMP)
#pragma omp atomic
#endif
    ref_nwarn++;
  }
}
const char *ref_last_message(void) { return ref_msg; }

/* wall time of the last ref_run's step loop (window set-up excluded) */
static double ref_loop_seconds = 0.0;
double ref_last_loop_seconds(void) { return ref_loop_seconds; }
static double ref_now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ---- allocation (emsalloc.h) ---- */
double *d_alloc_1d(int n1) { return (double *)calloc((size_t)(n1 > 0 ? n1 : 1), sizeof(double)); }
void d_free_1d(double *p) { free(p); }
int *i_alloc_1d(int n1) { return (int *)calloc((size_t)(n1 > 0 ? n1 : 1), sizeof(int)); }
void i_free_1d(int *p) { free(p); }
short *s_alloc_1d(int n1) { return (short *)calloc((size_t)(n1 > 0 ? n1 : 1), sizeof(short)); }
void s_free_1d(short *p) { free(p); }

/* ---- no-ops for a closed window with passive tracers ---- */
double dp_clock() { return 0.0; }
void dp_tracer_step() {}
void advect_diffuse_lag(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void alerts_w(geometry_t *w, int m) { (void)w; (void)m; }
void average_OBC_corner(geometry_t *w, open_bdrys_t *o, double *v, int m) { (void)w; (void)o; (void)v; (void)m; }
double bc_leastsq(double a, double b, double c, double d) { (void)a; (void)b; (void)c; (void)d; return 0.0; }
double bc_polint(double a, double b, double c) { (void)a; (void)b; (void)c; return 0.0; }
double bdry_value_w(geometry_t *w, window_t *d, win_priv_t *c, open_bdrys_t *o,
                    bdry_details_t *b, int x, int y, double t) {
  (void)w; (void)d; (void)c; (void)o; (void)b; (void)x; (void)y; (void)t; return 0.0;
}
void calc_dhd(geometry_t *w, window_t *d, win_priv_t *c, int n) { (void)w; (void)d; (void)c; (void)n; }
void calc_swr(geometry_t *w, window_t *d, win_priv_t *c, double *s, int i) { (void)w; (void)d; (void)c; (void)s; (void)i; }
int check_unstable(geometry_t *w, window_t *d, win_priv_t *c, int m) { (void)w; (void)d; (void)c; (void)m; return 0; }
void debug_c(geometry_t *w, int v, int m) { (void)w; (void)v; (void)m; }
void density_gc(geometry_t *w, window_t *d, win_priv_t *c, int cs, int *map) { (void)w; (void)d; (void)c; (void)cs; (void)map; }
void density_w(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void diag_numbers(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void dump_regions(master_t *m) { (void)m; }
void fill_multidt_aux(master_t *m, geometry_t *w, window_t *d) { (void)m; (void)w; (void)d; }
double get_profile_rms(double *a, double *b, int cs, int *z) { (void)a; (void)b; (void)cs; (void)z; return 0.0; }
void get_tend(geometry_t *w, int *v, int e, double *a, double *b, double *t) { (void)w; (void)v; (void)e; (void)a; (void)b; (void)t; }
void global_interp(geometry_t *g, double *A, int nz) { (void)g; (void)A; (void)nz; }
void mass_diag(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void mld(geometry_t *w, window_t *d, win_priv_t *c, int cs, int cb, double *tm, double *bm, int *css, int *ktb) {
  (void)w; (void)d; (void)c; (void)cs; (void)cb; (void)tm; (void)bm; (void)css; (void)ktb;
}
void mldk(geometry_t *w, window_t *d, win_priv_t *c, int cs, int cb, double *tm, double *bm, int *css, int *ktb) {
  (void)w; (void)d; (void)c; (void)cs; (void)cb; (void)tm; (void)bm; (void)css; (void)ktb;
}
void nor_vert_prof(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
int parseline(char *l, char **s, int m) { (void)l; (void)s; (void)m; return 0; }
void perc_diag(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void prep_semi_lagrange_atc(geometry_t *w) { (void)w; }
void prm_flush_line(FILE *fp) { (void)fp; }
int prm_get_time_in_secs(FILE *fp, char *k, double *v) { (void)fp; (void)k; (void)v; return 0; }
int prm_read_char(FILE *fp, char *k, char *p) { (void)fp; (void)k; (void)p; return 0; }
int prm_read_int(FILE *fp, char *k, int *p) { (void)fp; (void)k; (void)p; return 0; }
int prm_skip_to_end_of_key(FILE *fp, char *k) { (void)fp; (void)k; return 0; }
void read_blocks(FILE *fp, char *k, int *nb, int **li, int **lj) { (void)fp; (void)k; (void)nb; (void)li; (void)lj; }
int read_regioni(master_t *m, char *r, double *id) { (void)m; (void)r; (void)id; return 0; }
void region_flux_coup(geometry_t *w, window_t *d, win_priv_t *c, double *Fx, double *Fy, double *Fz, double dt, int n) {
  (void)w; (void)d; (void)c; (void)Fx; (void)Fy; (void)Fz; (void)dt; (void)n;
}
void region_mass(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void region_volume_flux_coup(geometry_t *w, window_t *d, win_priv_t *c, double dt, double t) {
  (void)w; (void)d; (void)c; (void)dt; (void)t;
}
void reset_means(geometry_t *w, window_t *d, win_priv_t *c, int m) { (void)w; (void)d; (void)c; (void)m; }
void semi_lagrange(geometry_t *w, window_t *d, win_priv_t *c, double *t) { (void)w; (void)d; (void)c; (void)t; }
void semi_lagrange_atc(geometry_t *w, window_t *d, win_priv_t *c, double *t, double *n, int x) {
  (void)w; (void)d; (void)c; (void)t; (void)n; (void)x;
}
void semi_lagrange_c(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
#if !defined(REF_WITH_VEL3D)
void set_flux_3d(geometry_t *w, window_t *d, win_priv_t *c, int m) { (void)w; (void)d; (void)c; (void)m; }
#endif
void set_sbc(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void ss_tracer(geometry_t *w, window_t *d, win_priv_t *c, int n, double *dtr, double dt) {
  (void)w; (void)d; (void)c; (void)n; (void)dtr; (void)dt;
}
void steric(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void streamline_atc(geometry_t *w, window_t *d, win_priv_t *c, int x) { (void)w; (void)d; (void)c; (void)x; }
void surf_relax(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }
void tracer_decay(geometry_t *w, window_t *d, win_priv_t *c, double dec, double *t, tracer_info_t *tr) {
  (void)w; (void)d; (void)c; (void)dec; (void)t; (void)tr;
}
ts_point_t tsflush;
void vorticity(geometry_t *w, window_t *d, win_priv_t *c) { (void)w; (void)d; (void)c; }

/* ---- the harness ---- */
#define DA(n) d_alloc_1d(n)
#define IA(n) i_alloc_1d(n)

typedef struct ref_window {
  geometry_t *win;
  window_t *dat;
  win_priv_t *con;
  int nthreads;
} ref_window;

static void *mutable(const void *p) { return (void *)p; }

static ref_window *ref_make(const shoc_tr_geom *g, shoc_tr_state *st,
                            const shoc_tr_opts *op, int nthreads) {
  ref_window *r = (ref_window *)calloc(1, sizeof(ref_window));
  geometry_t *w = (geometry_t *)calloc(1, sizeof(geometry_t));
  window_t *d = (window_t *)calloc(1, sizeof(window_t));
  win_priv_t *c = (win_priv_t *)calloc(1, sizeof(win_priv_t));
  int S = g->sgsiz, S2 = g->sgsizS, ntr = st->ntr;
  r->win = w; r->dat = d; r->con = c; r->nthreads = nthreads;
  if (!master) master = (master_t *)calloc(1, sizeof(master_t));
#if defined(HAVE_OMP)
  master->trans_num_omp = nthreads;
  /* the tracer loop's work arrays exist for nthreads threads: run that many,
   * as SHOC's driver does (model/hd/control/dp.c:155) */
  omp_set_num_threads(nthreads > 1 ? nthreads : 1);
#endif

  /* geometry_t */
  w->wn = 1;
  w->nz = g->nz;
  w->sgsiz = S; w->sgsizS = S2;
  w->n3_t = g->n3_t; w->a3_t = g->a3_t; w->b3_t = g->b3_t; w->v3_t = g->v3_t;
  w->n2_t = g->n2_t; w->a2_t = g->a2_t; w->b2_t = g->b2_t; w->v2_t = g->v2_t;
  w->w3_t = mutable(g->w3_t); w->w2_t = mutable(g->w2_t); w->bot_t = mutable(g->bot_t);
  w->v3_e1 = g->v3_e1; w->v3_e2 = g->v3_e2;
  w->w3_e1 = mutable(g->w3_e1); w->w3_e2 = mutable(g->w3_e2);
  w->xp1 = mutable(g->xp1); w->xm1 = mutable(g->xm1); w->yp1 = mutable(g->yp1);
  w->ym1 = mutable(g->ym1); w->zp1 = mutable(g->zp1); w->zm1 = mutable(g->zm1);
  w->m2d = mutable(g->m2d);
  w->s2i = mutable(g->s2i); w->s2j = mutable(g->s2j); w->s2k = mutable(g->s2k);
  w->nbpt = g->nbpt; w->bpt = mutable(g->bpt); w->bin = mutable(g->bin);
  w->h1au1 = mutable(g->h1au1); w->h2au2 = mutable(g->h2au2);
  w->h1au2 = mutable(g->h1au2); w->h2au1 = mutable(g->h2au1);
  w->h1acell = mutable(g->h1acell); w->h2acell = mutable(g->h2acell);
  w->cellarea = mutable(g->cellarea); w->botz = mutable(g->botz);
  w->gridz = mutable(g->gridz);
  w->sur_t = st->sur_t; w->nsur_t = st->nsur_t;
  w->nobc = 0; w->naux_t = 0; w->ngsed = 0; w->zoomf = 1;

  /* window_t */
  d->ntr = ntr;
  d->tr_wc = st->tr_wc;
  d->u1 = mutable(st->u1); d->u2 = mutable(st->u2); d->w = mutable(st->w);
  d->u1flux3d = mutable(st->u1flux3d); d->u2flux3d = mutable(st->u2flux3d);
  d->Kz = mutable(st->Kz); d->dzu1 = mutable(st->dzu1); d->dzu2 = mutable(st->dzu2);
  d->eta = mutable(st->eta);
  d->dt = d->dttr = st->dt;
  d->tno = d->sno = -1;

  /* win_priv_t */
  c->trasc = op->trasc; c->ultimate = op->ultimate; c->stab = op->stab;
  c->hmin = op->hmin;
  c->alertf = NONE;
  c->trflux = -1; c->trtend = -1;
  c->ntbdy = op->ntbdy; c->tbdy = mutable(op->tbdy);
  c->ntdif_v = op->ntdif_v; c->tdif_v = mutable(op->tdif_v);
  c->advect = mutable(op->advect); c->diffuse = mutable(op->diffuse);
  c->mintr = mutable(op->mintr); c->maxtr = mutable(op->maxtr);
  c->u1kh = st->u1kh ? mutable(st->u1kh) : DA(S);
  c->u2kh = st->u2kh ? mutable(st->u2kh) : DA(S);
  c->oldeta = mutable(st->oldeta);
  c->sflux = IA(ntr);
  for (int n = 0; n < ntr; n++) c->sflux[n] = -1;
  c->obctr = IA(ntr);
  c->trname = (char **)calloc((size_t)ntr, sizeof(char *));
  for (int n = 0; n < ntr; n++) c->trname[n] = "tracer";
  c->Ds = DA(S2); c->Hn1 = DA(S2); c->Hn2 = DA(S2); c->Hs = DA(S2);
  c->mdx = DA(S2); c->mdy = DA(S2); c->one = DA(S2);
  for (int i = 0; i < S2; i++) c->Ds[i] = c->Hn1[i] = c->Hn2[i] = c->mdx[i] = c->mdy[i] = c->one[i] = 1.0;
  c->dz = DA(S);
  c->w1 = DA(S); c->w2 = DA(S); c->w3 = DA(S); c->w4 = DA(S); c->w5 = DA(S);
  c->w6 = DA(S); c->w7 = DA(S); c->w8 = DA(S); c->w9 = DA(S); c->w10 = DA(S);
  c->d1 = DA(S2); c->d2 = DA(S2); c->d3 = DA(S2); c->d4 = DA(S2);
  c->s1 = IA(S); c->i1 = IA(S2); c->i2 = IA(S2); c->i3 = IA(S2); c->i4 = IA(S2); c->i5 = IA(S2);
  c->v1 = DA(g->nz + 1); c->v2 = DA(g->nz + 1); c->v3 = DA(g->nz + 1); c->v4 = DA(g->nz + 1);
  c->v5 = DA(g->nz + 1); c->v6 = DA(g->nz + 1); c->v7 = DA(g->nz + 1);
  c->tr_mod = DA(S); c->tr_mod_x = DA(S); c->tr_mod_y = DA(S); c->tr_mod_z = DA(S);
  if (nthreads > 1) {
    c->w1n = (double **)calloc((size_t)nthreads, sizeof(double *));
    c->w2n = (double **)calloc((size_t)nthreads, sizeof(double *));
    c->w3n = (double **)calloc((size_t)nthreads, sizeof(double *));
    c->w4n = (double **)calloc((size_t)nthreads, sizeof(double *));
    c->tr_modn = (double **)calloc((size_t)nthreads, sizeof(double *));
    c->tr_modn_x = (double **)calloc((size_t)nthreads, sizeof(double *));
    c->tr_modn_y = (double **)calloc((size_t)nthreads, sizeof(double *));
    c->tr_modn_z = (double **)calloc((size_t)nthreads, sizeof(double *));
    for (int t = 0; t < nthreads; t++) {
      c->w1n[t] = DA(S); c->w2n[t] = DA(S); c->w3n[t] = DA(S); c->w4n[t] = DA(S);
      c->tr_modn[t] = DA(S); c->tr_modn_x[t] = DA(S); c->tr_modn_y[t] = DA(S);
      c->tr_modn_z[t] = DA(S);
    }
  }
  return r;
}

static void ref_free(ref_window *r) {
  win_priv_t *c = r->con;
  free(c->sflux); free(c->obctr); free(c->trname);
  free(c->Ds); free(c->Hn1); free(c->Hn2); free(c->Hs); free(c->mdx); free(c->mdy); free(c->one);
  free(c->dz); free(c->w1); free(c->w2); free(c->w3); free(c->w4); free(c->w5);
  free(c->w6); free(c->w7); free(c->w8); free(c->w9); free(c->w10);
  free(c->d1); free(c->d2); free(c->d3); free(c->d4);
  free(c->s1); free(c->i1); free(c->i2); free(c->i3); free(c->i4); free(c->i5);
  free(c->v1); free(c->v2); free(c->v3); free(c->v4); free(c->v5); free(c->v6); free(c->v7);
  free(c->tr_mod); free(c->tr_mod_x); free(c->tr_mod_y); free(c->tr_mod_z);
  if (r->nthreads > 1) {
    for (int t = 0; t < r->nthreads; t++) {
      free(c->w1n[t]); free(c->w2n[t]); free(c->w3n[t]); free(c->w4n[t]);
      free(c->tr_modn[t]); free(c->tr_modn_x[t]); free(c->tr_modn_y[t]); free(c->tr_modn_z[t]);
    }
    free(c->w1n); free(c->w2n); free(c->w3n); free(c->w4n);
    free(c->tr_modn); free(c->tr_modn_x); free(c->tr_modn_y); free(c->tr_modn_z);
  }
  free(r->win); free(r->dat); free(r->con); free(r);
}

/* Reference functions (declared in the reference's proto.h). */
void set_lateral_BC_tr(double **tr, int ntr, int sgbpt, int *bpt, int *bin);
void set_dz(geometry_t *window, window_t *windat, win_priv_t *wincon);
int advect_diffuse(geometry_t *window, window_t *windat, win_priv_t *wincon);
void vert_diffuse_3d(geometry_t *window, window_t *windat, win_priv_t *wincon);

/* Runs nsteps reference tracer steps.  nthreads > 1 uses the reference's
 * own OpenMP tracer loop (build with -fopenmp -DHAVE_OMP). */
int ref_run(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op,
            int nsteps, int nthreads, shoc_tr_diag *diag) {
  ref_window *r = ref_make(g, st, op, nthreads);
  geometry_t *w = r->win;
  window_t *d = r->dat;
  win_priv_t *c = r->con;
  int rc = SHOC_TR_OK;
  ref_err = 0;
  ref_nwarn = 0;
  ref_msg[0] = 0;
  if (setjmp(ref_jmp)) {
    ref_jmp_armed = 0;
    rc = ref_err ? ref_err : SHOC_TR_EUNSUPPORTED;
    if (diag) diag->nwarn = ref_nwarn;
    ref_free(r);
    return rc;
  }
  ref_jmp_armed = 1;
  const double t0 = ref_now();
  for (int s = 0; s < nsteps; s++) {
    set_lateral_BC_tr(d->tr_wc, d->ntr, w->nbpt, w->bpt, w->bin);
    set_dz(w, d, c);
    if (advect_diffuse(w, d, c)) {
      rc = ref_err ? ref_err : SHOC_TR_ESUBSTEP;
      break;
    }
    vert_diffuse_3d(w, d, c);
    d->nstep++;
    d->t += d->dt;
  }
  ref_loop_seconds = ref_now() - t0;
  ref_jmp_armed = 0;
  if (diag) {
    diag->nwarn = ref_nwarn;
    diag->vc = c->vc;
    diag->vcs = c->vcs;
    diag->dtm = c->b1;
    diag->nsub = 0;
  }
  ref_free(r);
  return rc;
}

/* ---- the other per-column tridiagonal solves ---- */
void tridiagonal(geometry_t *window, int cs, int cb, double *C, double *Cm1, double *Cp1,
                 double *rhs, double *var, double minvar);
void implicit_vdiff_at_cc(geometry_t *window, window_t *windat, win_priv_t *wincon, double *var,
                          double *Kz, double *dzcell, double *dzface, double *fb, double *ft,
                          int *ctp, int *cbt, int cc, double *Splus, double *Sminus,
                          double *scale, double *C, double *Cp1, double *Cm1, double dt);

/* The reference's closure solve (tridiagonal, model/hd/closure/MY2-5.c:499)
 * on every water column of the window: from the bottom cell bot_t[cc] to the
 * surface cell st->nsur_t[cc] (a column whose surface is its sediment cell
 * is dry and left out).  C, Cm1, Cp1 and rhs are [sgsiz] arrays by cell (the
 * row of the cell's layer); the reference takes them by layer, so each
 * column's rows are gathered into layer arrays first.  var [sgsiz]. */
int ref_tridiag(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op,
                const double *C, const double *Cm1, const double *Cp1, const double *rhs,
                double *var, double minvar) {
  ref_window *r = ref_make(g, st, op, 1);
  geometry_t *w = r->win;
  win_priv_t *c = r->con;
  const int nz = g->nz;
  w->wincon = c;
  c->v11 = DA(nz + 1);
  c->v12 = DA(nz + 1);
  double *lC = DA(nz + 1), *lCm1 = DA(nz + 1), *lCp1 = DA(nz + 1), *lr = DA(nz + 1);
  int rc = SHOC_TR_OK;
  ref_err = 0;
  if (setjmp(ref_jmp)) {
    rc = ref_err ? ref_err : SHOC_TR_EUNSUPPORTED;
  } else {
    ref_jmp_armed = 1;
    for (int cc = 1; cc <= g->b2_t; cc++) {
      const int cs = st->nsur_t[cc], cb = g->bot_t[cc];
      if (cs == g->zm1[cs]) continue;
      for (int cl = cb, k = g->s2k[cb];; cl = g->zp1[cl], k++) {
        lC[k] = C[cl]; lCm1[k] = Cm1[cl]; lCp1[k] = Cp1[cl]; lr[k] = rhs[cl];
        if (cl == cs) break;
      }
      tridiagonal(w, cs, cb, lC, lCm1, lCp1, lr, var, minvar);
    }
  }
  ref_jmp_armed = 0;
  free(lC); free(lCm1); free(lCp1); free(lr);
  free(c->v11); free(c->v12);
  ref_free(r);
  return rc;
}

/* The reference's single-column implicit diffusion (implicit_vdiff_at_cc,
 * model/hd/tracers/tracers.c:7407) on every water column: var [sgsiz] by
 * cell is gathered into the layer vector the reference works on (as its
 * caller swr_assimilation does, tracers.c:4030-4045), diffused with the
 * coefficients C, Cm1, Cp1 and thicknesses dzcell [sgsiz], the bottom and
 * top fluxes fb, ft and the scale [sgsizS], the sources Splus, Sminus
 * [sgsiz] (or NULL), and scattered back.  No thin layers: i4 = the surface. */
int ref_vdiff_cols(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op,
                   double *var, const double *dzcell, const double *C, const double *Cm1,
                   const double *Cp1, const double *fb, const double *ft, const double *Splus,
                   const double *Sminus, const double *scale, double dt) {
  ref_window *r = ref_make(g, st, op, 1);
  geometry_t *w = r->win;
  window_t *d = r->dat;
  win_priv_t *c = r->con;
  const int nz = g->nz;
  w->wincon = c;
  int *ctp = IA(g->b2_t + 1), *cbt = IA(g->b2_t + 1);
  double *temp = DA(nz + 1);
  int n = 0;
  for (int cc = 1; cc <= g->b2_t; cc++) {
    const int cs = st->nsur_t[cc];
    if (cs == g->zm1[cs]) continue;
    n++;
    ctp[n] = cs;
    cbt[n] = g->bot_t[cc];
    c->i4[n] = cs;
  }
  int rc = SHOC_TR_OK;
  ref_err = 0;
  if (setjmp(ref_jmp)) {
    rc = ref_err ? ref_err : SHOC_TR_EUNSUPPORTED;
  } else {
    ref_jmp_armed = 1;
    for (int cc = 1; cc <= n; cc++) {
      const int cs = ctp[cc], cb = cbt[cc];
      for (int cl = cs, k = g->s2k[cs];; cl = g->zm1[cl], k--) {
        temp[k] = var[cl];
        if (cl == cb) break;
      }
      implicit_vdiff_at_cc(w, d, c, temp, NULL, mutable(dzcell), NULL, mutable(fb),
                           mutable(ft), ctp, cbt, cc, mutable(Splus), mutable(Sminus),
                           mutable(scale), mutable(C), mutable(Cp1), mutable(Cm1), dt);
      for (int cl = cs, k = g->s2k[cs];; cl = g->zm1[cl], k--) {
        var[cl] = temp[k];
        if (cl == cb) break;
      }
    }
  }
  ref_jmp_armed = 0;
  free(ctp); free(cbt); free(temp);
  ref_free(r);
  return rc;
}

/* ---- the window structs for other checkers (the shim check) ---- */
void *ref_window_new(const shoc_tr_geom *g, shoc_tr_state *st, const shoc_tr_opts *op) {
  return ref_make(g, st, op, 1);
}
geometry_t *ref_window_geom(void *r) { return ((ref_window *)r)->win; }
window_t *ref_window_data(void *r) { return ((ref_window *)r)->dat; }
win_priv_t *ref_window_con(void *r) { return ((ref_window *)r)->con; }
void ref_window_delete(void *r) { ref_free((ref_window *)r); }
