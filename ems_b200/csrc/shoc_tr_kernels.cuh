// shoc_tr_kernels.cuh -- sm_100a kernels of the SHOC tracer step.
//
// Device layout: tracers and per-cell fields stay in SHOC's sparse layout
// (index = SHOC sparse coordinate), so 32 adjacent wet columns at one layer
// are 32 consecutive cells and a warp's loads coalesce; host<->device copies
// are plain memcpys.  One thread owns one (column, tracer) pair and walks its
// column bottom to top: horizontal and vertical face values, the ULTIMATE
// limiter, the flux divergence, the interior update, surf_conc and tr_bounds,
// and on the last sub-step the Thomas forward sweep; then it back-substitutes
// top to bottom.  The tridiagonal LU factors do not depend on the tracer and
// are built once per step per column.
//
// FP64 arithmetic follows model/hd/tracers/tracers.c operation by operation
// (compiled with --fmad=false, IEEE division): results are bitwise equal to
// the reference's on the same inputs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "shoc_tr.h"

namespace shoc {

constexpr double kSF = 0.8;        // tracers.c:427
constexpr double kMinVal = 1e-10;  // tracers.c:428
constexpr double kClipEps = 1e-5;  // tracers.c:3230

// per-cell flags (cflag)
constexpr uint8_t CF_WET = 1;   // in w3_t[1..a3_t]
constexpr uint8_t CF_E1 = 2;    // in w3_e1[1..v3_e1]
constexpr uint8_t CF_E2 = 4;    // in w3_e2[1..v3_e2]

// status bits (OR-ed on the device, mapped to SHOC_TR_* on the host)
constexpr int ST_PIVOT = 1;
constexpr int ST_NAN = 2;
constexpr int ST_LASTDRY = 4;  // column v2_t not processed: reference keeps a stale vcs1
constexpr int ST_SCRATCH = 8;
constexpr int ST_GEOM = 16;    // a column walk left its column (inconsistent maps / state)

// per-column flags
constexpr int COL_WET = 1;      // in the cells-to-process list s1
constexpr int COL_SINGLE = 2;   // one-layer column in vert_diffuse_3d
constexpr int COL_SERIAL = 4;   // tr_bounds thin fix can couple tracers: serial path
constexpr int COL_THIN = 8;     // tr_bounds thin-surface test is on
constexpr int COL_NOSOLVE = 16; // degenerate implicit-solve range: status raised, no solve
constexpr int COL_STAGED = 32;  // handled by the FP32-mixed column-tile kernels

// ---------------------------------------------------------------------------
// 16-bit compensation of an FP32-stored value (the SHOC_TR_FP32_COMP
// precision).  A value v stored as v32 = (float)v (round to nearest, so
// |v - v32| <= ulp(v32) / 2) keeps beside it the residual r = v - v32 as a
// bfloat16 (the upper half of r's FP32 bits: 8 significant bits, rounded
// toward zero, as is r's own conversion to FP32); v32 + r gives v back to
// about 2^-32 of its size, and reading
// it back is one shift.  Without it a value whose change per step is below
// half an FP32 ulp is rounded back to the same FP32 number every step.
// Rounding r toward zero keeps the decoded value inside v32's rounding
// interval (at most half an ulp away, a tie only where v itself was one and
// v32 is the even neighbour): converting it to FP32 gives v32 back and
// encoding again gives the same bits, so the drop-in step's trip through
// FP64 host arrays changes nothing.
__device__ __forceinline__ float lo_val(int16_t q) {
  return __uint_as_float((uint32_t)(uint16_t)q << 16);
}
__device__ __forceinline__ int16_t lo_bits(float r) {
  return isfinite(r) ? (int16_t)(__float_as_uint(r) >> 16) : (int16_t)0;
}
__device__ __forceinline__ int16_t lo_enc(double v, float v32) {
  return lo_bits(__double2float_rz(v - (double)v32));
}
// lo_enc, and what the returned compensation decodes to in dec
__device__ __forceinline__ int16_t lo_round(double v, float v32, double &dec) {
  const int16_t q = lo_enc(v, v32);
  dec = (double)lo_val(q);
  return q;
}
__device__ __forceinline__ double lo_dec(int16_t q, float) { return (double)lo_val(q); }

// 2D face metrics of one direction, precomputed per surface-layer cell:
// d = d3/d4 weight, db/df = 2/(h_m+h_0), 2/(h_0+h_p), h_m/h_0/h_p = metric
// at the backward neighbour / the cell / the forward neighbour.
struct Face2D {
  double d, db, df, hm, h0, hp;
};

struct ColInfo {
  int s;       // advection surface cell: the lower of old and new surface
  int co;      // old surface cell (wincon->i3)
  int cs;      // new surface cell: top of the implicit solve (wincon->i2)
  int cbs;     // bottom of the implicit solve (cbt)
  int flags;
  int ks;      // layer of s
};

struct Geo {
  int S, S2, nz, ncol, v2col;  // v2col: 0-based index of column v2_t
  const int *xp1, *xm1, *yp1, *ym1, *zp1, *zm1, *m2d;
  const uint8_t *cflag;
  const int *col_top, *col_bot;  // surface-layer and bottom cell per column
  const int *col_kb;             // layer index of the bottom cell per column
  const int *kof;                // layer index of every cell (s2k)
  const int *colntr;             // tracers updated per column (numbers below it)
  const double *h1au1, *h2au2, *h1au2, *h2au1, *h1acell, *h2acell, *cellarea, *botz;
  const double *gridz;
  const Face2D *fx, *fy;         // [S2]
};

struct Flow {
  const double *u1, *u2, *w, *u1flux3d, *u2flux3d, *Kz;
  const double *dzu1, *dzu2, *u1kh, *u2kh;
  const double *eta, *oldeta;
  double dt;
};

struct Work {
  double *dz, *w5, *w9, *dbz, *dfz;     // per step
  double *w6, *w7, *w8;                 // per sub-step
  double *vd_cm1, *vd_div, *vd_ud, *vd_dzdt;
  int *sur_t, *nsur_t;                  // [ncol] 0-based column
  ColInfo *col;                         // [ncol]
  int *status;
  unsigned long long *dtm_bits;
  unsigned long long *nwarn;
  int *serial_list, *serial_count;
  // FP32-mixed path: layer thickness and LU factors {dzdt, cm1, 1/div, ud}
  float *dz32;
  float4 *lu32;
};

// FP32 copies of the flow fields (FP32-mixed path), made by set_flow.
struct Flow32 {
  const double *u1_64, *u2_64;  // the FP64 velocities (FP32_COMP face set-up)
  const float *u1, *u2, *w;  // FP32 copies for the Courant numbers
  const double *u1flux3d, *u2flux3d, *w64;  // the FP64 arrays of Flow: volume fluxes
  const float *khx, *khy;  // dzu1 h2au1 u1kh / h1au1 and the e2 analogue
};

struct Opt {
  int trasc, ultimate, substep;
  double hmin;
  int tiled;  // the scheme has tile kernels (QUICKEST, Van Leer); else every
              // column takes the general path
};

// Per-tracer attributes (device arrays indexed by tracer number).
struct TrSet {
  int ntr;              // tracers in the handle
  int nslot;            // tracers this launch processes
  int ntb;              // of which advected / diffused (tbdy), the first ntb slots
  const int *slot_tr;   // slot -> tracer number, tbdy order then the rest
  const uint8_t *trf;   // TR_* flags per tracer
  const double *mintr, *maxtr;
};
constexpr uint8_t TR_TBDY = 1, TR_ADV = 2, TR_HDIFF = 4, TR_VDIFF = 8;

struct SubStep {
  double dtu, trem;          // this sub-step (tracers.c:717-720)
  double subeta_f;           // 1 + (dtu - trem)/dt, for subeta (:753-754)
  double osub_f;             // same factor of the previous sub-step
  int first;                 // osubeta = oldeta on the first sub-step
};

// ---------------------------------------------------------------------------
// face values

// QUICKEST on a non-uniform grid (quickest, tracers.c:1870-1884): tm2..tp1 are
// the tracer at i-2, i-1, i, i+1 of the face's cell, cr the Courant number.
__device__ __forceinline__ double quickest_face(double cr, const Face2D &m, double tm2,
                                                double tm1, double t0, double tp1) {
  double face = m.d * (t0 - tm1) + tm1;
  double grad = t0 - tm1;
  double curv = 0.0;
  if (cr > 0.0)
    curv = m.db * (m.hm * t0 + m.h0 * tm2) - 2.0 * tm1;
  else if (cr < 0.0)
    curv = m.df * (m.h0 * tp1 + m.hp * tm1) - 2.0 * t0;
  return face - 0.5 * cr * grad - (1.0 - cr * cr) * curv / 6.0;
}

// Vertical QUICKEST (tracers.c:1911-1927) with w5 and the w9 factors.
__device__ __forceinline__ double quickest_zface(double cz, double w5, double db, double df,
                                                 double w9m, double w90, double w9p,
                                                 double tm2, double tm1, double t0,
                                                 double tp1) {
  double face = w5 * (t0 - tm1) + tm1;
  double grad = t0 - tm1;
  double curv = 0.0;
  if (cz > 0.0)
    curv = db * (w9m * t0 + w90 * tm2) - 2.0 * tm1;
  else if (cz < 0.0)
    curv = df * (w90 * tp1 + w9p * tm1) - 2.0 * t0;
  return face - 0.5 * cz * grad - (1.0 - cz * cz) * curv / 6.0;
}

// Van Leer (van_leer_do, tracers.c:2102-2117); F unchanged (0) when vel == 0.
__device__ __forceinline__ double vanleer_face(double vel, double cn, double tm2, double tm1,
                                               double t0, double tp1) {
  double df;
  if (vel > 0.0) {
    df = (tm1 - tm2) * (t0 - tm1);
    if (df > 0.0)
      df = 2.0 * df / (t0 - tm2);
    else
      df = 0.0;
    return tm1 + 0.5 * (1.0 - cn) * df;
  } else if (vel < 0.0) {
    df = (t0 - tm1) * (tp1 - t0);
    if (df > 0.0)
      df = 2.0 * df / (tp1 - tm1);
    else
      df = 0.0;
    return t0 - 0.5 * (1.0 + cn) * df;
  }
  return 0.0;
}

// ULTIMATE limiter on one face (ulimate_filter, tracers.c:3526-3554).
__device__ __forceinline__ double ultimate_face(double cr, double F, double tm2, double tm1,
                                                double t0, double tp1) {
  if (cr == 0.0) return F;
  double tc, tu, td;
  if (cr > 0.0) {
    tc = tm1;
    tu = tm2;
    td = t0;
  } else {
    tc = t0;
    tu = tp1;
    td = tm1;
  }
  double diff = td - tu;
  double nc = 0.0, nu = 0.0;
  if (diff != 0.0) {
    nc = (tc - tu) / diff;
    nu = (F - tu) / diff;
  }
  if (nc >= 0.0 && nc <= 1.0) {
    if (nu > 1.0)
      F = td;
    else if (nu < nc)
      F = tu + nc * (td - tu);
    else if (nu > nc / fabs(cr))
      F = tu + nc * (td - tu) / fabs(cr);
  } else
    F = tu + nc * (td - tu);
  return F;
}

// Face values of the other schemes (advect's dispatch, tracers.c:1509-1527),
// tm2..tp1 the tracer at i-2, i-1, i, i+1 of the face's cell:
//   order2_do (:1690-1709)        d (t0 - tm1) + tm1 (d: d3 / d4 / w5)
//   order4_do (:1757-1776)        (7 (tm1 + t0) - (tp1 + tm2)) / 12
//   quickest_uniform (:1944-2031) QUICKEST with uniform-grid curvature
//   order2_upwind_do (:3008-3036) the upwind pair weighted by the Courant number
__device__ __forceinline__ double order2_face(double d, double tm1, double t0) {
  return d * (t0 - tm1) + tm1;
}
__device__ __forceinline__ double order4_face(double tm2, double tm1, double t0, double tp1) {
  return (7.0 * (tm1 + t0) - (tp1 + tm2)) / 12.0;
}
__device__ __forceinline__ double quickest_co_face(double cr, double tm2, double tm1, double t0,
                                                   double tp1) {
  double face = 0.5 * (t0 + tm1);
  double grad = t0 - tm1;
  double curv = 0.0;
  if (cr > 0.0)
    curv = t0 - 2.0 * tm1 + tm2;
  else if (cr < 0.0)
    curv = tp1 - 2.0 * t0 + tm1;
  return face - 0.5 * cr * grad - (1.0 - cr * cr) * curv / 6.0;
}
__device__ __forceinline__ double order2_uw_face(double vel, double cn, double tm2, double tm1,
                                                 double t0, double tp1) {
  if (vel > 0.0) return 0.5 * (3.0 - cn) * tm1 - 0.5 * (1.0 - cn) * tm2;
  if (vel < 0.0) return 0.5 * (3.0 - cn) * t0 - 0.5 * (1.0 - cn) * tp1;
  return 0.0;
}
// order1 (:1584-1617): the upwind value times the volume flux, split by sign
// (w6..w9 of :497-513), with no limiter
__device__ __forceinline__ double order1_flux(double U, double tm1, double t0) {
  const double up = 0.5 * (U + fabs(U)), dn = 0.5 * (U - fabs(U));
  return up * tm1 + dn * t0;
}

// Face value of a horizontal face of scheme trasc before the limiter; eb: the
// face is an interior face (w3_e1 / w3_e2), the only faces the centred and
// second-order upwind schemes and Van Leer fill.
__device__ __forceinline__ double hface_value(int trasc, bool eb, double cr, double vel,
                                              const Face2D &m, double tm2, double tm1,
                                              double t0, double tp1) {
  switch (trasc) {
    case SHOC_TR_QUICKEST: return quickest_face(cr, m, tm2, tm1, t0, tp1);
    case SHOC_TR_QUICKEST_CO: return quickest_co_face(cr, tm2, tm1, t0, tp1);
    case SHOC_TR_VANLEER: return eb ? vanleer_face(vel, cr, tm2, tm1, t0, tp1) : 0.0;
    case SHOC_TR_ORDER2: return eb ? order2_face(m.d, tm1, t0) : 0.0;
    case SHOC_TR_ORDER4: return eb ? order4_face(tm2, tm1, t0, tp1) : 0.0;
    case SHOC_TR_ORDER2_UW: return eb ? order2_uw_face(vel, cr, tm2, tm1, t0, tp1) : 0.0;
  }
  return 0.0;
}

// Final e1 flux through the west face of wet cell c (advect + hor_diffuse):
// tm2..tp1 = tr at xm1[xm1[c]], xm1[c], c, xp1[c].
__device__ __forceinline__ double flux_x(const Geo &G, const Flow &F, const Work &W,
                                         const Opt &O, uint8_t fl, bool adv, bool hdiff, int c,
                                         int c2, double tm2, double tm1, double t0,
                                         double tp1) {
  double v = 0.0;
  if (adv && O.trasc == SHOC_TR_ORDER1) {
    v = order1_flux(F.u1flux3d[c], tm1, t0);
  } else if (adv) {
    double cr = W.w6[c];
    v = hface_value(O.trasc, (fl & CF_E1) != 0, cr, F.u1[c], G.fx[c2], tm2, tm1, t0, tp1);
    if (O.ultimate && (fl & CF_E1)) v = ultimate_face(cr, v, tm2, tm1, t0, tp1);
    v *= F.u1flux3d[c];
  }
  if (hdiff) {
    double csx = F.dzu1[c] * G.h2au1[c2] * 1.0;
    v -= (csx * F.u1kh[c] * (t0 - tm1) / G.h1au1[c2]);
  }
  return v;
}

__device__ __forceinline__ double flux_y(const Geo &G, const Flow &F, const Work &W,
                                         const Opt &O, uint8_t fl, bool adv, bool hdiff, int c,
                                         int c2, double tm2, double tm1, double t0,
                                         double tp1) {
  double v = 0.0;
  if (adv && O.trasc == SHOC_TR_ORDER1) {
    v = order1_flux(F.u2flux3d[c], tm1, t0);
  } else if (adv) {
    double cr = W.w7[c];
    v = hface_value(O.trasc, (fl & CF_E2) != 0, cr, F.u2[c], G.fy[c2], tm2, tm1, t0, tp1);
    if (O.ultimate && (fl & CF_E2)) v = ultimate_face(cr, v, tm2, tm1, t0, tp1);
    v *= F.u2flux3d[c];
  }
  if (hdiff) {
    double csy = F.dzu2[c] * G.h1au2[c2] * 1.0;
    v -= (csy * F.u2kh[c] * (t0 - tm1) / G.h2au2[c2]);
  }
  return v;
}

// Vertical flux through the bottom face of s1 cell c (advect, :1571-1574).
// w9m/w90/w9p = w9 at zm1, c, zp1; tm2..tp1 = tr at zm2, zm1, c, zp1.
__device__ __forceinline__ double flux_z(const Flow &F, const Work &W, const Opt &O, int c,
                                         double w9m, double w90, double w9p, double tm2,
                                         double tm1, double t0, double tp1, double dtu) {
  const double wc = F.w[c];
  if (O.trasc == SHOC_TR_ORDER1)  // order1 (:1611-1616)
    return dtu * (0.5 * (wc + fabs(wc)) * tm1 + 0.5 * (wc - fabs(wc)) * t0);
  double cz = W.w8[c];
  double v;
  switch (O.trasc) {
    case SHOC_TR_QUICKEST:
      v = quickest_zface(cz, W.w5[c], W.dbz[c], W.dfz[c], w9m, w90, w9p, tm2, tm1, t0, tp1);
      break;
    case SHOC_TR_VANLEER: v = vanleer_face(wc, cz, tm2, tm1, t0, tp1); break;
    case SHOC_TR_QUICKEST_CO: v = quickest_co_face(cz, tm2, tm1, t0, tp1); break;
    case SHOC_TR_ORDER2: v = order2_face(W.w5[c], tm1, t0); break;
    case SHOC_TR_ORDER4: v = order4_face(tm2, tm1, t0, tp1); break;
    case SHOC_TR_ORDER2_UW: v = order2_uw_face(wc, cz, tm2, tm1, t0, tp1); break;
    default: v = 0.0;
  }
  if (O.ultimate) v = ultimate_face(cz, v, tm2, tm1, t0, tp1);
  return v * (wc * dtu);
}

}  // namespace shoc

namespace shoc {

// Per-thread Thomas storage: the main kernel keeps sol(k) in shared memory
// (layer-major, conflict free), the serial kernel in a local array.
struct SmemSol {
  double *base;
  int stride;
  __device__ __forceinline__ double &at(int k) { return base[(size_t)k * stride]; }
};
constexpr int kSerialMaxLayers = 128;
struct LocalSol {
  double v[kSerialMaxLayers];
  __device__ __forceinline__ double &at(int k) { return v[k]; }
};

// One (column, tracer) pair through one sub-step: advection (QUICKEST or Van
// Leer, ULTIMATE), horizontal diffusion, flux divergence, interior update
// (advect_diffuse, tracers.c:849-925), surf_conc (:3047-3207), tr_bounds
// (:3217-3324) and, when LAST, the implicit vertical diffusion
// (implicit_vdiff_tr, :4067-4214) with the LU factors from k_set_dz.
//
// The loop over layers runs from kstart (the lowest bottom layer of the warp)
// to the surface layer, so the lanes of a warp touch one layer at a time and
// their loads coalesce; a lane acts once k reaches its own bottom layer.
// c3_moved carries tr_bounds' thin-surface cursor between tracers of one
// column (tracers.c:3250-3270 does not reset it); the main kernel only runs
// columns where the cursor cannot move.  TR is the tracer storage type
// (double, or float for the FP32-mixed path); arithmetic is FP64 either way.
template <bool LAST, class Sol, class TR>
__device__ __forceinline__ void column_pass(const Geo &G, const Flow &F, const Work &W,
                                            const Opt &O, const TrSet &T, const SubStep &ss,
                                            const TR *__restrict__ tri,
                                            TR *__restrict__ tro, int col, int n, int kstart,
                                            bool act, Sol &sol, bool &c3_moved,
                                            unsigned long long &warn, int &stat) {
  ColInfo ci = {0, 0, 0, 0, 0, 0};
  int cbot = 0, ctop = 0, kb = G.nz;
  if (act) {
    ci = W.col[col];
    cbot = G.col_bot[col];
    ctop = G.col_top[col];
    kb = G.col_kb[col];
  }
  const uint8_t tf = T.trf[n];
  const bool tbdy = (tf & TR_TBDY) != 0;
  const bool wet = (ci.flags & COL_WET) != 0;
  const bool upd = tbdy && wet;
  const bool adv = upd && (tf & TR_ADV);
  const bool hd = upd && (tf & TR_HDIFF);
  const bool vdf = LAST && (tf & TR_VDIFF) && wet;
  const bool vd = vdf && !(ci.flags & (COL_SINGLE | COL_NOSOLVE));
  const double dtu = ss.dtu;
  const int c2 = ctop;
  const double area = act ? G.cellarea[c2] : 1.0;
  const double mn = T.mintr[n], mx = T.maxtr[n];
  const int s = ci.s, co = ci.co, cs = ci.cs, cbs = ci.cbs;
  // sub-step surface elevations (tracers.c:746-756, :1027-1031)
  double sub = 0.0, osub = 0.0;
  if (upd) {
    double eta = F.eta[c2], oe = F.oldeta[c2];
    sub = oe + ss.subeta_f * (eta - oe);
    osub = ss.first ? oe : oe + ss.osub_f * (eta - oe);
  }

  int c = cbot, czp1 = 0, czp2 = 0;
  double t0 = 0.0, tp1 = 0.0, tp2 = 0.0, tm1 = 0.0, tm2 = 0.0;
  double w9m = 0.0, w90 = 0.0, w9p = 0.0, w9pp = 0.0;
  double Fzb = 0.0, surftr = 0.0, wbot = 0.0, dzs = 0.0, svol = 0.0;
  double a_below = 0.0, solp = 0.0, ts_old = 0.0;
  int phase = 0, k_s = 0, k_cs = 0;

  for (int k = kstart; k < G.nz; ++k) {
    if (!act || k < kb) continue;
    if (k == kb) {
      c = cbot;
      t0 = tri[c];
      tm1 = t0;  // sediment ghost holds the bottom value (tracers.c:827-830)
      tm2 = t0;
      czp1 = G.zp1[c];
      czp2 = G.zp1[czp1];
      tp1 = tri[czp1];
      tp2 = tri[czp2];
      w9m = 0.0;  // w9 of the sediment cell
      w90 = W.w9[c];
      w9p = W.w9[czp1];
      w9pp = W.w9[czp2];
      int sed = G.zm1[c];
      tro[sed] = (TR)(tbdy ? t0 : tri[sed]);
    } else {
      c = czp1;
      czp1 = czp2;
      czp2 = G.zp1[czp1];
      tm2 = tm1;
      tm1 = t0;
      t0 = tp1;
      tp1 = tp2;
      tp2 = tri[czp2];
      w9m = w90;
      w90 = w9p;
      w9p = w9pp;
      w9pp = W.w9[czp2];
    }
    if (c == cs) k_cs = k;
    if (!upd) {
      tro[c] = (TR)(t0);
      if (isnan(t0)) stat |= ST_NAN;
      if (vd && c <= cbs && c >= cs) {
        double dzdt = W.vd_dzdt[c];
        double rhs = dzdt * t0;
        double sl;
        if (c == cbs) {
          rhs = rhs + 0.0;
          sl = rhs / W.vd_div[c];
        } else {
          if (c == cs) rhs = rhs - 0.0;
          sl = (rhs - W.vd_cm1[c] * solp) / W.vd_div[c];
        }
        sol.at(k) = sl;
        solp = sl;
      }
      continue;
    }
    // horizontal fluxes and their divergence (dtracer, tracers.c:888-892)
    double dtr = 0.0;
    if (adv || hd) {
      const int xm1 = G.xm1[c], xp1 = G.xp1[c], ym1 = G.ym1[c], yp1 = G.yp1[c];
      const uint8_t fc = G.cflag[c], fe = G.cflag[xp1], fn = G.cflag[yp1];
      const double txm1 = tri[xm1], txp1 = tri[xp1], tym1 = tri[ym1], typ1 = tri[yp1];
      const double txm2 = tri[G.xm1[xm1]], tym2 = tri[G.ym1[ym1]];
      double Fxw = flux_x(G, F, W, O, fc, adv, hd, c, c2, txm2, txm1, t0, txp1);
      double Fys = flux_y(G, F, W, O, fc, adv, hd, c, c2, tym2, tym1, t0, typ1);
      double Fxe = 0.0, Fyn = 0.0;
      if (fe & CF_WET)
        Fxe = flux_x(G, F, W, O, fe, adv, hd, xp1, G.m2d[xp1], txm1, t0, txp1, tri[G.xp1[xp1]]);
      else if (adv && O.trasc == SHOC_TR_ORDER1)  // order1 fills the ghost cells' faces too
        Fxe = order1_flux(F.u1flux3d[xp1], t0, txp1);
      if (fn & CF_WET)
        Fyn = flux_y(G, F, W, O, fn, adv, hd, yp1, G.m2d[yp1], tym1, t0, typ1, tri[G.yp1[yp1]]);
      else if (adv && O.trasc == SHOC_TR_ORDER1)
        Fyn = order1_flux(F.u2flux3d[yp1], t0, typ1);
      dtr = (Fxe - Fxw + Fyn - Fys) * dtu;
    }
    if (c > s) {
      // interior cell (tracers.c:912-925); Ds = Hn1 = 1 in z coordinates
      if (k == kb && adv) Fzb = flux_z(F, W, O, c, w9m, w90, w9p, tm2, tm1, t0, tp1, dtu);
      double Fzt = adv ? flux_z(F, W, O, czp1, w90, w9p, w9pp, tm1, t0, tp1, tp2, dtu) : 0.0;
      double a = t0 * 1.0;
      a -= ((dtr / area + (Fzt - Fzb)) / W.dz[c]);
      a /= 1.0;
      Fzb = Fzt;
      if (czp1 == s) a_below = a;
      // tr_bounds clip and range check (:3278-3293)
      if (mn <= kClipEps && a < mn) a = mn;
      if (a < mn || a > mx) warn++;
      tro[c] = (TR)(a);
      if (isnan(a)) stat |= ST_NAN;
      if (vd && c <= cbs && c >= cs) {
        double dzdt = W.vd_dzdt[c];
        double rhs = dzdt * a;
        double sl;
        if (c == cbs) {
          rhs = rhs + 0.0;
          sl = rhs / W.vd_div[c];
        } else {
          sl = (rhs - W.vd_cm1[c] * solp) / W.vd_div[c];
        }
        sol.at(k) = sl;
        solp = sl;
      }
    } else {
      if (c == s) {
        // surf_conc set-up (:3097-3112)
        k_s = k;
        ts_old = t0;
        if (k == kb && adv) Fzb = flux_z(F, W, O, c, w9m, w90, w9p, tm2, tm1, t0, tp1, dtu);
        double fcbot = -Fzb * area;
        surftr = -fcbot;
        wbot = (c == cbot) ? G.botz[c2] : G.gridz[c];
        dzs = sub - wbot;
        svol = dzs * area;
        phase = 1;
      }
      if (phase == 1) {
        if (c != co) {
          double wtop = G.gridz[czp1];
          surftr += (t0 * area * (wtop - wbot) - dtr);
          wbot = G.gridz[czp1];
        } else {
          double wb = (c == cbot) ? G.botz[c2] : G.gridz[c];
          surftr += (t0 * area * (osub - wb) - dtr);
          phase = 2;
        }
      } else if (phase == 2) {
        surftr -= (dtr);
      }
    }
  }
  if (!act || !upd) {
    if (act && vdf && (ci.flags & COL_SINGLE)) {
      // one-layer column (tracers.c:4125-4132): max(dzcell, hmin)
      double h = W.dz[cs] > O.hmin ? W.dz[cs] : O.hmin;
      double v = tro[cs];
      tro[cs] = (TR)(v + F.dt * (0.0 - 0.0) / h);
      if (isnan(v)) stat |= ST_NAN;
    } else if (act && vd) {
      double x = sol.at(k_cs);
      double a = tro[cs];
      double fin = a + (x - a) * 1.0;
      tro[cs] = (TR)(fin);
      if (isnan(fin)) stat |= ST_NAN;
      double udp = W.vd_ud[cs];
      int cc = cs, k = k_cs;
      while (cc != cbs && k > kb) {
        cc = G.zm1[cc];
        --k;
        x = sol.at(k) - udp * x;
        a = tro[cc];
        fin = a + (x - a) * 1.0;
        tro[cc] = (TR)(fin);
        if (isnan(fin)) stat |= ST_NAN;
        udp = W.vd_ud[cc];
      }
    }
    return;
  }
  // surface value (tracers.c:944-961, :3199-3206)
  double vs = ts_old;
  if (adv) {
    double sv;
    if (svol == 0.0 || (surftr < 0.0 && dzs <= O.hmin))
      sv = 0.0;
    else
      sv = surftr / svol;
    vs = (G.botz[c2] > 0.0 && W.dz[s] < O.hmin) ? ts_old : sv;
  }
  // tr_bounds thin-surface fix (:3250-3272)
  if ((ci.flags & COL_THIN) && (vs < mn || vs > mx)) {
    if (!c3_moved) vs = a_below;
    if (s != ctop) c3_moved = true;
  }
  if (mn <= kClipEps && vs < mn) vs = mn;
  if (vs < mn || vs > mx) warn++;
  if (isnan(vs)) stat |= ST_NAN;
  // surface and the cells above it (:3309-3323)
  {
    int cc = s;
    tro[cc] = (TR)(vs);
    for (int it = 0; cc != ctop && it < G.nz; ++it) {
      cc = G.zp1[cc];
      tro[cc] = (TR)(vs);
    }
  }
  if (!vdf) return;
  if (ci.flags & COL_SINGLE) {
    double h = W.dz[cs] > O.hmin ? W.dz[cs] : O.hmin;
    tro[cs] = (TR)(vs + F.dt * (0.0 - 0.0) / h);
    return;
  }
  // Thomas forward over the surface cell and the cells above it up to cs
  {
    int cc = s, k = k_s;
    for (;;) {
      if (cc <= cbs && cc >= cs) {
        double dzdt = W.vd_dzdt[cc];
        double rhs = dzdt * vs;
        double sl;
        if (cc == cbs) {
          rhs = rhs + 0.0;
          sl = rhs / W.vd_div[cc];
        } else {
          if (cc == cs) rhs = rhs - 0.0;
          sl = (rhs - W.vd_cm1[cc] * solp) / W.vd_div[cc];
        }
        sol.at(k) = sl;
        solp = sl;
      }
      if (cc == cs || cc == ctop || k >= G.nz - 1) break;
      cc = G.zp1[cc];
      ++k;
    }
  }
  // back substitution and update (:4197-4205)
  {
    double x = sol.at(k_cs);
    double a = (cs > s) ? tro[cs] : vs;
    double fin = a + (x - a) * 1.0;
    tro[cs] = (TR)(fin);
    if (isnan(fin)) stat |= ST_NAN;
    double udp = W.vd_ud[cs];
    int cc = cs, k = k_cs;
    while (cc != cbs && k > kb) {
      cc = G.zm1[cc];
      --k;
      x = sol.at(k) - udp * x;
      a = (cc > s) ? tro[cc] : vs;
      fin = a + (x - a) * 1.0;
      tro[cc] = (TR)(fin);
      if (isnan(fin)) stat |= ST_NAN;
      udp = W.vd_ud[cc];
    }
  }
}

}  // namespace shoc
