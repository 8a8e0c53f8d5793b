// shoc_tr_stage.cuh -- layer-synchronous transport kernels (the fast path).
//
// A block owns 32 adjacent wet columns (one per lane) and NW tracers (one
// per warp).  All warps walk the columns' layers together, bottom to top.
// Everything that does not depend on the tracer -- the cell and its
// neighbours' sparse indices, Courant numbers, face coefficients, layer
// thickness, the implicit solve's LU factors -- is staged for the 32 cells of
// the next layer into shared memory while the tracer warps work on the
// current one (double buffer, one __syncthreads per layer).  Tracer warps
// then only issue the loads of their own tracer's stencil values; the values
// of x-neighbours that are lanes of the same warp come through shuffles, and
// so does the flux through the east face (the west face of the next lane).
// The flux divergence of cell k is finished one layer late, once the flux
// through its top face (the bottom face of cell k+1) is known.
//
// Columns whose free surface crosses a layer face during the step, whose
// tr_bounds thin-surface cursor couples tracers, or whose implicit solve is
// degenerate go through the general column path (column_pass) instead.
#pragma once
#include "shoc_tr_kernels.cuh"

namespace shoc {

// Columns the staged kernels handle: wet, surface cell unchanged this step
// (s == co == cs), implicit solve spanning the whole column (or one layer).
__device__ __forceinline__ bool staged_column(const ColInfo &ci, int cbot) {
  if (!(ci.flags & COL_WET)) return false;
  if (ci.flags & (COL_SERIAL | COL_NOSOLVE)) return false;
  if (ci.s != ci.co || ci.s != ci.cs) return false;
  if (!(ci.flags & COL_SINGLE) && ci.cbs != cbot) return false;
  return true;
}

constexpr int SH_XM1 = 1, SH_XM2 = 2, SH_XP1 = 4, SH_XP2 = 8;

// ===========================================================================
// FP32-mixed policy: FP32 tracers, face values and Thomas sweeps; FP64 flux
// divergence, surface column-mass sum (Neumaier), implicit-solve residual and
// one refinement step.

namespace f32 {

// QUICKEST (quickest(), tracers.c:1870-1884) is, for a given sign of the
// Courant number, linear in the four stencil values:
//   F = w0 tm2 + w1 tm1 + w2 t0 + w3 tp1
// with the tracer-independent weights folded by the staging warps from
// a = d - cr/2, b = (1 - cr^2)/6 and the upwind curvature factors A, B:
//   cr > 0: w0 = -b B, w1 = 1 - a + 2b, w2 = a - b A, w3 = 0
//   cr < 0: w0 = 0,    w1 = 1 - a - b B, w2 = a + 2b, w3 = -b A
//   cr = 0: w1 = 1 - d, w2 = d
// Van Leer keeps w0 = (1 -+ cr)/2 and its flux-limiter form.  Then ULTIMATE
// (ircr = 1/|cr|), times the volume flux U, minus K (t0 - tm1) for horizontal
// diffusion.  A face that carries nothing has all weights, U and K zero.
struct Face {
  float w0, w1, w2, w3, ircr, U, K;
  int bits;
};
constexpr int FB_POS = 1, FB_NEG = 2, FB_ULT = 4;

struct Stage {
  int c, zp1;
  int xm1, xm2, xp1, xp2, ym1, ym2, yp1, yp2;
  int share;
  int pad;
  Face fxw, fxe, fys, fyn, fzb;
  float idz;
  int pad2;
};

// per-column metric factors of one horizontal direction (precomputed once)
struct Face2 {
  float d, Ap, Bp, Am, Bm;  // A+/B+ = db*hm, db*h0; A-/B- = df*h0, df*hp
  float ih;                 // 1 / h1au1 (x) or 1 / h2au2 (y) of the face's column
};

__device__ __forceinline__ void face_zero(Face &f) {
  f.w0 = f.w1 = f.w2 = f.w3 = 0.f;
  f.ircr = f.U = f.K = 0.f;
  f.bits = 0;
}

// weights of one face from its Courant number and metric factors
__device__ __forceinline__ void set_face(Face &f, bool quick, float cr, float d, float Ap,
                                         float Bp, float Am, float Bm, float U, bool ult,
                                         float K) {
  f.bits = (cr > 0.f ? FB_POS : 0) | (cr < 0.f ? FB_NEG : 0) | ((ult && cr != 0.f) ? FB_ULT : 0);
  if (quick) {
    const float a = d - 0.5f * cr, b = (1.f - cr * cr) * (1.f / 6.f);
    if (cr > 0.f) {
      f.w0 = -b * Bp;
      f.w1 = 1.f - a + 2.f * b;
      f.w2 = a - b * Ap;
      f.w3 = 0.f;
    } else if (cr < 0.f) {
      f.w0 = 0.f;
      f.w1 = 1.f - a - b * Bm;
      f.w2 = a + 2.f * b;
      f.w3 = -b * Am;
    } else {
      f.w0 = 0.f;
      f.w1 = 1.f - d;
      f.w2 = d;
      f.w3 = 0.f;
    }
  } else {
    f.w0 = cr > 0.f ? 0.5f * (1.f - cr) : 0.5f * (1.f + cr);
    f.w1 = f.w2 = f.w3 = 0.f;
  }
  f.ircr = cr != 0.f ? __fdividef(1.f, fabsf(cr)) : 0.f;
  f.U = U;
  f.K = K;
}

// one face value: tm2..tp1 at i-2..i+1 of the face's cell
template <bool QUICK, bool ULT>
__device__ __forceinline__ float face(const Face &f, bool adv, bool hd, float tm2, float tm1,
                                      float t0, float tp1) {
  float F = 0.f;
  if (adv) {
    const bool pos = (f.bits & FB_POS) != 0;
    if (QUICK) {
      F = f.w0 * tm2 + f.w1 * tm1 + f.w2 * t0 + f.w3 * tp1;
    } else {
      const bool neg = (f.bits & FB_NEG) != 0;
      const float p = pos ? (tm1 - tm2) : (t0 - tm1), q = pos ? (t0 - tm1) : (tp1 - t0);
      const float den = pos ? (t0 - tm2) : (tp1 - tm1);
      const float pq = p * q;
      const float df = pq > 0.f ? 2.f * __fdividef(pq, den) : 0.f;
      F = pos ? tm1 + f.w0 * df : (neg ? t0 - f.w0 * df : 0.f);
    }
    if (ULT && (f.bits & FB_ULT)) {
      // ulimate_filter (tracers.c:3526-3554) as selects
      const float tc = pos ? tm1 : t0, tu = pos ? tm2 : tp1, td = pos ? t0 : tm1;
      const float diff = td - tu;
      const float r = __fdividef(1.f, diff);
      const float nc = (tc - tu) * r, nu = (F - tu) * r;
      const float ncd = nc * diff;
      const float lim = tu + ncd;
      float G = F;
      if (nu > nc * f.ircr) G = tu + ncd * f.ircr;
      if (nu < nc) G = lim;
      if (nu > 1.f) G = td;
      if (!(nc >= 0.f && nc <= 1.f)) G = lim;
      // Upwind and downwind values equal in FP32: in FP64 they almost always
      // differ by a few ulps, nc is then huge and the limiter falls back to
      // upwind (tc); follow that rather than the exact-tie case (which
      // leaves the face unlimited), so FP32 rounding of the stored tracer
      // does not flip the limiter's decision.
      F = (diff == 0.f) ? (tc != tu ? tc : F) : G;
    }
    F *= f.U;
  }
  if (hd) F -= f.K * (t0 - tm1);
  return F;
}

// ---------------------------------------------------------------------------
// Staging of one layer (FP32 policy).  part: 0 indices, 1 x faces, 2 y faces,
// 3 z face, thickness and LU factors.  Every part walks its lane's column.

struct Walk {   // per-lane column walk of one staging part
  int c;        // cell at the current layer (0 when not started / inactive)
  float dzm2, dzm1, dz0;  // thickness window of part 3
};

constexpr int kParts = 7;  // 0 indices, 1-4 horizontal faces, 5 z face, 6 thickness + LU

__device__ __forceinline__ void stage_hface(Face &f, int c, bool x, const Geo &G, const Flow32 &F3,
                                            const Opt &O, bool any_hd, float fdtu,
                                            const Face2 *m2) {
  const uint8_t EB = x ? CF_E1 : CF_E2;
  const uint8_t fc = G.cflag[c];
  const bool quick = O.trasc == SHOC_TR_QUICKEST;
  if (!(fc & CF_WET)) {  // a ghost: the face carries nothing
    face_zero(f);
    return;
  }
  const Face2 m = m2[G.m2d[c]];
  const float cr = (x ? F3.u1[c] : F3.u2[c]) * fdtu * m.ih;
  const float K = any_hd ? (x ? F3.khx[c] : F3.khy[c]) : 0.f;
  if (!quick && !(fc & EB)) {  // Van Leer advects interior faces only
    face_zero(f);
    f.K = K;
    return;
  }
  set_face(f, quick, cr, m.d, m.Ap, m.Bp, m.Am, m.Bm, x ? F3.u1flux3d[c] : F3.u2flux3d[c],
           O.ultimate && (fc & EB), K);
}

__device__ __forceinline__ void stage_part(int part, int k, int lane, bool act, int kb, int ks,
                                           int cbot, const Geo &G, const Flow32 &F3,
                                           const Work &W, const Opt &O, bool any_hd,
                                           double dtu, const Face2 *fx2, const Face2 *fy2,
                                           Stage *st, int *colC, float4 *colLU, Walk &wk) {
  const bool on = act && k >= kb;
  int c = 0;
  if (on) c = (k == kb) ? cbot : G.zp1[wk.c];
  wk.c = c;
  Stage &S = st[lane];
  const float fdtu = (float)dtu;
  switch (part) {
    case 0: {
      int zp1 = 0, xm1 = 0, xp1 = 0, ym1 = 0, yp1 = 0, xm2 = 0, xp2 = 0, ym2 = 0, yp2 = 0;
      if (on) {
        zp1 = G.zp1[c];
        xm1 = G.xm1[c];
        xp1 = G.xp1[c];
        ym1 = G.ym1[c];
        yp1 = G.yp1[c];
        xm2 = G.xm1[xm1];
        xp2 = G.xp1[xp1];
        ym2 = G.ym1[ym1];
        yp2 = G.yp1[yp1];
      }
      const int cu1 = __shfl_up_sync(0xffffffffu, c, 1), cu2 = __shfl_up_sync(0xffffffffu, c, 2);
      const int cd1 = __shfl_down_sync(0xffffffffu, c, 1),
                cd2 = __shfl_down_sync(0xffffffffu, c, 2);
      int sh = 0;
      if (on) {
        if (lane >= 1 && cu1 && xm1 == cu1) sh |= SH_XM1;
        if (lane >= 2 && cu2 && xm2 == cu2) sh |= SH_XM2;
        if (lane <= 30 && cd1 && xp1 == cd1) sh |= SH_XP1;
        if (lane <= 29 && cd2 && xp2 == cd2) sh |= SH_XP2;
      }
      S.c = c;
      S.zp1 = zp1;
      S.xm1 = xm1; S.xm2 = xm2; S.xp1 = xp1; S.xp2 = xp2;
      S.ym1 = ym1; S.ym2 = ym2; S.yp1 = yp1; S.yp2 = yp2;
      S.share = sh;
      colC[k * 32 + lane] = c;
      break;
    }
    case 1:
      if (on) stage_hface(S.fxw, c, true, G, F3, O, any_hd, fdtu, fx2); else face_zero(S.fxw);
      break;
    case 2:
      if (on) stage_hface(S.fxe, G.xp1[c], true, G, F3, O, any_hd, fdtu, fx2); else face_zero(S.fxe);
      break;
    case 3:
      if (on) stage_hface(S.fys, c, false, G, F3, O, any_hd, fdtu, fy2); else face_zero(S.fys);
      break;
    case 4:
      if (on) stage_hface(S.fyn, G.yp1[c], false, G, F3, O, any_hd, fdtu, fy2); else face_zero(S.fyn);
      break;
    case 5: {
      Face &fz = S.fzb;
      if (!on) {
        face_zero(fz);
        break;
      }
      const int zp1 = G.zp1[c];
      if (k == kb) {
        wk.dzm2 = 0.f;  // thickness of the sediment cell (never set by set_dz)
        wk.dzm1 = 0.f;
      } else {
        wk.dzm2 = wk.dzm1;
        wk.dzm1 = wk.dz0;
      }
      wk.dz0 = W.dz32[c];
      if (k > ks) {  // above the surface: no z face
        face_zero(fz);
        break;
      }
      const float dzp1 = W.dz32[zp1];
      const float w9m = 0.5f * (wk.dzm1 + wk.dzm2);
      const float w90 = 0.5f * (wk.dz0 + wk.dzm1);
      // w9 of the cell above; the surface-layer cell maps onto itself
      const float w9p = (zp1 == c) ? w90 : 0.5f * (dzp1 + wk.dz0);
      const float wv = F3.w[c] * fdtu;
      const float cz = __fdividef(wv, w90);
      const float db = __fdividef(2.f, w9m + w90), df = __fdividef(2.f, w90 + w9p);
      set_face(fz, O.trasc == SHOC_TR_QUICKEST, cz, __fdividef(wk.dzm1, wk.dzm1 + wk.dz0),
               db * w9m, db * w90, df * w90, df * w9p, wv, O.ultimate != 0, 0.f);
      break;
    }
    default: {  // 6
      if (!on) break;
      S.idz = __fdividef(1.f, W.dz32[c]);
      colLU[k * 32 + lane] = (k <= ks) ? W.lu32[c] : make_float4(0.f, 0.f, 0.f, 0.f);
      break;
    }
  }
}

__device__ __forceinline__ void neumaier_add(double &s, double &comp, double v) {
  double u = s + v;
  comp += (fabs(s) >= fabs(v)) ? (s - u) + v : (v - u) + s;
  s = u;
}

}  // namespace f32

// ---------------------------------------------------------------------------
// The FP32-mixed staged transport kernel.
//
// Shared memory: Stage[3][32] | int colC[nz][32] | float4 colLU[nz][32] |
// float Sv[nz][nw][32] (per tracer-lane Thomas storage).
template <bool LAST, bool QUICK, bool ULT>
__global__ void __launch_bounds__(256) k_stage32(Geo G, Flow F, Flow32 F3, Work W, Opt O,
                                                 TrSet T, SubStep ss, const f32::Face2 *fx2,
                                                 const f32::Face2 *fy2,
                                                 const float *__restrict__ tri,
                                                 float *__restrict__ tro, int nw, int nchunk,
                                                 int any_hd) {
  using namespace f32;
  extern __shared__ __align__(16) unsigned char smem[];
  Stage *stg = reinterpret_cast<Stage *>(smem);                       // [3][32] ring
  int *colC = reinterpret_cast<int *>(stg + 3 * 32);                   // [nz][32]
  float4 *colLU = reinterpret_cast<float4 *>(colC + G.nz * 32);        // [nz][32]
  float *Sv = reinterpret_cast<float *>(colLU + G.nz * 32);            // [nz][nw][32]

  const int lane = threadIdx.x, wy = threadIdx.y;
  const int tile = blockIdx.x / nchunk, chunk = blockIdx.x % nchunk;
  const int col = tile * 32 + lane;
  const int slot = chunk * nw + wy;
  const bool slot_ok = slot < T.nslot;

  // column set-up (every warp holds its lane's column)
  bool act = col < G.ncol;
  ColInfo ci = {0, 0, 0, 0, 0};
  int cbot = 0, c2 = 0, kb = G.nz, ks = 0;
  if (act) {
    ci = W.col[col];
    cbot = G.col_bot[col];
    c2 = G.col_top[col];
    act = staged_column(ci, cbot);
  }
  if (act) {
    kb = G.col_kb[col];
    ks = kb;
    int c = cbot;
    for (int it = 0; c != ci.s && it < G.nz; ++it) {  // layer of the surface cell
      c = G.zp1[c];
      ++ks;
    }
    if (c != ci.s || ks >= G.nz) {  // surface cell not in this column: leave it alone
      act = false;
      kb = G.nz;
    }
  }
  const int kstart = __reduce_min_sync(0xffffffffu, act ? kb : G.nz);
  int kmin = kstart;
  // block-wide minimum (all warps hold the same columns, so the warp value is it)

  // tracer of this warp
  const int n = slot_ok ? T.slot_tr[slot] : 0;
  const uint8_t tf = slot_ok ? T.trf[n] : 0;
  const bool tbdy = (tf & TR_TBDY) != 0;
  const bool adv = tbdy && (tf & TR_ADV);
  const bool hd = tbdy && (tf & TR_HDIFF);
  const bool vdf = LAST && (tf & TR_VDIFF);
  const bool single = (ci.flags & COL_SINGLE) != 0;
  const double mn = slot_ok ? T.mintr[n] : 0.0, mx = slot_ok ? T.maxtr[n] : 0.0;
  const float *tr = tri + (size_t)n * G.S;
  float *to = tro + (size_t)n * G.S;
  float *myS = Sv + wy * 32 + lane;
  const int sstride = nw * 32;
  const double dtu = ss.dtu;
  double area = 1.0, ia = 1.0, sub = 0.0, osub = 0.0, botz2 = 0.0;
  if (act) {
    area = G.cellarea[c2];
    ia = 1.0 / area;
    double eta = F.eta[c2], oe = F.oldeta[c2];
    sub = oe + ss.subeta_f * (eta - oe);
    osub = ss.first ? oe : oe + ss.osub_f * (eta - oe);
    botz2 = G.botz[c2];
  }

  // staging parts of this warp
  Walk wk[kParts];
  for (int q = 0; q < kParts; ++q) wk[q] = {0, 0.f, 0.f, 0.f};
  auto stage_layer = [&](int k) {
#pragma unroll
    for (int q = 0; q < kParts; ++q) {
      const int part = wy + q * nw;
      if (part < kParts)
        stage_part(part, k, lane, act, kb, ks, cbot, G, F3, W, O, any_hd != 0, dtu, fx2, fy2,
                   stg + (k % 3) * 32, colC, colLU, wk[q]);
    }
  };
  // layers are staged two ahead of the one being computed (3-slot ring);
  // each iteration also prefetches the next layer's tracer values
  if (kmin < G.nz) stage_layer(kmin);
  if (kmin + 1 < G.nz) stage_layer(kmin + 1);
  __syncthreads();

  // per tracer-lane walk state
  float tm2 = 0.f, tm1 = 0.f, t0 = 0.f, tp1 = 0.f;
  float Fzb_prev = 0.f;
  double dtr_prev = 0.0, idz_prev = 0.0, t_prev = 0.0;
  int c_prev = 0;
  double a_below = 0.0;
  double ssum = 0.0, scomp = 0.0;  // surface column mass (Neumaier)
  float fwd_prev = 0.f;            // Thomas forward carry
  double ts_old = 0.0, dtr_s = 0.0, Fzb_s = 0.0;
  long long nwarn = 0;
  const bool work = slot_ok && act;
  const bool hor = tbdy && (adv || hd);

  // tracer values of one layer, loaded one layer ahead of their use
  struct Pre {
    float t0, tp, xm1, xm2, xp1, xp2, ym1, ym2, yp1, yp2;
  };
  auto prefetch = [&](int k, Pre &p) {
    if (!(work && k >= kb && k < G.nz)) return;
    const Stage &S = stg[(k % 3) * 32 + lane];
    if (k == kb) p.t0 = tr[S.c];
    p.tp = tr[S.zp1];
    if (hor) {
      const int sh = S.share;
      p.ym1 = tr[S.ym1];
      p.ym2 = tr[S.ym2];
      p.yp1 = tr[S.yp1];
      p.yp2 = tr[S.yp2];
      if (!(sh & SH_XM1)) p.xm1 = tr[S.xm1];
      if (!(sh & SH_XM2)) p.xm2 = tr[S.xm2];
      if (!(sh & SH_XP1)) p.xp1 = tr[S.xp1];
      if (!(sh & (SH_XP1 | SH_XP2))) p.xp2 = tr[S.xp2];
    }
  };
  Pre cur = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  Pre nxt = cur;
  prefetch(kmin, cur);

  for (int k = kmin; k < G.nz; ++k) {
    if (k + 2 < G.nz) stage_layer(k + 2);
    prefetch(k + 1, nxt);
    const Stage &S = stg[(k % 3) * 32 + lane];
    const bool on = work && k >= kb;
    // vertical window
    if (on) {
      if (k == kb) {
        t0 = cur.t0;
        tm1 = t0;  // sediment ghost holds the bottom value (tracers.c:827-830)
        tm2 = t0;
      } else {
        tm2 = tm1;
        tm1 = t0;
        t0 = tp1;
      }
      tp1 = cur.tp;
    }
    // x-neighbour values from the neighbouring lanes
    const float u1v = __shfl_up_sync(0xffffffffu, t0, 1);
    const float u2v = __shfl_up_sync(0xffffffffu, t0, 2);
    const float d1v = __shfl_down_sync(0xffffffffu, t0, 1);
    const float d2v = __shfl_down_sync(0xffffffffu, t0, 2);
    float Fxw = 0.f, Fxe = 0.f, Fys = 0.f, Fyn = 0.f, Fzb = 0.f;
    if (on && hor) {
      const int sh = S.share;
      const float txm1 = (sh & SH_XM1) ? u1v : cur.xm1;
      const float txm2 = (sh & SH_XM2) ? u2v : cur.xm2;
      const float txp1 = (sh & SH_XP1) ? d1v : cur.xp1;
      Fxw = face<QUICK, ULT>(S.fxw, adv, hd, txm2, txm1, t0, txp1);
      Fys = face<QUICK, ULT>(S.fys, adv, hd, cur.ym2, cur.ym1, t0, cur.yp1);
      Fyn = face<QUICK, ULT>(S.fyn, adv, hd, cur.ym1, t0, cur.yp1, cur.yp2);
      if (!(sh & SH_XP1)) {
        const float txp2 = (sh & SH_XP2) ? d2v : cur.xp2;
        Fxe = face<QUICK, ULT>(S.fxe, adv, hd, txm1, t0, txp1, txp2);
      }
      if (adv) Fzb = face<QUICK, ULT>(S.fzb, true, false, tm2, tm1, t0, tp1);
    }
    const float Fnext = __shfl_down_sync(0xffffffffu, Fxw, 1);
    if (on) {
      if (S.share & SH_XP1) Fxe = Fnext;
      // FP64 flux divergence (tracers.c:888-892)
      const double dtr =
          (((double)Fxe - (double)Fxw) + ((double)Fyn - (double)Fys)) * dtu;
      // finish the cell below: its top-face flux is this cell's bottom face
      if (tbdy && k > kb && c_prev) {
        double a = t_prev - (dtr_prev * ia + ((double)Fzb - (double)Fzb_prev)) * idz_prev;
        if (k == ks) a_below = a;
        if (mn <= kClipEps && a < mn) a = mn;
        if (a < mn || a > mx) ++nwarn;
        const float a32 = (float)a;
        to[c_prev] = a32;
        if (vdf && !single) {  // Thomas forward (FP32) for layer k-1
          const float4 lu = colLU[(k - 1) * 32 + lane];
          const float s = (k - 1 == kb) ? lu.x * a32 * lu.z : (lu.x * a32 - lu.y * fwd_prev) * lu.z;
          myS[(k - 1) * sstride] = s;
          fwd_prev = s;
        }
      }
      if (k == kb) to[G.zm1[S.c]] = tbdy ? t0 : tr[G.zm1[S.c]];  // sediment ghost
      if (!tbdy) {
        to[S.c] = t0;
        if (vdf && !single && k <= ks) {
          const float4 lu = colLU[k * 32 + lane];
          const float s = (k == kb) ? lu.x * t0 * lu.z : (lu.x * t0 - lu.y * fwd_prev) * lu.z;
          myS[k * sstride] = s;
          fwd_prev = s;
        }
      } else if (k < ks) {
        c_prev = S.c;
        t_prev = (double)t0;
        dtr_prev = dtr;
        idz_prev = (double)S.idz;
        Fzb_prev = Fzb;
      } else if (k == ks) {
        // surf_conc with s == co (tracers.c:3097-3206): column mass in FP64
        c_prev = 0;
        ts_old = (double)t0;
        Fzb_s = (double)Fzb;
        dtr_s = dtr;
        ssum = 0.0;
        scomp = 0.0;
        neumaier_add(ssum, scomp, Fzb_s * area);
        const double wb = (S.c == cbot) ? botz2 : G.gridz[S.c];
        neumaier_add(ssum, scomp, ts_old * area * (osub - wb));
        neumaier_add(ssum, scomp, -dtr);
      } else {
        neumaier_add(ssum, scomp, -dtr);  // cells above the surface
      }
    }
    cur = nxt;
    __syncthreads();
  }
  if (!work) return;
  if (!tbdy) {
    if (vdf && single) {
      const double h = (double)W.dz32[ci.s] > O.hmin ? (double)W.dz32[ci.s] : O.hmin;
      to[ci.s] = (float)((double)to[ci.s] + F.dt * (0.0 - 0.0) / h);
    }
  } else {
    // surface value
    double vs = ts_old;
    if (adv) {
      const double wb = (ci.s == cbot) ? botz2 : G.gridz[ci.s];
      const double dzs = sub - wb;
      const double svol = dzs * area;
      const double st = ssum + scomp;
      const double sv = (svol == 0.0 || (st < 0.0 && dzs <= O.hmin)) ? 0.0 : st / svol;
      vs = (botz2 > 0.0 && (double)W.dz32[ci.s] < O.hmin) ? ts_old : sv;
    }
    if ((ci.flags & COL_THIN) && (vs < mn || vs > mx)) vs = a_below;
    if (mn <= kClipEps && vs < mn) vs = mn;
    if (vs < mn || vs > mx) ++nwarn;
    const float vs32 = (float)vs;
    {
      int cc = ci.s;
      to[cc] = vs32;
      for (int it = 0; cc != c2 && it < G.nz; ++it) {
        cc = G.zp1[cc];
        to[cc] = vs32;
      }
    }
    if (vdf && single) {
      const double h = (double)W.dz32[ci.s] > O.hmin ? (double)W.dz32[ci.s] : O.hmin;
      to[ci.s] = (float)(vs + F.dt * (0.0 - 0.0) / h);
    } else if (vdf) {
      const float4 lu = colLU[ks * 32 + lane];
      const float s = (ks == kb) ? lu.x * vs32 * lu.z : (lu.x * vs32 - lu.y * fwd_prev) * lu.z;
      myS[ks * sstride] = s;
    }
  }
  if (vdf && !single) {
    // back substitution (FP32) with the FP64 residual of the row above
    //   r(j) = dzdt (a - x) - cm1 (x(j-1) - x) - cp1 (x(j+1) - x)
    // (the difference form of b - A x for A = dzdt I + the diffusion operator)
    float xj1 = 0.f, xj2 = 0.f;  // x(k+1), x(k+2)
    for (int k = ks; k >= kb; --k) {
      const float4 lu = colLU[k * 32 + lane];
      const float x = (k == ks) ? myS[k * sstride] : myS[k * sstride] - colLU[(k + 1) * 32 + lane].w * xj1;
      if (k < ks) {
        // residual of row j = k + 1
        const int j = k + 1;
        const float4 lj = colLU[j * 32 + lane];
        const int cj = colC[j * 32 + lane];
        const double aj = (j == ks) ? (double)(float)to[cj] : (double)to[cj];
        const double xj = xj1;
        double r = (double)lj.x * (aj - xj) - (double)lj.y * ((double)x - xj);
        if (j < ks) r -= (double)colLU[(j + 1) * 32 + lane].y * ((double)xj2 - xj);
        myS[j * sstride] = (float)r;
        to[cj] = xj1;  // x(j) replaces a(j) in the tracer array
      }
      xj2 = xj1;
      xj1 = x;
      (void)lu;
    }
    {  // residual of the bottom row (cm1 = 0 there)
      const int j = kb;
      const float4 lj = colLU[j * 32 + lane];
      const int cj = colC[j * 32 + lane];
      const double aj = (double)to[cj], xj = xj1;
      double r = (double)lj.x * (aj - xj);
      if (j < ks) r -= (double)colLU[(j + 1) * 32 + lane].y * ((double)xj2 - xj);
      myS[j * sstride] = (float)r;
      to[cj] = xj1;
    }
    // correction solve (FP32 forward and back) and update in FP64
    float up = 0.f;
    for (int k = kb; k <= ks; ++k) {
      const float4 lu = colLU[k * 32 + lane];
      const float r = myS[k * sstride];
      const float u = (k == kb) ? r * lu.z : (r - lu.y * up) * lu.z;
      myS[k * sstride] = u;
      up = u;
    }
    float dn = 0.f;
    int stat = 0;
    for (int k = ks; k >= kb; --k) {
      const float d = (k == ks) ? myS[k * sstride] : myS[k * sstride] - colLU[(k + 1) * 32 + lane].w * dn;
      const int c = colC[k * 32 + lane];
      const float fin = (float)((double)to[c] + (double)d);
      to[c] = fin;
      if (isnan(fin)) stat = ST_NAN;
      dn = d;
    }
    if (stat) atomicOr(W.status, stat);
    // cells above the surface keep the surface value: the copy-up above
  }
  if (nwarn) atomicAdd(W.nwarn, (unsigned long long)nwarn);
}

}  // namespace shoc
