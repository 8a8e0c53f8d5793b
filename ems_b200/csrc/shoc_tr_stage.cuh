// shoc_tr_stage.cuh -- FP32 face arithmetic of the FP32-mixed path and the
// test that picks the columns the column-tile kernel handles.
//
// Columns whose free surface crosses a layer face during the step, whose
// tr_bounds thin-surface cursor couples tracers, or whose implicit solve is
// degenerate go through the general column path (column_pass) instead.
#pragma once
#include "shoc_tr_kernels.cuh"

namespace shoc {

// Columns the column-tile kernel handles: wet, surface cell unchanged this step
// (s == co == cs), implicit solve spanning the whole column (or one layer).
__device__ __forceinline__ bool staged_column(const ColInfo &ci, int cbot) {
  if (!(ci.flags & COL_WET)) return false;
  if (ci.flags & (COL_SERIAL | COL_NOSOLVE)) return false;
  if (ci.s != ci.co || ci.s != ci.cs) return false;
  if (!(ci.flags & COL_SINGLE) && ci.cbs != cbot) return false;
  return true;
}

// ===========================================================================
// FP32-mixed policy: FP32 tracers, face values and Thomas sweeps; FP64
// face fluxes (FP32 face value times the FP64 volume flux), flux divergence
// and cell update, surface column-mass sum (Neumaier), implicit-solve
// residual and one refinement step, and the columns' FP64 mass carry.

namespace f32 {

// QUICKEST (quickest(), tracers.c:1870-1884) is, for a given sign of the
// Courant number, linear in the upwind-side value tu (tm2 for cr > 0, tp1 for
// cr < 0) and the two values beside the face.  With a = d - cr/2,
// b = (1 - cr^2)/6 and the upwind curvature factors A + B = 2 (db (hm + h0),
// df (h0 + hp)), the curvature is a sum of differences, so the face value is
//   F = tm1 + wg (t0 - tm1) + wa (tu - tc)
// (tc = tm1 for cr > 0, t0 for cr < 0) with the tracer-independent weights
//   cr > 0: wg = a - b A,  wa = -b B
//   cr < 0: wg = a + b B,  wa = -b A
//   cr = 0: wg = d,        wa = 0
// folded once per cell.  The weights multiply differences, so their FP32
// rounding (the same every step while the flow is steady) moves the face
// value by a fraction of the differences, not of the value itself.  Van Leer
// keeps wa = (1 -+ cr)/2 and its flux-limiter form.  Then ULTIMATE
// (ircr = 1/|cr|); the face value times the FP64 volume flux U, minus
// K (t0 - tm1) for horizontal diffusion, is the FP64 flux.  A face that
// carries nothing has all weights, U and K zero.
struct Face {
  float wg, wa, ircr, K;
  double U;
  double V;  // FP32_COMP: U / |cr| in FP64 (set_face64; 0 otherwise)
  int bits;
};
constexpr int FB_POS = 1, FB_NEG = 2, FB_ULT = 4;

// per-column metric factors of one horizontal direction (precomputed once)
struct Face2 {
  float d, Ap, Bp, Am, Bm;  // A+/B+ = db*hm, db*h0; A-/B- = df*h0, df*hp
  float ih;                 // 1 / h1au1 (x) or 1 / h2au2 (y) of the face's column
};

__device__ __forceinline__ void face_zero(Face &f) {
  f.wg = f.wa = 0.f;
  f.ircr = f.K = 0.f;
  f.U = f.V = 0.0;
  f.bits = 0;
}

// Weights of one face from its Courant number and metric factors, with every
// rounding explicit (FMA contraction cannot change them): two threads folding
// the same face from the same inputs get the same bits, so a cell's east
// (north, top) face computed by the cell itself equals its neighbour's own
// west (south, bottom) face, and no mass is made between them.
__device__ __forceinline__ void set_face(Face &f, bool quick, float cr, float d, float Ap,
                                         float Bp, float Am, float Bm, double U, bool ult,
                                         float K) {
  f.bits = (cr > 0.f ? FB_POS : 0) | (cr < 0.f ? FB_NEG : 0) | ((ult && cr != 0.f) ? FB_ULT : 0);
  if (quick) {
    const float a = __fmaf_rn(-0.5f, cr, d);
    const float b = __fmul_rn(__fmaf_rn(-cr, cr, 1.f), 1.f / 6.f);
    if (cr > 0.f) {
      f.wg = __fmaf_rn(-b, Ap, a);
      f.wa = __fmul_rn(-b, Bp);
    } else if (cr < 0.f) {
      f.wg = __fmaf_rn(b, Bm, a);
      f.wa = __fmul_rn(-b, Am);
    } else {
      f.wg = d;
      f.wa = 0.f;
    }
  } else {
    f.wa = cr > 0.f ? __fmul_rn(0.5f, __fsub_rn(1.f, cr)) : __fmul_rn(0.5f, __fadd_rn(1.f, cr));
    f.wg = 0.f;
  }
  f.ircr = cr != 0.f ? __frcp_rn(fabsf(cr)) : 0.f;
  f.U = U;
  f.V = 0.0;
  f.K = K;
}

// FP32_COMP: set_face from the FP64 Courant number and metric factors, each
// weight formed in FP64 and rounded once, and V = U / |cr| in FP64: the
// volume flux per unit of tc - tu of a face ULTIMATE caps at its Courant
// bound (tu + (tc - tu) / |cr|).  That cap does not shrink with the Courant
// number, so it is applied in FP64 to compensated values (face_c).
__device__ __forceinline__ void set_face64(Face &f, bool quick, double cr, double d, double Ap,
                                           double Bp, double Am, double Bm, double U, bool ult,
                                           float K) {
  f.bits = (cr > 0.0 ? FB_POS : 0) | (cr < 0.0 ? FB_NEG : 0) | ((ult && cr != 0.0) ? FB_ULT : 0);
  if (quick) {
    const double a = d - 0.5 * cr, b = (1.0 - cr * cr) / 6.0;
    if (cr > 0.0) {
      f.wg = (float)(a - b * Ap);
      f.wa = (float)(-b * Bp);
    } else if (cr < 0.0) {
      f.wg = (float)(a + b * Bm);
      f.wa = (float)(-b * Am);
    } else {
      f.wg = (float)d;
      f.wa = 0.f;
    }
  } else {
    f.wa = (float)(cr > 0.0 ? 0.5 * (1.0 - cr) : 0.5 * (1.0 + cr));
    f.wg = 0.f;
  }
  const double ir = cr != 0.0 ? 1.0 / fabs(cr) : 0.0;
  f.ircr = (float)ir;
  f.U = U;
  f.V = U * ir;
  f.K = K;
}

// One face flux, every rounding explicit: the QUICKEST or Van Leer face value
// from the values tm2..tp1 at i-2..i+1 of the face's cell (FP32), then
// ULTIMATE, times the FP64 volume flux, minus the horizontal-diffusion term.
template <bool QUICK, bool ULT>
__device__ __forceinline__ double face(const Face &f, bool adv, bool hd, float tm2, float tm1,
                                       float t0, float tp1) {
  double flux = 0.0;
  if (adv) {
    const bool pos = (f.bits & FB_POS) != 0;
    const float tu = pos ? tm2 : tp1;
    float F;
    if (QUICK) {
      const float tc = pos ? tm1 : t0;
      F = __fmaf_rn(f.wa, __fsub_rn(tu, tc), __fmaf_rn(f.wg, __fsub_rn(t0, tm1), tm1));
    } else {
      const bool neg = (f.bits & FB_NEG) != 0;
      const float p = pos ? __fsub_rn(tm1, tm2) : __fsub_rn(t0, tm1);
      const float q = pos ? __fsub_rn(t0, tm1) : __fsub_rn(tp1, t0);
      const float den = pos ? __fsub_rn(t0, tm2) : __fsub_rn(tp1, tm1);
      const float pq = __fmul_rn(p, q);
      const float df = pq > 0.f ? __fmul_rn(2.f, __fdiv_rn(pq, den)) : 0.f;
      F = pos ? __fmaf_rn(f.wa, df, tm1) : (neg ? __fmaf_rn(-f.wa, df, t0) : 0.f);
    }
    if (ULT) {
      // ulimate_filter (tracers.c:3526-3554) without its divisions: with
      // s = sign(td - tu) and the normalised variables scaled back by
      // |td - tu|, nc in [0, 1] is 0 <= c <= d, nu > 1 is a > d, nu < nc is
      // a < c and nu > nc / |cr| is a > c / |cr|; tu + nc (td - tu) is tc.
      // Upwind and downwind values equal in FP32 (d = 0) limit to tc unless
      // tc equals them too: in FP64 they almost always differ by a few ulps
      // and the limiter falls back to upwind, so FP32 rounding of the stored
      // tracer does not flip the limiter's decision.
      const float tc = pos ? tm1 : t0, td = pos ? t0 : tm1;
      const float diff = __fsub_rn(td, tu);
      const float sg = diff < 0.f ? -1.f : 1.f;
      const float d = fabsf(diff);
      const float c = __fmul_rn(__fsub_rn(tc, tu), sg), a = __fmul_rn(__fsub_rn(F, tu), sg);
      const float q = __fmul_rn(c, f.ircr);
      float G = F;
      if (a > q) G = __fmaf_rn(sg, q, tu);
      if (a < c) G = tc;
      if (a > d) G = td;
      if (!(c >= 0.f && c <= d)) G = tc;
      // computed for every face and selected, so the faces of a cell stay
      // one straight-line block the compiler can interleave
      F = (f.bits & FB_ULT) ? G : F;
    }
    flux = __dmul_rn((double)F, f.U);
  }
  if (hd) flux = __dsub_rn(flux, (double)__fmul_rn(f.K, __fsub_rn(t0, tm1)));
  return flux;
}

// FP32_COMP face flux: face() on compensated values, each value the stored
// FP32 one (tm2..tp1) plus its compensation (lm2..lp1).  Differences are
// the stored difference plus the compensations' difference (FP32, accurate
// to their own size), so the limiter decides as on the FP64 values.  The face
// value is a base value (a stored value) plus a correction (its compensation
// and the FP32 increment), and the flux U (base + correction) in FP64; a face
// capped at ULTIMATE's Courant bound carries U (tu + lu) + V (tc - tu), the
// second term with the FP64 V.
template <bool QUICK, bool ULT>
__device__ __forceinline__ double face_c(const Face &f, bool adv, bool hd, float tm2, float tm1,
                                         float t0, float tp1, float lm2, float lm1, float l0,
                                         float lp1) {
  const bool pos = (f.bits & FB_POS) != 0;
  const float tu = pos ? tm2 : tp1, tc = pos ? tm1 : t0;
  const float lu = pos ? lm2 : lp1, lc = pos ? lm1 : l0;
  const float g01 = __fadd_rn(__fsub_rn(t0, tm1), __fsub_rn(l0, lm1));  // t0 - tm1
  const float dc = __fadd_rn(__fsub_rn(tc, tu), __fsub_rn(lc, lu));   // tc - tu
  float base, lbase, inc;
  if (QUICK) {
    inc = __fmaf_rn(f.wa, -dc, __fmul_rn(f.wg, g01));
    base = tm1;
    lbase = lm1;
  } else {
    const bool neg = (f.bits & FB_NEG) != 0;
    const float p = pos ? __fadd_rn(__fsub_rn(tm1, tm2), __fsub_rn(lm1, lm2)) : g01;
    const float q = pos ? g01 : __fadd_rn(__fsub_rn(tp1, t0), __fsub_rn(lp1, l0));
    const float den = pos ? __fadd_rn(__fsub_rn(t0, tm2), __fsub_rn(l0, lm2))
                          : __fadd_rn(__fsub_rn(tp1, tm1), __fsub_rn(lp1, lm1));
    const float pq = __fmul_rn(p, q);
    const float df = pq > 0.f ? __fmul_rn(2.f, __fdiv_rn(pq, den)) : 0.f;
    inc = pos ? __fmul_rn(f.wa, df) : (neg ? -__fmul_rn(f.wa, df) : 0.f);
    base = pos ? tm1 : (neg ? t0 : 0.f);
    lbase = pos ? lm1 : (neg ? l0 : 0.f);
  }
  // the face value as base + lb, and the capped face's difference dq
  float b = base, lb = __fadd_rn(lbase, inc), dq = 0.f;
  if (ULT) {
    const float td = pos ? t0 : tm1, ld = pos ? l0 : lm1;
    const float dd = __fadd_rn(__fsub_rn(td, tu), __fsub_rn(ld, lu));  // td - tu
    // F - tu: the base is tc, or td for QUICKEST with the flow negative
    const float dF = __fadd_rn((QUICK && !pos) ? dd : dc, inc);
    const float sg = dd < 0.f ? -1.f : 1.f;
    const float d = fabsf(dd), c = __fmul_rn(dc, sg), a = __fmul_rn(dF, sg);
    const float q = __fmul_rn(c, f.ircr);
    // the limiter's cases in the order that decides them: outside the
    // monotone range tc; above td td; below tc tc; above the cap the cap
    const bool lim = (f.bits & FB_ULT) != 0;
    const bool out = !(c >= 0.f && c <= d), above = a > d;
    const bool selc = lim && (out || (!above && a < c));
    const bool seld = lim && !out && above;
    const bool selq = lim && !out && !above && !(a < c) && a > q;
    b = selc ? tc : (seld ? td : (selq ? tu : b));
    lb = selc ? lc : (seld ? ld : (selq ? lu : lb));
    dq = selq ? dc : 0.f;
  }
  // U (b + lb) + V dq, V = U / |cr| (zero dq unless capped)
  double flux = adv ? __fma_rn(f.V, (double)dq, __dmul_rn(f.U, __dadd_rn((double)b, (double)lb)))
                    : 0.0;
  if (hd) flux = __dsub_rn(flux, (double)__fmul_rn(f.K, g01));
  return flux;
}

// Neumaier compensated sum; the explicitly rounded operations keep the
// compiler from contracting them when FMA contraction is on.
__device__ __forceinline__ void neumaier_add(double &s, double &comp, double v) {
  const double u = __dadd_rn(s, v);
  comp += (fabs(s) >= fabs(v)) ? __dadd_rn(__dsub_rn(s, u), v) : __dadd_rn(__dsub_rn(v, u), s);
  s = u;
}

}  // namespace f32

}  // namespace shoc
