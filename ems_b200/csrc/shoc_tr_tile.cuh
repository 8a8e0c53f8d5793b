// shoc_tr_tile.cuh -- the FP32-mixed transport kernels of the columns whose
// surface cell stays in its layer during the step (staged columns).
//
// One sub-step is two launches:
//
//  k_adv32  advection and horizontal diffusion (advect_diffuse, tracers.c:
//           849-925): one thread per wet cell, in SHOC's cell order (layer by
//           layer, i fastest), so a warp's cells are adjacent cells of one
//           layer and its loads coalesce.  The thread folds its cell's
//           tracer-independent face coefficients once (QUICKEST weights,
//           ULTIMATE 1/|cr|, volume flux, horizontal-diffusion factor) and
//           then loops over the advected tracers: the stencil values are
//           independent loads, the west-face flux of the next lane's cell is
//           this cell's east-face flux (shuffle), and every face a cell
//           computes for itself is rounded as its neighbour rounds it.  The
//           flux divergence and the new value are FP64.  Output, in the
//           destination tracer array (FP32): the new value of cells below
//           the surface, the horizontal flux divergence of the surface cell
//           and the cells above it; beside it, the FP32 rounding residual of
//           each of those values (value - stored, so stored + residual is the
//           FP64 value to 2^-48); the surface cell's bottom-face flux goes to
//           a per-(tracer, column) array.
//
//  k_vd32   one thread per (column, tracer): tr_bounds (tracers.c:3217-3324),
//           surf_conc's column-mass balance (:3097-3206, FP64 Neumaier), the
//           copy above the surface and, on the last sub-step, the implicit
//           vertical diffusion (implicit_vdiff_tr, :4067-4214) as an FP32
//           Thomas sweep, an FP64 residual and one FP32 correction solve,
//           with the column's FP64 mass carry (column_finish).  A block owns
//           32 columns of similar depth (a static depth-sorted column order)
//           so its lanes loop over similar layer ranges; the columns' values,
//           residuals, LU factors and FP64 thicknesses are staged into shared
//           memory in one batch of asynchronous copies.
//
// Mass carry.  Storing FP32 values loses mass at every rounding (and the
// FP32 solve conserves the column mass only to its residual).  Per (tracer,
// column) the kernels keep, in FP64, the mass the stored values owe the
// column: carry' = carry + M_exact - M_stored, where M_exact is the FP64 mass
// the sub-step computed (the FP64 advected values, the surf_conc surface
// value, tr_bounds' clipping) and M_stored the mass of what was stored.  The
// carry goes back into the column at the next sub-step as a uniform shift of
// its values (carry / (area x depth)), inside the solve's FP64 residual when
// there is a solve, so the stored values plus the carry conserve mass to
// FP64 round-off and the carry stays within a few FP32 ulps of the column
// mass.  The mass diagnostic adds it.  Columns whose surface moves during the
// step (eta != oldeta) keep their carry as it is.
//
// The cells of a column at every layer come from a static layer-by-column
// table, so no thread walks a column to find them.
#pragma once
#include "shoc_tr_stage.cuh"

namespace shoc {

// Static per-cell / per-layer tables of the tile kernels (built once at
// handle creation from the geometry maps).
struct Tile {
  const int *cellk;  // [nz][ncolp] cell of column col at layer k (0: none)
  const int4 *nb1;   // [S] xm1, xp1, ym1, yp1
  const int4 *nb2;   // [S] xm1(xm1), xp1(xp1), ym1(ym1), yp1(yp1)
  const int2 *m2e;   // [S] m2d(xp1), m2d(yp1)
  const uint8_t *fl; // [S] cflag(c) | xp1 wet, E1 | yp1 wet, E2 (FL_*)
  const int *kof;    // [S] layer index of each cell (s2k)
  const int4 *nbz;   // [S] zm1, zm1(zm1), zp1, zp1(zp1)
  const int *colof;  // [S] 0-based column of each wet cell
  const int *wet;    // [nwet] the wet cells (w3_t order)
  const int *vdcol;  // [ncolp] columns in k_vd32 order: whole tiles of 32
                     // adjacent columns, shallow tiles first (-1: padding)
  int nclass;        // k_vd32 depth classes: tiles [ctile[i], ctile[i+1]) have
  int ctile[5];      //   no cell below layer cbase[i]
  int cbase[4];
  const int4 *colrec;  // [ncolp] bottom cell, surface-layer cell, bottom layer
  int ncolp;         // columns rounded up to whole tiles
  int nwet;
};
constexpr int FL_XP_WET = 8, FL_XP_E1 = 16, FL_YP_WET = 32, FL_YP_E2 = 64;

// asynchronous global -> shared copies; a thread waits for its own copies
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The column `col` of a tile kernel: whether the tile kernels handle it this
// step (k_set_dz decides, COL_STAGED), its bottom and surface layers, 2D cell
// and bottom cell.  (The layer-by-column cell table agrees with the maps:
// handle creation checks every column's layers.)
struct TileCol {
  ColInfo ci;
  int cbot, c2, kb, ks;
  bool act;
};
__device__ __forceinline__ TileCol tile_column(const Geo &G, const Work &W, const Tile &Tl,
                                               int col) {
  TileCol t;
  t.ci = {0, 0, 0, 0, 0, 0};
  t.cbot = t.c2 = t.ks = 0;
  t.kb = G.nz;
  t.act = false;
  if (col >= 0 && col < G.ncol) {
    t.ci = W.col[col];
    const int4 r = Tl.colrec[col];
    if (t.ci.flags & COL_STAGED) {
      t.act = true;
      t.cbot = r.x;
      t.c2 = r.y;
      t.kb = r.z;
      t.ks = t.ci.ks;
    }
  }
  return t;
}

namespace f32 {

// Face coefficients of one horizontal face at a cell with the given flags
// (cr = u dt / h, rounded by the caller as __fmul_rn(__fmul_rn(u, dt), 1/h)).
__device__ __forceinline__ void hface(Face &f, bool wet, bool eb, bool quick, bool ult,
                                      float cr, double U, float K, const Face2 &m) {
  if (!wet) {  // a ghost: the face carries nothing
    face_zero(f);
    return;
  }
  if (!quick && !eb) {  // Van Leer advects interior faces only
    face_zero(f);
    f.K = K;
    return;
  }
  set_face(f, quick, cr, m.d, m.Ap, m.Bp, m.Am, m.Bm, U, ult && eb, K);
}

// Vertical face at the bottom of a cell from the thicknesses of the two cells
// below it (dzm2, dzm1), the cell (dz0) and the one above (dzp1; the
// surface-layer cell maps onto itself, top != 0), and w * dtu (wv in FP32
// for the Courant number, U in FP64 for the flux); IEEE divisions, so the
// cell below folds its top face to the same bits.
__device__ __forceinline__ void zface(Face &f, bool quick, bool ult, float dzm2, float dzm1,
                                      float dz0, float dzp1, bool top, float wv, double U) {
  const float w9m = __fmul_rn(0.5f, __fadd_rn(dzm1, dzm2));
  const float w90 = __fmul_rn(0.5f, __fadd_rn(dz0, dzm1));
  const float w9p = top ? w90 : __fmul_rn(0.5f, __fadd_rn(dzp1, dz0));
  const float cz = __fdiv_rn(wv, w90);
  const float db = __fdiv_rn(2.f, __fadd_rn(w9m, w90)), df = __fdiv_rn(2.f, __fadd_rn(w90, w9p));
  set_face(f, quick, cz, __fdiv_rn(dzm1, __fadd_rn(dzm1, dz0)), __fmul_rn(db, w9m),
           __fmul_rn(db, w90), __fmul_rn(df, w90), __fmul_rn(df, w9p), U, ult, 0.f);
}

}  // namespace f32

// ---------------------------------------------------------------------------
// k_adv32

constexpr int kAdvBlock = 256;     // k_adv64
// k_adv32: 128 threads, 5 blocks per SM (at most 102 registers a thread: 20
// warps per SM where 256-thread blocks fit 16; measured 13.0 ms against 14.3
// on stiff2048)
constexpr int kAdv32Block = 128, kAdv32MinBlocks = 5;
constexpr int kAdvGroup = 1;       // tracers whose loads a thread issues together
// dynamic shared memory of k_adv32 with uniform flags: the double-buffered
// stencil values of a group of tracers per thread
constexpr size_t kAdvSmem = (size_t)2 * kAdvGroup * 13 * kAdv32Block * sizeof(float);
constexpr int kMaxTracers = 256;   // tracers a handle of the FP32-mixed path may carry

// MODE: 0 tracers with their own advect / diffuse flags, 1 every advected
// tracer advected without horizontal diffusion, 2 advected with it.
// COMP (FP32_COMP): faces set up in FP64 (set_face64) and every stencil
// value read with its compensation from loi (face_c); 4 blocks per SM.
template <bool QUICK, bool ULT, int MODE, bool COMP>
__global__ void __launch_bounds__(kAdv32Block, COMP ? 4 : kAdv32MinBlocks) k_adv32(Geo G, Flow32 F3, Work W, TrSet T,
                                                     SubStep ss, Tile Tl,
                                                     const f32::Face2 *__restrict__ fx2,
                                                     const f32::Face2 *__restrict__ fy2,
                                                     const float *__restrict__ tri,
                                                     float *__restrict__ tro,
                                                     float *__restrict__ rso,
                                                     double *__restrict__ fzs, int any_hd,
                                                     const int16_t *__restrict__ loi) {
  using namespace f32;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ int sTr[kMaxTracers], sTf[kMaxTracers];
  const int i = blockIdx.x * kAdv32Block + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int nz = G.nz;
  for (int s = threadIdx.x; s < T.ntb; s += kAdv32Block) {
    const int n = T.slot_tr[s];
    sTr[s] = n;
    sTf[s] = T.trf[n];
  }
  __syncthreads();

  // this thread's cell and its column (ntc: tracers carried by the column)
  int c = 0, col = 0, kb = nz, ks = 0, k = 0, c2 = 0, ntc = 0;
  if (i < Tl.nwet) {
    c = Tl.wet[i];
    col = Tl.colof[c];
    k = Tl.kof[c];
    const TileCol tc = tile_column(G, W, Tl, col);
    if (tc.act) {
      kb = tc.kb;
      ks = tc.ks;
      c2 = tc.c2;
      ntc = G.colntr[col];
    } else {
      c = 0;
    }
  }
  const bool on = c != 0;
  int4 n1 = make_int4(0, 0, 0, 0), n2 = n1, nzv = n1;
  int2 me = make_int2(0, 0);
  int fl = 0;
  if (on) {
    n1 = Tl.nb1[c];
    n2 = Tl.nb2[c];
    nzv = Tl.nbz[c];
    me = Tl.m2e[c];
    fl = Tl.fl[c];
  }
  // x-neighbours that are the cells of neighbouring lanes
  const int cu1 = __shfl_up_sync(FULL, c, 1), cu2 = __shfl_up_sync(FULL, c, 2);
  const int cd1 = __shfl_down_sync(FULL, c, 1), cd2 = __shfl_down_sync(FULL, c, 2);
  const bool sxm1 = on && lane >= 1 && cu1 && n1.x == cu1;
  const bool sxm2 = on && lane >= 2 && cu2 && n2.x == cu2;
  const bool sxp1 = on && lane <= 30 && cd1 && n1.y == cd1;
  const bool sxp2 = on && lane <= 29 && cd2 && n2.y == cd2;

  // tracer-independent face coefficients
  const double dtu = ss.dtu;
  const float fdtu = (float)dtu;
  const bool hdf = any_hd != 0;
  Face fw, fs, fn, fe, fzb, fzt;
  face_zero(fw);
  face_zero(fs);
  face_zero(fn);
  face_zero(fe);
  face_zero(fzb);
  face_zero(fzt);
  double idz = 0.0, ia = 0.0;
  if (on && COMP) {
    // FP64 Courant numbers (tracers.c:730-736) and metric factors
    auto hset = [&](Face &f, bool wet, bool eb, double u, double h, const Face2D &m, double U,
                    float K) {
      if (!wet) {
        face_zero(f);
      } else if (!QUICK && !eb) {  // Van Leer advects interior faces only
        face_zero(f);
        f.K = K;
      } else {
        set_face64(f, QUICK, u * dtu / h, m.d, m.db * m.hm, m.db * m.h0, m.df * m.h0,
                   m.df * m.hp, U, ULT && eb, K);
      }
    };
    // the face at the bottom of cell cc (below it zm, above it zp), from the
    // work arrays as quickest_zface takes them
    auto zset = [&](Face &f, int cc, int zm, int zp) {
      const double w90 = W.w9[cc];
      set_face64(f, QUICK, F3.w64[cc] * dtu / (w90 * 1.0), W.w5[cc], W.dbz[cc] * W.w9[zm],
                 W.dbz[cc] * w90, W.dfz[cc] * w90, W.dfz[cc] * W.w9[zp],
                 __dmul_rn(F3.w64[cc], dtu), ULT, 0.f);
    };
    hset(fw, fl & CF_WET, fl & CF_E1, F3.u1_64[c], G.h1au1[c2], G.fx[c2], F3.u1flux3d[c],
         hdf ? F3.khx[c] : 0.f);
    hset(fs, fl & CF_WET, fl & CF_E2, F3.u2_64[c], G.h2au2[c2], G.fy[c2], F3.u2flux3d[c],
         hdf ? F3.khy[c] : 0.f);
    if (fl & FL_YP_WET) {
      const int yp = n1.w;
      hset(fn, true, fl & FL_YP_E2, F3.u2_64[yp], G.h2au2[me.y], G.fy[me.y], F3.u2flux3d[yp],
           hdf ? F3.khy[yp] : 0.f);
    }
    if (!sxp1 && (fl & FL_XP_WET)) {
      const int xp = n1.y;
      hset(fe, true, fl & FL_XP_E1, F3.u1_64[xp], G.h1au1[me.x], G.fx[me.x], F3.u1flux3d[xp],
           hdf ? F3.khx[xp] : 0.f);
    }
    if (k <= ks) {
      zset(fzb, c, nzv.x, nzv.z);
      if (k < ks) zset(fzt, nzv.z, c, nzv.w);  // the bottom face of the cell above
    }
    idz = 1.0 / W.dz[c];
    ia = 1.0 / G.cellarea[c2];
  } else if (on) {
    const Face2 mx = fx2[c2], my = fy2[c2];
    hface(fw, fl & CF_WET, fl & CF_E1, QUICK, ULT, __fmul_rn(__fmul_rn(F3.u1[c], fdtu), mx.ih),
          F3.u1flux3d[c], hdf ? F3.khx[c] : 0.f, mx);
    hface(fs, fl & CF_WET, fl & CF_E2, QUICK, ULT, __fmul_rn(__fmul_rn(F3.u2[c], fdtu), my.ih),
          F3.u2flux3d[c], hdf ? F3.khy[c] : 0.f, my);
    if (fl & FL_YP_WET) {
      const int yp = n1.w;
      const Face2 mn = fy2[me.y];
      hface(fn, true, fl & FL_YP_E2, QUICK, ULT, __fmul_rn(__fmul_rn(F3.u2[yp], fdtu), mn.ih),
            F3.u2flux3d[yp], hdf ? F3.khy[yp] : 0.f, mn);
    }
    if (!sxp1 && (fl & FL_XP_WET)) {
      const int xp = n1.y;
      const Face2 mxe = fx2[me.x];
      hface(fe, true, fl & FL_XP_E1, QUICK, ULT, __fmul_rn(__fmul_rn(F3.u1[xp], fdtu), mxe.ih),
            F3.u1flux3d[xp], hdf ? F3.khx[xp] : 0.f, mxe);
    }
    const float dz0 = W.dz32[c];
    if (k <= ks) {
      // thicknesses below, at and above the cell (the sediment has none, the
      // surface-layer cell maps onto itself)
      const float dzm1 = W.dz32[nzv.x], dzm2 = W.dz32[nzv.y];
      const bool top = (nzv.z == c);
      const float dzp1 = W.dz32[nzv.z];
      zface(fzb, QUICK, ULT, dzm2, dzm1, dz0, dzp1, top, __fmul_rn(F3.w[c], fdtu),
            __dmul_rn(F3.w64[c], dtu));
      if (k < ks) {  // the bottom face of the cell above
        const bool top1 = (nzv.w == nzv.z);
        const float dzp2 = W.dz32[nzv.w];
        zface(fzt, QUICK, ULT, dzm1, dz0, dzp1, dzp2, top1, __fmul_rn(F3.w[nzv.z], fdtu),
              __dmul_rn(F3.w64[nzv.z], dtu));
      }
    }
    idz = 1.0 / W.dz[c];  // the FP64 thickness: the update conserves mass to FP64 round-off
    ia = 1.0 / G.cellarea[c2];
  }
  // vertical neighbours (bottom: the sediment ghost holds the bottom value,
  // tracers.c:827-830)
  const int vm1 = (k - 1 >= kb) ? nzv.x : c;
  const int vm2 = (k - 2 >= kb) ? nzv.y : vm1;
  const int vp1 = nzv.z, vp2 = nzv.w;
  const bool zf = k <= ks, zt = k < ks;
  const int ntb = T.ntb;

  // The advected tracers in groups of U: every stencil value of the group is
  // loaded before any of it is used, so a thread has U tracers' loads in
  // flight at once.
  constexpr int U = kAdvGroup;
  if constexpr (MODE != 0) {
    // uniform flags: every stencil value is loaded (threads without a cell,
    // and neighbours a cell does not use, read valid cells) and the face
    // code has no per-tracer branches
    constexpr bool HD = MODE == 2;
    constexpr int NQ = 13;
    const int idx[NQ] = {c,    n1.z, n2.z, n1.w, n2.w, vm1, vm2,
                         vp1,  vp2,  n1.x, n2.x, n1.y, n2.y};
    // the stencil values of the next group of tracers are copied into this
    // thread's slots of a double buffer while the current group is computed
    extern __shared__ float pf[];  // [2][U][NQ][kAdv32Block]
    auto issue = [&](int s0, int buf) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int s = s0 + u < ntb ? s0 + u : s0;
        const float *tr = tri + (size_t)sTr[s] * G.S;
        float *d = pf + (buf * U + u) * NQ * kAdv32Block + threadIdx.x;
#pragma unroll
        for (int q = 0; q < NQ; ++q) cp_async4(d + q * kAdv32Block, tr + idx[q]);
      }
      cp_async_commit();
    };
    issue(0, 0);
    static_assert(U == 1, "the compensations are loaded for one tracer at a time");
    for (int s0 = 0, g = 0; s0 < ntb; s0 += U, ++g) {
      // COMP: the stencil's compensations, in flight while the stencil
      // values' copies complete
      int16_t lq[NQ];
      if constexpr (COMP) {
        const int16_t *Lp = loi + (size_t)sTr[s0] * G.S;
#pragma unroll
        for (int q = 0; q < NQ; ++q) lq[q] = Lp[idx[q]];
      }
      if (s0 + U < ntb) {
        issue(s0 + U, (g + 1) & 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      // tracers are ascending when columns carry different numbers of them
      if (!__any_sync(FULL, on && sTr[s0] < ntc)) continue;
      const float *P = pf + (g & 1) * U * NQ * kAdv32Block + threadIdx.x;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int s = s0 + u;
        if (s >= ntb) break;
        const float *v = P + u * NQ * kAdv32Block;
        const float t0 = v[0];
        const float tym1 = v[1 * kAdv32Block], tym2 = v[2 * kAdv32Block];
        const float typ1 = v[3 * kAdv32Block], typ2 = v[4 * kAdv32Block];
        const float tm1 = v[5 * kAdv32Block], tm2 = v[6 * kAdv32Block];
        const float tp1 = v[7 * kAdv32Block], tp2 = v[8 * kAdv32Block];
        const float txm1 = v[9 * kAdv32Block], txm2 = v[10 * kAdv32Block];
        const float txp1 = v[11 * kAdv32Block], txp2 = v[12 * kAdv32Block];
        double Fxw, Fys, Fyn, Fxe, Fzb;
        float l0 = 0.f, lm1 = 0.f, lm2 = 0.f, lp1 = 0.f, lp2 = 0.f;
        if constexpr (COMP) {
          l0 = lo_val(lq[0]);
          const float lym1 = lo_val(lq[1]), lym2 = lo_val(lq[2]);
          const float lyp1 = lo_val(lq[3]), lyp2 = lo_val(lq[4]);
          lm1 = lo_val(lq[5]);
          lm2 = lo_val(lq[6]);
          lp1 = lo_val(lq[7]);
          lp2 = lo_val(lq[8]);
          const float lxm1 = lo_val(lq[9]), lxm2 = lo_val(lq[10]);
          const float lxp1 = lo_val(lq[11]), lxp2 = lo_val(lq[12]);
          Fxw = face_c<QUICK, ULT>(fw, true, HD, txm2, txm1, t0, txp1, lxm2, lxm1, l0, lxp1);
          Fys = face_c<QUICK, ULT>(fs, true, HD, tym2, tym1, t0, typ1, lym2, lym1, l0, lyp1);
          Fyn = face_c<QUICK, ULT>(fn, true, HD, tym1, t0, typ1, typ2, lym1, l0, lyp1, lyp2);
          const double Fnext = __shfl_down_sync(FULL, Fxw, 1);
          Fxe = sxp1 ? Fnext
                     : face_c<QUICK, ULT>(fe, true, HD, txm1, t0, txp1, txp2, lxm1, l0, lxp1,
                                          lxp2);
          Fzb = zf ? face_c<QUICK, ULT>(fzb, true, false, tm2, tm1, t0, tp1, lm2, lm1, l0, lp1)
                   : 0.0;
        } else {
          Fxw = face<QUICK, ULT>(fw, true, HD, txm2, txm1, t0, txp1);
          Fys = face<QUICK, ULT>(fs, true, HD, tym2, tym1, t0, typ1);
          Fyn = face<QUICK, ULT>(fn, true, HD, tym1, t0, typ1, typ2);
          const double Fnext = __shfl_down_sync(FULL, Fxw, 1);
          Fxe = sxp1 ? Fnext : face<QUICK, ULT>(fe, true, HD, txm1, t0, txp1, txp2);
          Fzb = zf ? face<QUICK, ULT>(fzb, true, false, tm2, tm1, t0, tp1) : 0.0;
        }
        const int n = sTr[s];
        if (!on || n >= ntc) continue;
        // FP64 flux divergence (tracers.c:888-892)
        const double dtr = ((Fxe - Fxw) + (Fyn - Fys)) * dtu;
        double a = dtr;
        if (zt) {
          const double Fzt =
              COMP ? face_c<QUICK, ULT>(fzt, true, false, tm1, t0, tp1, tp2, lm1, l0, lp1, lp2)
                   : face<QUICK, ULT>(fzt, true, false, tm1, t0, tp1, tp2);
          const double t0d = COMP ? (double)t0 + (double)l0 : (double)t0;
          a = t0d - (dtr * ia + (Fzt - Fzb)) * idz;
        } else if (zf) {
          fzs[(size_t)n * G.ncol + col] = Fzb;
        }
        const float val = (float)a;
        tro[(size_t)n * G.S + c] = val;
        rso[(size_t)n * G.S + c] = (float)(a - (double)val);
      }
    }
  } else {
  for (int s0 = 0; s0 < ntb; s0 += U) {
    float v[U][13];  // t0, y-2..y+2, z-2..z+2, x-2..x+2 (off-tile x only)
    float lv[U][13];  // COMP: their compensations (x-neighbours read for every cell)
    int nn[U], tf[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int s = s0 + u;
      nn[u] = s < ntb ? sTr[s] : 0;
      tf[u] = s < ntb ? sTf[s] : 0;
      const float *__restrict__ tr = tri + (size_t)nn[u] * G.S;
      const bool hor = on && (tf[u] & (TR_ADV | TR_HDIFF));
      const bool vz = on && (tf[u] & TR_ADV) && zf;
      v[u][0] = on && s < ntb ? tr[c] : 0.f;
      v[u][1] = hor ? tr[n1.z] : 0.f;
      v[u][2] = hor ? tr[n2.z] : 0.f;
      v[u][3] = hor ? tr[n1.w] : 0.f;
      v[u][4] = hor ? tr[n2.w] : 0.f;
      v[u][5] = vz ? tr[vm1] : 0.f;
      v[u][6] = vz ? tr[vm2] : 0.f;
      v[u][7] = vz ? tr[vp1] : 0.f;
      v[u][8] = (vz && zt) ? tr[vp2] : 0.f;
      v[u][9] = (hor && !sxm1) ? tr[n1.x] : 0.f;
      v[u][10] = (hor && !sxm2) ? tr[n2.x] : 0.f;
      v[u][11] = (hor && !sxp1) ? tr[n1.y] : 0.f;
      v[u][12] = (hor && !sxp1 && !sxp2) ? tr[n2.y] : 0.f;
      if constexpr (COMP) {
        const int16_t *L = loi + (size_t)nn[u] * G.S;
        lv[u][0] = on && s < ntb ? lo_val(L[c]) : 0.f;
        lv[u][1] = hor ? lo_val(L[n1.z]) : 0.f;
        lv[u][2] = hor ? lo_val(L[n2.z]) : 0.f;
        lv[u][3] = hor ? lo_val(L[n1.w]) : 0.f;
        lv[u][4] = hor ? lo_val(L[n2.w]) : 0.f;
        lv[u][5] = vz ? lo_val(L[vm1]) : 0.f;
        lv[u][6] = vz ? lo_val(L[vm2]) : 0.f;
        lv[u][7] = vz ? lo_val(L[vp1]) : 0.f;
        lv[u][8] = (vz && zt) ? lo_val(L[vp2]) : 0.f;
        lv[u][9] = hor ? lo_val(L[n1.x]) : 0.f;
        lv[u][10] = hor ? lo_val(L[n2.x]) : 0.f;
        lv[u][11] = hor ? lo_val(L[n1.y]) : 0.f;
        lv[u][12] = hor ? lo_val(L[n2.y]) : 0.f;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int s = s0 + u;
      if (s >= ntb) break;
      const bool adv = (tf[u] & TR_ADV) != 0, hd = (tf[u] & TR_HDIFF) != 0;
      const float t0 = v[u][0];
      const float u1v = __shfl_up_sync(FULL, t0, 1), u2v = __shfl_up_sync(FULL, t0, 2);
      const float d1v = __shfl_down_sync(FULL, t0, 1), d2v = __shfl_down_sync(FULL, t0, 2);
      double Fxw = 0.0, Fxe = 0.0, Fys = 0.0, Fyn = 0.0, Fzb = 0.0, Fzt = 0.0;
      if (on && (adv || hd)) {
        const float txm1 = sxm1 ? u1v : v[u][9];
        const float txm2 = sxm2 ? u2v : v[u][10];
        const float txp1 = sxp1 ? d1v : v[u][11];
        const float tym1 = v[u][1], tym2 = v[u][2], typ1 = v[u][3], typ2 = v[u][4];
        if constexpr (COMP) {
          const float *l = lv[u];
          Fxw = face_c<QUICK, ULT>(fw, adv, hd, txm2, txm1, t0, txp1, l[10], l[9], l[0], l[11]);
          Fys = face_c<QUICK, ULT>(fs, adv, hd, tym2, tym1, t0, typ1, l[2], l[1], l[0], l[3]);
          Fyn = face_c<QUICK, ULT>(fn, adv, hd, tym1, t0, typ1, typ2, l[1], l[0], l[3], l[4]);
          if (!sxp1) {
            const float txp2 = sxp2 ? d2v : v[u][12];
            Fxe = face_c<QUICK, ULT>(fe, adv, hd, txm1, t0, txp1, txp2, l[9], l[0], l[11],
                                     l[12]);
          }
          if (adv && zf) {
            const float tm1 = v[u][5], tm2 = v[u][6], tp1 = v[u][7];
            Fzb = face_c<QUICK, ULT>(fzb, true, false, tm2, tm1, t0, tp1, l[6], l[5], l[0],
                                     l[7]);
            if (zt)
              Fzt = face_c<QUICK, ULT>(fzt, true, false, tm1, t0, tp1, v[u][8], l[5], l[0],
                                       l[7], l[8]);
          }
        } else {
          Fxw = face<QUICK, ULT>(fw, adv, hd, txm2, txm1, t0, txp1);
          Fys = face<QUICK, ULT>(fs, adv, hd, tym2, tym1, t0, typ1);
          Fyn = face<QUICK, ULT>(fn, adv, hd, tym1, t0, typ1, typ2);
          if (!sxp1) {
            const float txp2 = sxp2 ? d2v : v[u][12];
            Fxe = face<QUICK, ULT>(fe, adv, hd, txm1, t0, txp1, txp2);
          }
          if (adv && zf) {
            const float tm1 = v[u][5], tm2 = v[u][6], tp1 = v[u][7];
            Fzb = face<QUICK, ULT>(fzb, true, false, tm2, tm1, t0, tp1);
            if (zt) Fzt = face<QUICK, ULT>(fzt, true, false, tm1, t0, tp1, v[u][8]);
          }
        }
      }
      const double Fnext = __shfl_down_sync(FULL, Fxw, 1);
      if (!on || nn[u] >= ntc) continue;
      if (sxp1) Fxe = Fnext;
      // FP64 flux divergence (tracers.c:888-892)
      const double dtr = ((Fxe - Fxw) + (Fyn - Fys)) * dtu;
      double a = dtr;
      if (zt) {
        const double t0d = COMP ? (double)t0 + (double)lv[u][0] : (double)t0;
        a = t0d - (dtr * ia + (Fzt - Fzb)) * idz;
      }
      else if (k == ks)
        fzs[(size_t)nn[u] * G.ncol + col] = Fzb;
      const float val = (float)a;
      tro[(size_t)nn[u] * G.S + c] = val;
      rso[(size_t)nn[u] * G.S + c] = (float)(a - (double)val);
    }
  }
  }
}

// ---------------------------------------------------------------------------
// column_finish: the end of an FP32-mixed sub-step for one (column, tracer),
// shared by k_vd32 and the fused k_step32.

// Advected tracers' column sums from the advection: the FP64 mass of the
// advected values below the surface (sum of a dz), the FP64 horizontal
// divergence of the surface cell and the cells above it, and the surface
// cell's bottom-face flux.
struct ColSums {
  double m, dv, fzb;
};

// A0, S0: the column's values and Thomas storage from its bottom layer up, row
// stride sa; an advected tracer (tbdy) holds its advected values below the
// surface, any other tracer every layer's old value (A0 is overwritten, so is
// S0).  L0, C0, D0: LU factors, cells and FP64 thicknesses, row stride 32.
// RES: an advected tracer's A0 holds every layer's stored advection result
// and S0 its rounding residual (k_vd32), and the column sums cs.m and cs.dv
// are taken from them; else they come in cs (k_step32).
// carry: [ntr][ncol] (null: none).  Adds the values it flags to nwarn and
// sets bad for a NaN among what it stores.  The mass bookkeeping sums are
// plain FP64 sums of at most nz terms: their rounding (a few 1e-16 of the
// column mass, of either sign) is what the carry may miss per step.
template <bool LAST, bool RES>
__device__ __forceinline__ void column_finish(const Geo &G, const Flow &F, const Work &W,
                                              const Opt &O, const TrSet &T, const SubStep &ss,
                                              const TileCol &tc, int col, int n, bool tbdy,
                                              bool adv, bool vdf, float *A0, float *S0, int sa,
                                              const float4 *L0, const int *C0, const double *D0,
                                              const float *tr, float *to, double area, double ia,
                                              double idt, ColSums cs,
                                              double *carry, bool steady, long long &nwarn,
                                              bool &bad, int16_t *R0 = nullptr,
                                              const int16_t *li = nullptr,
                                              int16_t *lout = nullptr) {
  // FP32_COMP (R0, li, lout non-null): R0 keeps each row's value - stored
  // (the advection's rounding residual, or the old value's compensation) in
  // the compensation's format for the solve's residual and the final value;
  // li is the tracer's compensation on the way in, lout on the way out
  const ColInfo &ci = tc.ci;
  const int kb = tc.kb, nz = G.nz, c2 = tc.c2;
  const int nk = tc.ks - kb;  // cells below the surface cell
  const bool single = (ci.flags & COL_SINGLE) != 0;
  const bool solve = vdf && !single;
  const double mn = T.mintr[n], mx = T.maxtr[n];
  const double dzs_old = (double)W.dz32[ci.s];
  // surface value before the sub-step
  const double ts_old = (double)tr[ci.s] + (li ? lo_dec(li[ci.s], tr[ci.s]) : 0.0);
  const double dzs = D0[nk * 32];
  // FP64 mass bookkeeping per unit area: what the step computed (mxs) and
  // what is stored (mss)
  double mxs = 0.0, mss = 0.0;
  long long nw = 0;
  double vs = ts_old;  // the surface value
  double H = dzs;      // the water depth the carry is spread over
  // tr_bounds clip and range check (:3278-3293) of the cells below the
  // surface (advected tracers); a < mn and a > mx of a float a, exactly, as
  // float compares
  const float mnf = (float)mn, mn_up = __double2float_ru(mn), mx_dn = __double2float_rd(mx);
  const bool clip = tbdy && mn <= kClipEps;
  if (RES && tbdy) {  // the divergence at and above the surface: stored + residual
    double dv = 0.0;
    for (int j = nk; j < nz - kb; ++j) dv += (double)A0[j * sa] + (double)S0[j * sa];
    cs.dv = dv;
  }
  if (!tbdy) {
    vs = (double)A0[nk * sa];
    if (li) vs += lo_dec(li[C0[nk * 32]], A0[nk * sa]);
    for (int j = nk + 1; j < nz - kb; ++j) {
      to[C0[j * 32]] = A0[j * sa];
      if (lout) lout[C0[j * 32]] = li[C0[j * 32]];
      bad |= isnan(A0[j * sa]);
    }
  }
  // one pass up the column below the surface: the computed mass (an
  // advected tracer's FP64 values are stored + residual, or come in cs.m),
  // the clip, the depth and, with a solve, the FP32 forward sweep
  float fwd = 0.f;  // the bottom row's cm1 is 0
  double m = 0.0;
  for (int j = 0; j < nk; ++j) {
    float a = A0[j * sa];
    const double dz = D0[j * 32];
    H += dz;
    // the row's value - stored: the advection's rounding residual, or the
    // old value's compensation
    double r = 0.0;
    if (tbdy && RES) r = (double)S0[j * sa];
    else if (!tbdy && li) r = lo_dec(li[C0[j * 32]], a);
    if (!tbdy || RES) m += ((double)a + r) * dz;
    if (clip && a < mn_up) {
      mxs += ((double)mnf - ((double)a + r)) * dz;
      a = mnf;
      r = 0.0;
    }
    if (R0) R0[j * sa] = lo_bits((float)r);
    if (tbdy) {
      nw += (a < mn_up || a > mx_dn);
      A0[j * sa] = a;
    }
    if (solve) {
      const float4 lu = L0[j * 32];
      fwd = (lu.x * a - lu.y * fwd) * lu.z;
      S0[j * sa] = fwd;
    }
  }
  mxs += (tbdy && !RES) ? cs.m : m;
  if (tbdy) {
    const double a_below =
        nk > 0 ? (double)A0[(nk - 1) * sa] + (R0 ? (double)lo_val(R0[(nk - 1) * sa]) : 0.0)
               : 0.0;
    // surf_conc with s == co (tracers.c:3097-3206): column mass in FP64
    if (adv) {
      const double wb = (ci.s == tc.cbot) ? G.botz[c2] : G.gridz[ci.s];
      const double eta = F.eta[c2], oe = F.oldeta[c2];
      const double osub = ss.first ? oe : oe + ss.osub_f * (eta - oe);
      const double sub = oe + ss.subeta_f * (eta - oe);
      double ssum = 0.0, scomp = 0.0;
      f32::neumaier_add(ssum, scomp, __dmul_rn(cs.fzb, area));
      f32::neumaier_add(ssum, scomp, __dmul_rn(__dmul_rn(ts_old, area), osub - wb));
      f32::neumaier_add(ssum, scomp, -cs.dv);
      const double dzn = sub - wb;
      const double svol = dzn * area;
      const double st = ssum + scomp;
      const double sv = (svol == 0.0 || (st < 0.0 && dzn <= O.hmin)) ? 0.0 : st / svol;
      vs = (G.botz[c2] > 0.0 && dzs_old < O.hmin) ? ts_old : sv;
    }
    if ((ci.flags & COL_THIN) && (vs < mn || vs > mx)) vs = a_below;
    if (mn <= kClipEps && vs < mn) vs = mn;
    if (vs < mn || vs > mx) ++nw;
    bad |= isnan(vs);
    const float vs32 = (float)vs;
    const int16_t qs = lout ? lo_enc(vs, vs32) : (int16_t)0;
    for (int j = nk + 1; j < nz - kb; ++j) {
      to[C0[j * 32]] = vs32;
      if (lout) lout[C0[j * 32]] = qs;
    }
  }
  mxs += vs * dzs;
  const double carry_in = (carry && steady) ? carry[(size_t)n * G.ncol + col] : 0.0;
  // the carry goes back as a uniform shift of the column's values
  const double dl = H > 0.0 ? carry_in * ia / H : 0.0;
  if (H > 0.0) mxs += carry_in * ia;
  // stores one final value: FP32 (and, FP32_COMP, its compensation); adds
  // what is stored to the stored mass
  auto store = [&](int c, double v, double dz) {
    const float fin = (float)v;
    to[c] = fin;
    bad |= isnan(fin);
    double st = (double)fin;
    if (lout) {
      double dec;
      lout[c] = lo_round(v, fin, dec);
      st += dec;
    }
    mss += st * dz;
  };
  if (!solve) {
    // the values as they are, plus the carry's shift (tr_bounds has run)
    for (int j = 0; j < nk; ++j)
      store(C0[j * 32], (double)A0[j * sa] + (R0 ? (double)lo_val(R0[j * sa]) : 0.0) + dl,
            D0[j * 32]);
    const double h = dzs_old > O.hmin ? dzs_old : O.hmin;
    store(ci.s, (vdf && single) ? vs + dl + F.dt * (0.0 - 0.0) / h : vs + dl, dzs);
  } else {
    // the surface row of the forward sweep
    {
      const float4 lu = L0[nk * 32];
      A0[nk * sa] = (float)vs;
      fwd = (lu.x * (float)vs - lu.y * fwd) * lu.z;
      S0[nk * sa] = fwd;
    }
    // back substitution (FP32), x(j) replacing s(j), and one row behind it
    // the FP64 residual of b - A x for A = dz/dt I + the diffusion operator,
    //   r(j) = dz/dt (a + dl - x) - cm1 (x(j-1) - x) - cp1 (x(j+1) - x)
    // (cp1(j) = cm1(j+1); the bottom row has no cm1 term, the top row no cp1
    // term), which replaces a(j).  Its diagonal is the FP64 dz / dt, so the
    // refined solve keeps the column mass the mass diagnostic measures; cm1
    // is the FP32 factor's (the FP64 one, staged as well, changed neither
    // the maximum nor the RMS error over 1000 stiff2048 steps, and its
    // shared memory cost warps).  The FP64 copies of x and of the factors are
    // carried from row to row.
    float x1 = fwd;
    float4 l1 = L0[nk * 32];
    double xd1 = (double)x1, xd2 = 0.0, l2y = 0.0;
    double dzdt1 = dzs * idt;
    for (int j = nk - 1; j >= 0; --j) {
      const float x = S0[j * sa] - l1.w * x1;
      S0[j * sa] = x;
      const double xd = (double)x, l1y = (double)l1.y;
      const double aj1 =
          ((j + 1 == nk) ? vs
                         : (double)A0[(j + 1) * sa] +
                               (R0 ? (double)lo_val(R0[(j + 1) * sa]) : 0.0)) +
          dl;
      double r = dzdt1 * (aj1 - xd1) - l1y * (xd - xd1);
      if (j + 1 < nk) r = r - l2y * (xd2 - xd1);
      A0[(j + 1) * sa] = (float)r;
      x1 = x;
      xd2 = xd1;
      xd1 = xd;
      l2y = l1y;
      l1 = L0[j * 32];
      dzdt1 = D0[j * 32] * idt;
    }
    {
      const double a0 =
          ((nk == 0) ? vs : (double)A0[0] + (R0 ? (double)lo_val(R0[0]) : 0.0)) + dl;
      double r = dzdt1 * (a0 - xd1);
      if (nk > 0) r = r - l2y * (xd2 - xd1);
      A0[0] = (float)r;
    }
    // correction solve (FP32 forward and back) and the update in FP64
    float u = 0.f;
    for (int j = 0; j <= nk; ++j) {
      const float4 lu = L0[j * 32];
      u = (A0[j * sa] - lu.y * u) * lu.z;
      A0[j * sa] = u;
    }
    float d = A0[nk * sa];
    store(C0[nk * 32], (double)S0[nk * sa] + (double)d, dzs);
    for (int j = nk - 1; j >= 0; --j) {
      d = A0[j * sa] - L0[(j + 1) * 32].w * d;
      store(C0[j * 32], (double)S0[j * sa] + (double)d, D0[j * 32]);
    }
  }
  if (carry && steady) carry[(size_t)n * G.ncol + col] = (mxs - mss) * area;
  nwarn += nw;
}

// ---------------------------------------------------------------------------
// k_vd32

// k_vd32: a block is one tile of 32 columns and nw warps (at most
// kVd32MaxWarps); the tile's tracer-independent column arrays are staged
// once and each warp steps its share of the tracers through them (PF: with
// the next tracer's column staged while the current one is solved).
constexpr int kVd32MaxWarps = 16;
// shared memory of k_vd32 (bytes) for columns of at most nd layers:
// LU float4[nd][32], thicknesses double[nd][32], colC int[nd][32], A, S
// float[nd][nw][32] (twice with pf: the next tracer's column is staged
// while the current one is solved), with comp (FP32_COMP) R, compensations
// int16[nd][nw][32]
inline size_t vd32_smem(int nd, int nw, bool pf = false, bool comp = false) {
  return (size_t)nd * 32 * (16 + 8 + 4) + (size_t)(pf ? 4 : 2) * nd * nw * 32 * 4 +
         (comp ? (size_t)nd * nw * 32 * 2 : 0);
}

// COMP: FP32_COMP, each value's 16-bit compensation read from loi and
// written to loo ([ntr][S] like the values)
template <bool LAST, bool PF, bool COMP>
__global__ void __launch_bounds__(kVd32MaxWarps * 32) k_vd32(Geo G, Flow F, Work W, Opt O,
                                                             TrSet T, SubStep ss, Tile Tl,
                                                             const float4 *__restrict__ lu32,
                                                             const float *__restrict__ tri,
                                                             float *__restrict__ tro,
                                                             const float *__restrict__ rsi,
                                                             double *__restrict__ carry,
                                                             const double *__restrict__ fzs,
                                                             const int16_t *__restrict__ loi,
                                                             int16_t *__restrict__ loo,
                                                             int nw, int tile0, int kbase) {
  extern __shared__ __align__(16) unsigned char smem[];
  // the arrays hold layers kbase .. nz-1 (every column of this launch's
  // tiles starts at or above kbase), row r = layer - kbase
  const int nz = G.nz, nd = nz - kbase;
  float4 *LU = reinterpret_cast<float4 *>(smem);          // [nd][32]
  double *DZ = reinterpret_cast<double *>(LU + nd * 32);  // [nd][32]
  int *colC = reinterpret_cast<int *>(DZ + nd * 32);      // [nd][32]
  // per buffer (two with PF): A, S float [nd][nw][32]; then R (COMP)
  float *const bufs = reinterpret_cast<float *>(colC + nd * 32);

  const int lane = threadIdx.x, wy = threadIdx.y;
  const int tile = tile0 + blockIdx.x;
  const int col = Tl.vdcol[tile * 32 + lane];
  const int sa = nw * 32;

  const TileCol tc = tile_column(G, W, Tl, col);
  bool act = tc.act;
  if (act && tc.kb < kbase) {  // not in this launch's depth class
    act = false;
    if (wy == 0) atomicOr(W.status, ST_GEOM);
  }
  const int kb = tc.kb, ks = tc.ks, cbot = tc.cbot, c2 = tc.c2;
  // the tile's tracer-independent column arrays, once for every tracer
  const int kmin = __reduce_min_sync(0xffffffffu, act ? kb : nz);
  for (int k = kmin + wy; k < nz; k += nw) {
    const int c = (act && k >= kb) ? Tl.cellk[(size_t)k * Tl.ncolp + col] : 0;
    const int r = k - kbase;
    colC[r * 32 + lane] = c;
    if (LAST && c && k <= ks) cp_async16(&LU[r * 32 + lane], &lu32[c]);
    if (c && k <= ks) cp_async8(&DZ[r * 32 + lane], &W.dz[c]);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  if (!act) return;

  const size_t off = (size_t)wy * 32 + lane + (size_t)(kb - kbase) * sa;
  auto A0of = [&](int b) { return bufs + (size_t)b * 2 * nd * sa + off; };
  auto S0of = [&](int b) { return bufs + (size_t)b * 2 * nd * sa + (size_t)nd * sa + off; };
  int16_t *const R0 =
      COMP ? reinterpret_cast<int16_t *>(bufs + (size_t)(PF ? 4 : 2) * nd * sa) + off : nullptr;
  const float4 *const L0 = LU + (kb - kbase) * 32 + lane;
  const int *const C0 = colC + (kb - kbase) * 32 + lane;
  const double *const D0 = DZ + (kb - kbase) * 32 + lane;
  const double area = G.cellarea[c2], ia = 1.0 / area;
  const bool steady = F.eta[c2] == F.oldeta[c2];
  const int ntc = G.colntr[col];
  const int sed = G.zm1[cbot];
  // the column's values of slot s into buffer b, one batch of asynchronous
  // copies: advection results and their rounding residuals (advected
  // tracers; the residuals go to the Thomas storage until the sweep) or the
  // old values (the rest)
  auto stage = [&](int s, int b) {
    const int n = T.slot_tr[s];
    const bool tb = (T.trf[n] & TR_TBDY) != 0;
    const float *src = (tb ? tro : tri) + (size_t)n * G.S;
    float *const A0 = A0of(b), *const S0 = S0of(b);
    for (int j = 0; j < nz - kb; ++j) cp_async4(&A0[j * sa], src + C0[j * 32]);
    if (tb) {
      const float *rs = rsi + (size_t)n * G.S;
      for (int j = 0; j < nz - kb; ++j) cp_async4(&S0[j * sa], rs + C0[j * 32]);
    }
    cp_async_commit();
  };
  // warp wy takes the tracers wy, wy + nw, ... the column carries
  auto next = [&](int s) {
    for (; s < T.nslot; s += nw)
      if (T.slot_tr[s] < ntc) return s;
    return T.nslot;
  };
  long long nwarn = 0;
  bool bad = false;  // a NaN among the values this thread stores
  int slot = next(wy), b = 0;
  if (PF && slot < T.nslot) stage(slot, 0);
  while (slot < T.nslot) {
    const int nxt = next(slot + nw);
    if (PF) {  // the next tracer's column is copied while this one is solved
      if (nxt < T.nslot) {
        stage(nxt, b ^ 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
    } else {
      stage(slot, 0);
    }
    const int n = T.slot_tr[slot];
    const int tf = T.trf[n];
    const bool tbdy = (tf & TR_TBDY) != 0;
    const bool adv = tbdy && (tf & TR_ADV);
    const bool vdf = LAST && (tf & TR_VDIFF);
    const float *tr = tri + (size_t)n * G.S;
    float *to = tro + (size_t)n * G.S;
    to[sed] = tbdy ? tr[cbot] : tr[sed];  // sediment ghost (tracers.c:827-830)
    const int16_t *li = COMP ? loi + (size_t)n * G.S : nullptr;
    int16_t *lo = COMP ? loo + (size_t)n * G.S : nullptr;
    if (COMP) lo[sed] = tbdy ? li[cbot] : li[sed];
    const ColSums cs{0.0, 0.0, adv ? fzs[(size_t)n * G.ncol + col] : 0.0};
    if (!PF) cp_async_wait<0>();
    column_finish<LAST, true>(G, F, W, O, T, ss, tc, col, n, tbdy, adv, vdf, A0of(b), S0of(b),
                              sa, L0, C0, D0, tr, to, area, ia, 1.0 / F.dt, cs, carry, steady,
                              nwarn, bad, R0, li, lo);
    slot = nxt;
    if (PF) b ^= 1;
  }
  if (bad) atomicOr(W.status, ST_NAN);
  if (nwarn) atomicAdd(W.nwarn, (unsigned long long)nwarn);
}

}  // namespace shoc
