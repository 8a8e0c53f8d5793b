// shoc_tr_fused.cuh -- the FP32-mixed transport sub-step as ONE kernel per
// sub-step: advection and horizontal diffusion (advect_diffuse, tracers.c:
// 849-925), tr_bounds (:3217-3324), surf_conc (:3047-3207) and, on the last
// sub-step, the implicit vertical diffusion (vert_diffuse_3d /
// implicit_vdiff_tr, :3893-3953, :4067-4214) of a tile of 32 water columns
// over all its layers and tracers, with an FP64 per-column mass carry.
//
// A block owns one tile of tx x (32 / tx) columns (tx = 8, 16 or 32, a
// launch parameter the autotuner chooses; lane = tx * iy + ix for the column
// at (i0 + ix, j0 + iy)) and runs two phases:
//
//  A  advection, layer chunk by layer chunk from the top down: warp w holds
//     layer k0 - w of the chunk, so a thread holds one cell and folds its
//     tracer-independent face coefficients once, then loops over the
//     advected tracers two at a time with no block barrier in the loop.  Of
//     a cell's six face fluxes it computes the west, south, bottom and top
//     ones; the east and north fluxes are the west / south fluxes of the
//     lanes at ix + 1 / iy + 1 (shuffles), computed by the cell itself where
//     that neighbour is not in the tile.  The flux divergence and the
//     interior update are FP64; the new value of every cell below the
//     surface goes to the output array (FP32).  Per (column, tracer) the
//     exact FP64 mass of those values (the sum of a * dz), the FP64
//     divergence of the surface cell and the cells above it, and the surface
//     cell's bottom-face flux are accumulated: each cell's contribution goes
//     to shared memory and one pass per chunk (and group of tracers) adds
//     them up in layer order, so the sums do not depend on the schedule.
//  B  one thread per (column, tracer): tr_bounds, surf_conc's
//     column-mass balance (FP64), the copy above the surface and, on the
//     last sub-step, the FP32 Thomas sweep with an FP64 residual and one FP32
//     correction solve, as k_vd32 (shoc_tr_tile.cuh) does.  The column's
//     values come back from the output array (written a few microseconds
//     earlier by phase A of the same block: an L2 round trip, not an HBM one)
//     in one batch of asynchronous copies; the LU factors and the layer
//     thicknesses were copied into shared memory while phase A ran.
//
// The column's end of the sub-step (tr_bounds, surf_conc, the solve and the
// FP64 mass carry) is column_finish, as in k_vd32 (shoc_tr_tile.cuh): the
// fused and the two-kernel sub-steps differ only in where the advected
// values' FP64 column sums come from (phase A's accumulators here, the
// advection kernel's rounding residuals there).
#pragma once
#include "shoc_tr_tile.cuh"

namespace shoc {

constexpr int kFusedThreads = 256;  // 8 warps: one layer of the chunk per warp in phase A
constexpr int kFusedWarps = kFusedThreads / 32;
constexpr int kFusedMaxTracers = 64;  // advected tracers the fused kernel's accumulators hold

struct Fused {
  const int *tcol;    // [ntile][32] column of each lane of each tile (-1: none)
  const int *tkmin;   // [ntile] lowest layer of the tile's columns
  int ntile;
  int tx;             // tile width along i (8, 16 or 32)
  double *carry;      // [ntr][ncol] FP64 mass the stored values owe each column
  int nwb;            // warps of phase B (tracers in flight per tile)
  int ngrp;           // advected tracers per phase-A reduction pass
};

// shared memory of k_step32 (bytes) for columns of at most nd layers, nwb
// phase-B warps, ntb advected tracers and reduction groups of ngrp tracers:
// LU float4 [nd][32], thicknesses double [nd][32], cells int [nd][32], a
// union of the phase-B column arrays float
// [2][nwb][nd][32] with the phase-A contributions double [8][ngrp][32]
// followed by its stencil double buffer float [2][13][256], the
// accumulators double [ntb][32] x 3, and the surface layer of each lane
constexpr int kStencil = 13;  // values of a cell's advection stencil
__host__ __device__ inline size_t fused_red(int ngrp) {
  return (size_t)kFusedWarps * ngrp * 32 * 8;
}
__host__ __device__ inline size_t fused_union(int nd, int nwb, int ngrp) {
  const size_t a = (size_t)2 * nwb * nd * 32 * 4;
  const size_t r = fused_red(ngrp) + (size_t)2 * kStencil * kFusedThreads * 4;
  return a > r ? a : r;
}
inline size_t fused_smem(int nd, int nwb, int ntb, int ngrp) {
  return (size_t)nd * 32 * (16 + 8) + (size_t)nd * 32 * 4 + fused_union(nd, nwb, ngrp) +
         (size_t)ntb * 32 * (8 + 8 + 8) + 32 * 4;
}


// ---------------------------------------------------------------------------

template <bool QUICK, bool ULT, bool LAST>
__global__ void __launch_bounds__(kFusedThreads, 2)
    k_step32(Geo G, Flow F, Flow32 F3, Work W, Opt O, TrSet T, SubStep ss, Tile Tl, Fused Fu,
             const f32::Face2 *__restrict__ fx2, const f32::Face2 *__restrict__ fy2,
             const float *__restrict__ tri, float *__restrict__ tro, int any_hd, int kbase) {
  using namespace f32;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nz = G.nz, nd = nz - kbase, nwb = Fu.nwb, ntb = T.ntb, ngrp = Fu.ngrp;
  float4 *LU = reinterpret_cast<float4 *>(smem);                  // [nd][32]
  double *DZ = reinterpret_cast<double *>(LU + nd * 32);          // [nd][32]
  int *colC = reinterpret_cast<int *>(DZ + nd * 32);              // [nd][32]
  unsigned char *uni = reinterpret_cast<unsigned char *>(colC + nd * 32);
  float *A = reinterpret_cast<float *>(uni);                      // [nwb][nd][32]
  float *Sv = A + nwb * nd * 32;                                  // [nwb][nd][32]
  double *red = reinterpret_cast<double *>(uni);                  // [8][ngrp][32]
  float *pf = reinterpret_cast<float *>(uni + fused_red(ngrp));   // [2][13][256]
  double *accM = reinterpret_cast<double *>(uni + fused_union(nd, nwb, ngrp));  // [ntb][32]
  double *accD = accM + ntb * 32;                                 // [ntb][32]
  double *accF = accD + ntb * 32;                                 // [ntb][32]
  int *sks = reinterpret_cast<int *>(accF + ntb * 32);            // [32]

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int tile = blockIdx.x;
  const int col = Fu.tcol[tile * 32 + lane];
  const TileCol tc = tile_column(G, W, Tl, col);
  const int kb = tc.kb, ks = tc.ks, cbot = tc.cbot, c2 = tc.c2;
  const int ntc = tc.act ? G.colntr[col] : 0;
  const int kmin = Fu.tkmin[tile];

  // the cells of the tile's columns and, on the last sub-step, their LU
  // factors, copied while phase A runs
  for (int k = kmin + w; k < nz; k += kFusedWarps) {
    const int c = (tc.act && k >= kb) ? Tl.cellk[(size_t)k * Tl.ncolp + col] : 0;
    const int r = k - kbase;
    colC[r * 32 + lane] = c;
    if (LAST && c && k <= ks) cp_async16(&LU[r * 32 + lane], &W.lu32[c]);
    if (c && k <= ks) cp_async8(&DZ[r * 32 + lane], &W.dz[c]);
  }
  cp_async_commit();
  for (int i = threadIdx.x; i < ntb * 32; i += kFusedThreads) {
    accM[i] = 0.0;
    accD[i] = 0.0;
    accF[i] = 0.0;
  }
  if (w == 0) sks[lane] = tc.act ? ks : -1;
  __syncthreads();

  // ---------------- phase A: advection, one layer of the chunk per warp
  const double dtu = ss.dtu;
  const float fdtu = (float)dtu;
  const bool hdf = any_hd != 0;
  const double area = tc.act ? G.cellarea[c2] : 1.0;
  const double ia = 1.0 / area;
  int nstat = 0;
  for (int k0 = nz - 1; k0 >= kmin; k0 -= kFusedWarps) {
    const int k = k0 - w;
    const int c = k >= kmin ? colC[(k - kbase) * 32 + lane] : 0;
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
    // east / north neighbours that are the cells of the lanes at ix + 1 / iy + 1
    const int tx = Fu.tx;
    const int cE = __shfl_down_sync(FULL, c, 1), cN = __shfl_down_sync(FULL, c, tx);
    const bool sxp1 = on && (lane & (tx - 1)) != tx - 1 && cE != 0 && n1.y == cE;
    const bool syp1 = on && lane < 32 - tx && cN != 0 && n1.w == cN;
    const bool zf = on && k <= ks, zt = on && k < ks;
    Face fw, fs, fn, fe, fzb, fzt;
    f32::face_zero(fw);
    f32::face_zero(fs);
    f32::face_zero(fn);
    f32::face_zero(fe);
    f32::face_zero(fzb);
    f32::face_zero(fzt);
    double dz0d = 1.0, idz = 0.0;
    if (on) {
      const Face2 mx = fx2[c2], my = fy2[c2];
      hface(fw, fl & CF_WET, fl & CF_E1, QUICK, ULT,
                 __fmul_rn(__fmul_rn(F3.u1[c], fdtu), mx.ih), F3.u1flux3d[c],
                 hdf ? F3.khx[c] : 0.f, mx);
      hface(fs, fl & CF_WET, fl & CF_E2, QUICK, ULT,
                 __fmul_rn(__fmul_rn(F3.u2[c], fdtu), my.ih), F3.u2flux3d[c],
                 hdf ? F3.khy[c] : 0.f, my);
      if (!syp1 && (fl & FL_YP_WET)) {
        const int yp = n1.w;
        const Face2 mn = fy2[me.y];
        hface(fn, true, fl & FL_YP_E2, QUICK, ULT,
                   __fmul_rn(__fmul_rn(F3.u2[yp], fdtu), mn.ih), F3.u2flux3d[yp],
                   hdf ? F3.khy[yp] : 0.f, mn);
      }
      if (!sxp1 && (fl & FL_XP_WET)) {
        const int xp = n1.y;
        const Face2 mxe = fx2[me.x];
        hface(fe, true, fl & FL_XP_E1, QUICK, ULT,
                   __fmul_rn(__fmul_rn(F3.u1[xp], fdtu), mxe.ih), F3.u1flux3d[xp],
                   hdf ? F3.khx[xp] : 0.f, mxe);
      }
      const float dz0 = W.dz32[c];
      if (zf) {
        const float dzm1 = W.dz32[nzv.x], dzm2 = W.dz32[nzv.y];
        const bool top = (nzv.z == c);
        const float dzp1 = W.dz32[nzv.z];
        zface(fzb, QUICK, ULT, dzm2, dzm1, dz0, dzp1, top, __fmul_rn(F3.w[c], fdtu),
              __dmul_rn(F3.w64[c], dtu));
        if (zt) {  // the bottom face of the cell above, folded alike
          const bool top1 = (nzv.w == nzv.z);
          const float dzp2 = W.dz32[nzv.w];
          zface(fzt, QUICK, ULT, dzm1, dz0, dzp1, dzp2, top1, __fmul_rn(F3.w[nzv.z], fdtu),
                __dmul_rn(F3.w64[nzv.z], dtu));
        }
      }
      dz0d = W.dz[c];
      idz = 1.0 / dz0d;
    }
    // vertical neighbours (below the bottom: the sediment ghost holds the
    // bottom value, tracers.c:827-830)
    const int vm1 = (k - 1 >= kb) ? nzv.x : c;
    const int vm2 = (k - 2 >= kb) ? nzv.y : vm1;
    const int vp1 = nzv.z, vp2 = nzv.w;
    const bool needE = on && !sxp1, needN = on && !syp1;

    // the stencil of the cell: its own value, y-1, y-2, y+1, y+2, z-1, z-2,
    // z+1, z+2, x-1, x-2, x+1, x+2 (cells that are not used are valid cells)
    const int idx[kStencil] = {c,   n1.z, n2.z, n1.w, n2.w, vm1, vm2,
                               vp1, vp2,  n1.x, n2.x, n1.y, n2.y};
    // copies the stencil of slot s into this thread's slots of buffer b
    auto issue = [&](int s, int b) {
      const float *tr = tri + (size_t)T.slot_tr[s] * G.S;
      float *d = pf + b * kStencil * kFusedThreads + threadIdx.x;
#pragma unroll
      for (int q = 0; q < kStencil; ++q) cp_async4(d + q * kFusedThreads, tr + idx[q]);
      cp_async_commit();
    };
    for (int g0 = 0; g0 < ntb; g0 += ngrp) {
      const int g1 = min(ntb, g0 + ngrp);
      issue(g0, 0);
      for (int s = g0; s < g1; ++s) {
        const int b = (s - g0) & 1;
        if (s + 1 < g1) {
          issue(s + 1, b ^ 1);
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        const float *v = pf + b * kStencil * kFusedThreads + threadIdx.x;
        const int n = T.slot_tr[s];
        const int tf = T.trf[n];
        const bool adv = (tf & TR_ADV) != 0, hd = (tf & TR_HDIFF) != 0;
        const bool hor = on && (adv || hd), vz = on && adv && zf;
        const float t0 = v[0];
        const float tym1 = v[1 * kFusedThreads], tym2 = v[2 * kFusedThreads];
        const float typ1 = v[3 * kFusedThreads], typ2 = v[4 * kFusedThreads];
        const float tm1 = v[5 * kFusedThreads], tm2 = v[6 * kFusedThreads];
        const float tp1 = v[7 * kFusedThreads], tp2 = v[8 * kFusedThreads];
        const float txm1 = v[9 * kFusedThreads], txm2 = v[10 * kFusedThreads];
        const float txp1 = v[11 * kFusedThreads], txp2 = v[12 * kFusedThreads];
        const double Fw = hor ? face<QUICK, ULT>(fw, adv, hd, txm2, txm1, t0, txp1) : 0.0;
        const double Fs = hor ? face<QUICK, ULT>(fs, adv, hd, tym2, tym1, t0, typ1) : 0.0;
        double Fe = (hor && needE) ? face<QUICK, ULT>(fe, adv, hd, txm1, t0, txp1, txp2) : 0.0;
        double Fn = (hor && needN) ? face<QUICK, ULT>(fn, adv, hd, tym1, t0, typ1, typ2) : 0.0;
        const double Fb = vz ? face<QUICK, ULT>(fzb, true, false, tm2, tm1, t0, tp1) : 0.0;
        const double Ft = (vz && zt) ? face<QUICK, ULT>(fzt, true, false, tm1, t0, tp1, tp2)
                                     : 0.0;
        const double e = __shfl_down_sync(FULL, Fw, 1);
        const double nb = __shfl_down_sync(FULL, Fs, tx);
        if (sxp1) Fe = e;
        if (syp1) Fn = nb;
        double contrib = 0.0;
        if (on && n < ntc) {
          // FP64 flux divergence (tracers.c:888-892)
          const double dtr = ((Fe - Fw) + (Fn - Fs)) * dtu;
          if (zt) {
            const double a = (double)t0 - (dtr * ia + (Ft - Fb)) * idz;
            const float a32 = (float)a;
            tro[(size_t)n * G.S + c] = a32;
            nstat |= isnan(a32) ? ST_NAN : 0;
            contrib = a * dz0d;
          } else {
            contrib = dtr;
            if (k == ks) accF[s * 32 + lane] = Fb;
          }
        }
        red[(w * ngrp + (s - g0)) * 32 + lane] = contrib;
      }
      // the group's per (column, tracer) sums over the chunk's layers, in
      // layer order: a * dz below the surface, the divergence at and above it
      __syncthreads();
      for (int i = threadIdx.x; i < (g1 - g0) * 32; i += kFusedThreads) {
        const int sg = i >> 5, ln = i & 31, ksl = sks[ln];
        double m = 0.0, dv = 0.0;
        for (int ww = 0; ww < kFusedWarps; ++ww) {
          const int kk = k0 - ww;
          if (kk < kmin || ksl < 0) continue;
          const double v = red[(ww * ngrp + sg) * 32 + ln];
          if (kk < ksl) m += v; else dv += v;
        }
        accM[(g0 + sg) * 32 + ln] += m;
        accD[(g0 + sg) * 32 + ln] += dv;
      }
      __syncthreads();
    }
  }
  cp_async_wait<0>();
  __syncthreads();

  // ---------------- phase B: one thread per (column, tracer)
  if (w < nwb && tc.act) {
    float *const A0 = A + w * nd * 32 + lane + (kb - kbase) * 32;
    float *const S0 = Sv + w * nd * 32 + lane + (kb - kbase) * 32;
    const double *const D0 = DZ + (kb - kbase) * 32 + lane;
    const bool steady = F.eta[c2] == F.oldeta[c2];
    const int *const C0 = colC + (kb - kbase) * 32 + lane;
    const float4 *const L0 = LU + (kb - kbase) * 32 + lane;
    const int nk = ks - kb;  // cells below the surface cell
    const double idt = 1.0 / F.dt;  // the residual's diagonal is dz / dt in FP64
    long long nwarn = 0;
    for (int slot = w; slot < T.nslot; slot += nwb) {
      const int n = T.slot_tr[slot];
      if (n >= ntc) continue;  // tracer not carried in this column
      const int tf = T.trf[n];
      const bool tbdy = slot < ntb;
      const bool adv = tbdy && (tf & TR_ADV);
      const bool vdf = LAST && (tf & TR_VDIFF);
      const float *tr = tri + (size_t)n * G.S;
      float *to = tro + (size_t)n * G.S;
      // the column's values, one batch of asynchronous copies: advection
      // results below the surface (advected tracers) or the old values (the
      // rest, every layer)
      {
        const float *src = tbdy ? to : tr;
        const int nl = tbdy ? nk : nz - kb;
        for (int j = 0; j < nl; ++j) cp_async4(&A0[j * 32], src + C0[j * 32]);
        cp_async_commit();
      }
      {  // sediment ghost (tracers.c:827-830)
        const int sed = G.zm1[cbot];
        to[sed] = tbdy ? tr[cbot] : tr[sed];
      }
      const ColSums cs{accM[slot * 32 + lane], accD[slot * 32 + lane],
                       adv ? accF[slot * 32 + lane] : 0.0};
      bool bad = false;
      cp_async_wait<0>();
      column_finish<LAST, false>(G, F, W, O, T, ss, tc, col, n, tbdy, adv, vdf, A0, S0, 32, L0,
                                 C0, D0, tr, to, area, ia, idt, cs, Fu.carry, steady,
                                 nwarn, bad);
      if (bad) nstat |= ST_NAN;
    }
    if (nwarn) atomicAdd(W.nwarn, (unsigned long long)nwarn);
  }
  if (nstat) atomicOr(W.status, nstat);
}

}  // namespace shoc
