// shoc_tr_tile64.cuh -- the plain FP64 transport kernels of the staged columns
// (surface cell stays in its layer during the step), bitwise equal to the
// reference: the same two-kernel structure as the FP32-mixed path
// (shoc_tr_tile.cuh), with model/hd/tracers/tracers.c's arithmetic operation
// by operation (compiled without FMA contraction, IEEE division).
//
//  k_adv64  one thread per wet cell: the QUICKEST / Van Leer face values with
//           ULTIMATE and horizontal diffusion of the cell's west, south,
//           north, (east) and bottom and top faces (quickest :1819-1931,
//           ulimate_filter :3501-3557, van_leer_do :2087-2119, hor_diffuse
//           :3595-3668), the flux divergence and the interior update
//           (advect_diffuse :888-925).  The Courant numbers are formed in the
//           kernel exactly as :730-736 form them.
//  k_vd64   one thread per (column, tracer): tr_bounds (:3217-3324),
//           surf_conc (:3047-3207), the copy above the surface, and the
//           implicit vertical diffusion (implicit_vdiff_tr :4067-4214) with
//           the LU factors k_set_dz builds.
//
// Every face value is computed from the same operands in the same order as
// column_pass computes it (a cell's top face is the next cell's bottom face:
// the same call with the same arguments), so the results are identical.
#pragma once
#include "shoc_tr_tile.cuh"

namespace shoc {

// shared memory of k_vd64 (bytes) for columns of at most nd layers:
// colC int[nd][32], A, S double[nd][nw][32]
inline size_t vd64_smem(int nd, int nw) {
  return (size_t)nd * 32 * 4 + (size_t)2 * nd * nw * 32 * 8;
}

// One horizontal face (advect + hor_diffuse) at a cell with Courant number cr,
// velocity vel (Van Leer's sign), metric factors m, volume flux U; the
// diffusion term is (P (t0 - tm1)) / H with P = dzu h2au1 1.0 u1kh and
// H = h1au1 (x; the e2 analogue for y), as flux_x / flux_y form it.
template <bool QUICK, bool ULT>
__device__ __forceinline__ double hface64(bool eb, bool adv, bool hd, double cr, double vel,
                                          const Face2D &m, double U, double P, double H,
                                          double tm2, double tm1, double t0, double tp1) {
  double v = 0.0;
  if (adv) {
    if (QUICK)
      v = quickest_face(cr, m, tm2, tm1, t0, tp1);
    else if (eb)
      v = vanleer_face(vel, cr, tm2, tm1, t0, tp1);
    if (ULT && eb) v = ultimate_face(cr, v, tm2, tm1, t0, tp1);
    v *= U;
  }
  if (hd) v -= (P * (t0 - tm1) / H);
  return v;
}

// The vertical face of flux_z at cell c (below it zm, above it zp) with its
// Courant number cz = w dtu / w9 and w dtu precomputed; the work-array
// values are read here (cached loads) to keep them out of registers.
template <bool QUICK, bool ULT>
__device__ __forceinline__ double zface64(const Flow &F, const Work &W, int c, int zm, int zp,
                                          double cz, double wdtu, double tm2, double tm1,
                                          double t0, double tp1) {
  double v;
  if (QUICK)
    v = quickest_zface(cz, W.w5[c], W.dbz[c], W.dfz[c], W.w9[zm], W.w9[c], W.w9[zp], tm2, tm1,
                       t0, tp1);
  else
    v = vanleer_face(F.w[c], cz, tm2, tm1, t0, tp1);
  if (ULT) v = ultimate_face(cz, v, tm2, tm1, t0, tp1);
  return v * wdtu;
}

// ---------------------------------------------------------------------------
// k_adv64

template <bool QUICK, bool ULT, int MODE>
__global__ void __launch_bounds__(kAdvBlock, 2) k_adv64(Geo G, Flow F, Work W, TrSet T,
                                                     SubStep ss, Tile Tl,
                                                     const double *__restrict__ tri,
                                                     double *__restrict__ tro,
                                                     double *__restrict__ fzs, int any_hd) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ int sTr[kMaxTracers], sTf[kMaxTracers];
  const int i = blockIdx.x * kAdvBlock + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int nz = G.nz;
  for (int s = threadIdx.x; s < T.ntb; s += kAdvBlock) {
    const int n = T.slot_tr[s];
    sTr[s] = n;
    sTf[s] = T.trf[n];
  }
  __syncthreads();

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
  const int cd1 = __shfl_down_sync(FULL, c, 1);
  const bool sxp1 = on && lane <= 30 && cd1 && n1.y == cd1;

  // tracer-independent face data: Courant numbers and volume fluxes (the
  // metric factors and work arrays are read per face from cache)
  const double dtu = ss.dtu;
  const bool hdf = any_hd != 0;
  const int xp = n1.y, yp = n1.w, zp = nzv.z, zm = nzv.x;
  const bool e1 = fl & CF_E1, e2 = fl & CF_E2;
  const bool ewet = !sxp1 && (fl & FL_XP_WET), nwet = fl & FL_YP_WET;
  const bool e1e = fl & FL_XP_E1, e2n = fl & FL_YP_E2;
  double crw = 0.0, crs = 0.0, crn = 0.0, cre = 0.0, czb = 0.0, czt = 0.0;
  double Uw = 0.0, Us = 0.0, Un = 0.0, Ue = 0.0, wdb = 0.0, wdt = 0.0;
  const bool zf = on && k <= ks, ztop = on && k < ks;
  if (on) {
    // Courant numbers as tracers.c:730-736 (w6, w7, w8)
    crw = F.u1[c] * dtu / G.h1au1[c2];
    crs = F.u2[c] * dtu / G.h2au2[c2];
    Uw = F.u1flux3d[c];
    Us = F.u2flux3d[c];
    if (nwet) {
      crn = F.u2[yp] * dtu / G.h2au2[me.y];
      Un = F.u2flux3d[yp];
    }
    if (ewet) {
      cre = F.u1[xp] * dtu / G.h1au1[me.x];
      Ue = F.u1flux3d[xp];
    }
    if (zf) {
      czb = F.w[c] * dtu / (W.w9[c] * 1.0);
      wdb = F.w[c] * dtu;
    }
    if (ztop) {
      czt = F.w[zp] * dtu / (W.w9[zp] * 1.0);
      wdt = F.w[zp] * dtu;
    }
  }
  // hor_diffuse (tracers.c:3654-3667): csx = dzu1 h2au1 mdx, then
  // csx u1kh (t0 - tm1) / h1au1 (the e2 analogue for y)
  auto Px = [&](int cc, int cc2) { return F.dzu1[cc] * G.h2au1[cc2] * 1.0 * F.u1kh[cc]; };
  auto Py = [&](int cc, int cc2) { return F.dzu2[cc] * G.h1au2[cc2] * 1.0 * F.u2kh[cc]; };
  // vertical neighbours (bottom: the sediment ghost holds the bottom value)
  const int vm1 = (k - 1 >= kb) ? nzv.x : c;
  const int vm2 = (k - 2 >= kb) ? nzv.y : vm1;
  const int idx[13] = {c,   n1.z, n2.z, n1.w, n2.w, vm1, vm2,
                       zp,  nzv.w, n1.x, n2.x, n1.y, n2.y};
  const int ntb = T.ntb;

  for (int s = 0; s < ntb; ++s) {
    const int n = sTr[s];
    const int tf = sTf[s];
    if (!__any_sync(FULL, on && n < ntc)) continue;  // no lane carries it
    const bool adv = MODE != 0 || (tf & TR_ADV);
    const bool hd = MODE == 2 || (MODE == 0 && (tf & TR_HDIFF));
    const double *__restrict__ tr = tri + (size_t)n * G.S;
    double v[13];
#pragma unroll
    for (int q = 0; q < 13; ++q) v[q] = tr[idx[q]];
    const double t0 = v[0];
    const double tym1 = v[1], tym2 = v[2], typ1 = v[3], typ2 = v[4];
    const double tm1 = v[5], tm2 = v[6], tp1 = v[7], tp2 = v[8];
    const double txm1 = v[9], txm2 = v[10], txp1 = v[11], txp2 = v[12];
    const bool hor = adv || hd;
    double Fxw = 0.0, Fys = 0.0, Fyn = 0.0, Fxe = 0.0;
    if (on && hor) {
      const bool h = hdf && hd;
      Fxw = hface64<QUICK, ULT>(e1, adv, hd, crw, F.u1[c], G.fx[c2], Uw, h ? Px(c, c2) : 0.0,
                                G.h1au1[c2], txm2, txm1, t0, txp1);
      Fys = hface64<QUICK, ULT>(e2, adv, hd, crs, F.u2[c], G.fy[c2], Us, h ? Py(c, c2) : 0.0,
                                G.h2au2[c2], tym2, tym1, t0, typ1);
      if (nwet)
        Fyn = hface64<QUICK, ULT>(e2n, adv, hd, crn, F.u2[yp], G.fy[me.y], Un,
                                  h ? Py(yp, me.y) : 0.0, G.h2au2[me.y], tym1, t0, typ1, typ2);
      if (ewet)
        Fxe = hface64<QUICK, ULT>(e1e, adv, hd, cre, F.u1[xp], G.fx[me.x], Ue,
                                  h ? Px(xp, me.x) : 0.0, G.h1au1[me.x], txm1, t0, txp1, txp2);
    }
    const double Fnext = __shfl_down_sync(FULL, Fxw, 1);
    if (!on || n >= ntc) continue;
    if (sxp1) Fxe = Fnext;
    // dtracer (tracers.c:888-892)
    const double dtr = (Fxe - Fxw + Fyn - Fys) * dtu;
    double val;
    if (ztop) {
      // interior cell (tracers.c:912-925); Ds = Hn1 = 1 in z coordinates
      const double Fzb =
          adv ? zface64<QUICK, ULT>(F, W, c, zm, zp, czb, wdb, tm2, tm1, t0, tp1) : 0.0;
      const double Fzt =
          adv ? zface64<QUICK, ULT>(F, W, zp, c, nzv.w, czt, wdt, tm1, t0, tp1, tp2) : 0.0;
      double a = t0 * 1.0;
      a -= ((dtr / G.cellarea[c2] + (Fzt - Fzb)) / W.dz[c]);
      a /= 1.0;
      val = a;
    } else {
      val = dtr;
      if (k == ks)
        fzs[(size_t)n * G.ncol + col] =
            adv ? zface64<QUICK, ULT>(F, W, c, zm, zp, czb, wdb, tm2, tm1, t0, tp1) : 0.0;
    }
    tro[(size_t)n * G.S + c] = val;
  }
}

// ---------------------------------------------------------------------------
// k_vd64

template <bool LAST>
__global__ void __launch_bounds__(256) k_vd64(Geo G, Flow F, Work W, Opt O, TrSet T,
                                              SubStep ss, Tile Tl,
                                              const double *__restrict__ tri,
                                              double *__restrict__ tro,
                                              const double *__restrict__ fzs,
                                              const double *__restrict__ vdzdt,
                                              const double *__restrict__ vcm1,
                                              const double *__restrict__ vdiv,
                                              const double *__restrict__ vud, int nw,
                                              int nchunk, int tile0, int kbase) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nz = G.nz, nd = nz - kbase;
  double *A = reinterpret_cast<double *>(smem);          // [nd][nw][32]
  double *Sv = A + nd * nw * 32;                         // [nd][nw][32]
  int *colC = reinterpret_cast<int *>(Sv + nd * nw * 32);  // [nd][32]

  const int lane = threadIdx.x, wy = threadIdx.y;
  const int tile = tile0 + blockIdx.x / nchunk, chunk = blockIdx.x % nchunk;
  const int col = Tl.vdcol[tile * 32 + lane];
  const int slot = chunk * nw + wy;
  const int sa = nw * 32;

  const TileCol tc = tile_column(G, W, Tl, col);
  bool act = tc.act;
  if (act && tc.kb < kbase) {  // not in this launch's depth class
    act = false;
    if (chunk == 0 && wy == 0) atomicOr(W.status, ST_GEOM);
  }
  const int kb = tc.kb, ks = tc.ks, cbot = tc.cbot, c2 = tc.c2;
  const ColInfo ci = tc.ci;
  const int kmin = __reduce_min_sync(0xffffffffu, act ? kb : nz);
  for (int k = kmin + wy; k < nz; k += nw)
    colC[(k - kbase) * 32 + lane] = (act && k >= kb) ? Tl.cellk[(size_t)k * Tl.ncolp + col] : 0;
  __syncthreads();
  if (!act || slot >= T.nslot) return;

  const int n = T.slot_tr[slot];
  if (n >= G.colntr[col]) return;  // tracer not carried in this column
  const int tf = T.trf[n];
  const bool tbdy = (tf & TR_TBDY) != 0;
  const bool adv = tbdy && (tf & TR_ADV);
  const bool vdf = LAST && (tf & TR_VDIFF);
  const bool single = (ci.flags & COL_SINGLE) != 0;
  const bool solve = vdf && !single;
  const double *tr = tri + (size_t)n * G.S;
  double *to = tro + (size_t)n * G.S;
  double *const A0 = A + (kb - kbase) * sa + wy * 32 + lane;
  double *const S0 = Sv + (kb - kbase) * sa + wy * 32 + lane;
  const int *const C0 = colC + (kb - kbase) * 32 + lane;
  const int nk = ks - kb, nl = nz - kb;
  {  // the column: advection results (advected tracers) or the old values
    const double *src = tbdy ? to : tr;
    for (int j = 0; j < nl; ++j) cp_async8(&A0[j * sa], src + C0[j * 32]);
    cp_async_commit();
  }
  const double mn = T.mintr[n], mx = T.maxtr[n];
  {  // sediment ghost (tracers.c:827-830)
    const int sed = G.zm1[cbot];
    to[sed] = tbdy ? tr[cbot] : tr[sed];
  }
  const int cs = ci.s;  // the surface cell (= old and new surface)
  const double ts_old = tr[cs];
  const double area = G.cellarea[c2];
  cp_async_wait<0>();

  unsigned long long nwarn = 0;
  int stat = 0;
  double solp = 0.0;
  if (!tbdy) {
    // tracers without advection / diffusion keep their values, then diffuse
    for (int j = 0; j < nl; ++j) {
      to[C0[j * 32]] = A0[j * sa];
      if (isnan(A0[j * sa])) stat |= ST_NAN;
    }
    if (vdf && single) {
      const double h = W.dz[cs] > O.hmin ? W.dz[cs] : O.hmin;
      const double v = A0[nk * sa];
      to[cs] = v + F.dt * (0.0 - 0.0) / h;
    } else if (solve) {
#pragma unroll 4
      for (int j = 0; j <= nk; ++j) {
        const int cc = C0[j * 32];
        double rhs = __ldg(&vdzdt[cc]) * A0[j * sa];
        double sl;
        if (j == 0) {
          rhs = rhs + 0.0;
          sl = rhs / __ldg(&vdiv[cc]);
        } else {
          if (j == nk) rhs = rhs - 0.0;
          sl = (rhs - __ldg(&vcm1[cc]) * solp) / __ldg(&vdiv[cc]);
        }
        S0[j * sa] = sl;
        solp = sl;
      }
    }
  } else {
    double a_below = 0.0;
#pragma unroll 4
    for (int j = 0; j < nk; ++j) {
      const int cc = C0[j * 32];
      double a = A0[j * sa];
      if (j == nk - 1) a_below = a;
      // tr_bounds clip and range check (:3278-3293)
      if (mn <= kClipEps && a < mn) a = mn;
      if (a < mn || a > mx) nwarn++;
      if (isnan(a)) stat |= ST_NAN;
      if (solve) {
        A0[j * sa] = a;
        double rhs = __ldg(&vdzdt[cc]) * a;
        double sl;
        if (j == 0) {
          rhs = rhs + 0.0;
          sl = rhs / __ldg(&vdiv[cc]);
        } else {
          sl = (rhs - __ldg(&vcm1[cc]) * solp) / __ldg(&vdiv[cc]);
        }
        S0[j * sa] = sl;
        solp = sl;
      } else {
        to[cc] = a;
      }
    }
    // surf_conc with s == co (tracers.c:3097-3206)
    double vs = ts_old;
    if (adv) {
      const double Fzb = fzs[(size_t)n * G.ncol + col];
      const double fcbot = -Fzb * area;
      double surftr = -fcbot;
      const double wbot = (cs == cbot) ? G.botz[c2] : G.gridz[cs];
      const double eta = F.eta[c2], oe = F.oldeta[c2];
      const double sub = oe + ss.subeta_f * (eta - oe);
      const double osub = ss.first ? oe : oe + ss.osub_f * (eta - oe);
      const double dzs = sub - wbot;
      const double svol = dzs * area;
      surftr += (ts_old * area * (osub - wbot) - A0[nk * sa]);
      for (int j = nk + 1; j < nl; ++j) surftr -= (A0[j * sa]);
      double sv;
      if (svol == 0.0 || (surftr < 0.0 && dzs <= O.hmin))
        sv = 0.0;
      else
        sv = surftr / svol;
      vs = (G.botz[c2] > 0.0 && W.dz[cs] < O.hmin) ? ts_old : sv;
    }
    // tr_bounds thin-surface fix (:3250-3272); the cursor cannot move here
    if ((ci.flags & COL_THIN) && (vs < mn || vs > mx)) vs = a_below;
    if (mn <= kClipEps && vs < mn) vs = mn;
    if (vs < mn || vs > mx) nwarn++;
    if (isnan(vs)) stat |= ST_NAN;
    for (int j = nk; j < nl; ++j) to[C0[j * 32]] = vs;
    if (vdf && single) {
      const double h = W.dz[cs] > O.hmin ? W.dz[cs] : O.hmin;
      to[cs] = vs + F.dt * (0.0 - 0.0) / h;
    } else if (solve) {
      A0[nk * sa] = vs;
      double rhs = __ldg(&vdzdt[cs]) * vs;
      double sl;
      if (nk == 0) {
        rhs = rhs + 0.0;
        sl = rhs / __ldg(&vdiv[cs]);
      } else {
        rhs = rhs - 0.0;
        sl = (rhs - __ldg(&vcm1[cs]) * solp) / __ldg(&vdiv[cs]);
      }
      S0[nk * sa] = sl;
    }
  }
  if (solve) {
    // back substitution and update (:4197-4205)
    double x = S0[nk * sa];
    double a = A0[nk * sa];
    double fin = a + (x - a) * 1.0;
    to[cs] = fin;
    if (isnan(fin)) stat |= ST_NAN;
    double udp = __ldg(&vud[cs]);
#pragma unroll 4
    for (int j = nk - 1; j >= 0; --j) {
      const int cc = C0[j * 32];
      x = S0[j * sa] - udp * x;
      a = A0[j * sa];
      fin = a + (x - a) * 1.0;
      to[cc] = fin;
      if (isnan(fin)) stat |= ST_NAN;
      udp = __ldg(&vud[cc]);
    }
  }
  if (nwarn) atomicAdd(W.nwarn, nwarn);
  if (stat) atomicOr(W.status, stat);
}

}  // namespace shoc
