// shoc_tr_gpu.cu -- host side and per-step kernels of the B200 SHOC tracer
// step (C-ABI in include/shoc_tr_gpu.h).
//
// Per step, on the handle's stream:
//   k_reset     clears the per-step reductions
//   k_lateral   set_lateral_BC_tr (tracers.c:5574) into both tracer buffers
//   k_set_dz    one thread per column: set_dz (tracers.c:5731-5848), the
//               scheme work arrays w5/w9 (:561-567) and their 2/(w9+w9)
//               factors, the sub-step search (:591-668) as a min-reduction,
//               and the tracer-independent tridiagonal LU factors of
//               vert_diffuse_3d / implicit_vdiff_tr (:3841-3889, :4185-4195)
//   per sub-step:
//     k_courant   w6/w7/w8 (:726-737) of the general-path columns
//     k_adv32 + k_vd32 (FP32-mixed, shoc_tr_tile.cuh; or the one fused
//                 k_step32 of shoc_tr_fused.cuh, SHOC_TR_GPU_KERNELS=fused)
//                 or k_adv64 + k_vd64 (FP64, shoc_tr_tile64.cuh): the
//                 columns whose surface cell stays in its layer, one thread
//                 per cell, then one per (column, tracer)
//     k_serial    the other columns (surface crossing a layer face, thin-
//                 surface fix coupling tracers, degenerate solve range), one
//                 thread per column looping over tracers: column_pass
// Tracers ping-pong between two buffers; a step is captured in a CUDA graph
// once its sub-step schedule is known.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

#include "shoc_tr_gpu.h"
#include "shoc_tr_kernels.cuh"
#include "shoc_tr_launch.h"
#include "shoc_tr_tile64.cuh"

using namespace shoc;

namespace {

constexpr int kItermax = 20;  // tracers.c:430
constexpr int kSerialBlocks = 148 * 2;  // general-path kernel: one thread per listed column

struct Sched {
  double dtm = 0.0;
  std::vector<SubStep> sub;
};

}  // namespace

struct shoc_tr_gpu {
  int device = 0;
  int precision = SHOC_TR_FP64;
  cudaStream_t stream = nullptr;
  int ntr = 0, S = 0, S2 = 0, nz = 0, ncol = 0, nbpt = 0;
  Geo G{};
  Flow F{};
  Work W{};
  Opt O{};
  TrSet T{};
  int nslot = 0;
  bool any_vdiff = false, any_hdiff = false;
  double dt = 0.0;
  // device allocations
  std::vector<void *> allocs;
  void *tr[2] = {nullptr, nullptr};   // double (FP64) or float (FP32-mixed)
  size_t esize = sizeof(double);
  bool comp = false;                  // SHOC_TR_FP32_COMP: 16-bit compensation beside each value
  int16_t *lo[2] = {nullptr, nullptr};  // [ntr][S] compensation of tr[0] / tr[1]
  double *xfer = nullptr;             // one tracer of FP64, for FP32 upload / download
  Flow32 F3{};
  f32::Face2 *fx2 = nullptr, *fy2 = nullptr;
  Tile tl{};                          // static tables of the column-tile kernels
  float *rnd = nullptr;               // [ntr][S] FP32 rounding residual of k_adv32's values
  double *fzs64 = nullptr;            // [ntr][ncol] surface-cell bottom-face flux
  int adv_flags = 0;                  // 1 / 2: every advected tracer without / with hdiff
  double *cols = nullptr;             // column-solve entry points: their device arrays
  int *halo_send = nullptr, *halo_recv = nullptr;  // halo exchange plan (device cell lists)
  int *colown = nullptr;              // columns counted in the sub-step minimum (null: all)
  double dmin_set = 0.0;              // sub-step minimum imposed by the caller (0: own)
  int nhalo_send = 0, nhalo_recv = 0;
  struct Preamble {                   // transport-mode flow preamble (k_faces, k_wvel)
    bool on = false, ok = false;      // enabled; the window's face lists support it
    int n1 = 0, n2 = 0;               // e1 and e2 face columns
    int2 *fc = nullptr;               // [n1 + n2] {2D cell, bottom face cell}
    double *bz = nullptr;             // [n1 + n2] the faces' floors (botzu1 / botzu2)
    double *detadt = nullptr;         // [S2] surface velocity (wtop)
  } pre;
  Fused fu{};                         // FP32-mixed: the columns' mass carry; k_step32's tiles
  bool fused = false;                 // FP32-mixed sub-steps run k_step32
  size_t fused_bytes = 0;             // its dynamic shared memory
  struct FusedTiles {                 // k_step32 tiles of width 8, 16, 32
    const int *tcol = nullptr, *tkmin = nullptr;
    int ntile = 0;
  } ftile[3];
  int fnwb_max = 0;                   // phase-B warps k_step32 may have (0: no k_step32)
  std::vector<int> vd_depth;          // layers of the k_vd32 tiles, in their (sorted) order
  bool staged = false;                // column-tile fast path
  int cur = 0;
  int *bpt = nullptr, *bin = nullptr;
  // host mirror of the per-tracer flags
  std::vector<uint8_t> trf;
  // schedule / graph
  int probe_left = 2;
  bool have_sched = false;
  Sched sched;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long graph_launches[2] = {0, 0};
  int graph_nsub = -1;
  // tiling
  int tw = 8;
  bool vd_pf = false;  // k_vd32 stages the next tracer's column during the solve
  // profiling
  bool profile = false;
  struct ProfEv {
    int part;  // 0 transport of the last sub-step, 1 advection kernel, 2 column kernel
    cudaEvent_t a, b;
  };
  std::vector<ProfEv> ev;
  double prof_ms[3] = {0.0, 0.0, 0.0};
  int prof_n[3] = {0, 0, 0};
  long long launches = 0;
  // pinned readback
  unsigned long long *h_dtm = nullptr;
  int *h_status = nullptr;
  unsigned long long *h_nwarn = nullptr;
  int *h_counts = nullptr;
  int *d_counts = nullptr;  // [0] vcs, [1] vc
  int last_status = 0;
  long long warn_total = 0;
  // pipeline of the drop-in step on host arrays (made on its first use)
  std::vector<int> slot_host;       // slot -> tracer, as T.slot_tr
  cudaStream_t s_up = nullptr, s_dn = nullptr;  // host -> device, device -> host
  std::vector<cudaEvent_t> pev;     // [0] flow sent, then per chunk: sent, stepped
  double *xout = nullptr;           // FP32-mixed: one tracer of FP64 for the way back
  uint8_t *c3s = nullptr;           // [kItermax + 2][ncol] k_serial cursors between chunks
};

namespace {

#define CK(x)                                       \
  do {                                              \
    cudaError_t e_ = (x);                           \
    if (e_ != cudaSuccess) {                        \
      fprintf(stderr, "shoc_tr_gpu: %s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return SHOC_TR_ECUDA;                         \
    }                                               \
  } while (0)

// Makes a device current for the scope of one entry point and gives the
// caller's current device back on the way out, so a host model that drives
// several devices from one thread keeps its own choice.
struct DeviceScope {
  int prev = -1;
  bool ok = false;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

template <class T>
int dalloc(shoc_tr_gpu *h, T **p, size_t n) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
  if (e != cudaSuccess) return SHOC_TR_ENOMEM;
  h->allocs.push_back(q);
  *p = (T *)q;
  return 0;
}

template <class T>
int dupload(shoc_tr_gpu *h, T **p, const T *src, size_t n) {
  int rc = dalloc(h, p, n);
  if (rc) return rc;
  if (src && n) CK(cudaMemcpy(*p, src, n * sizeof(T), cudaMemcpyHostToDevice));
  else CK(cudaMemset(*p, 0, (n ? n : 1) * sizeof(T)));
  return 0;
}

// ---------------------------------------------------------------------------
// kernels

__global__ void k_reset(Work W, int *counts) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    *W.dtm_bits = 0x7ff0000000000000ull;  // +inf
    *W.serial_count = 0;
    counts[0] = 0;
    counts[1] = 0;
  }
}

// Lateral ghosts take their interior value (set_lateral_BC_tr): written into
// both tracer buffers so the value read during every sub-step, and the value
// left in the returned array, is the start-of-step one.  la / lb (FP32_COMP):
// the buffers' compensations, copied alike.
template <class TR>
__global__ void k_lateral(int nbpt, const int *bpt, const int *bin, const int *slot_tr,
                          int nslot, int S, TR *tra, TR *trb, int16_t *la = nullptr,
                          int16_t *lb = nullptr) {
  long long tot = (long long)nbpt * nslot;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    int n = slot_tr[i / nbpt], b = (int)(i % nbpt);
    size_t off = (size_t)n * S;
    TR v = tra[off + bin[b]];
    tra[off + bpt[b]] = v;
    trb[off + bpt[b]] = v;
    if (la) {
      const int16_t q = la[off + bin[b]];
      la[off + bpt[b]] = q;
      lb[off + bpt[b]] = q;
    }
  }
}

__device__ __forceinline__ void atomic_min_pos(unsigned long long *p, double v) {
  atomicMin(p, (unsigned long long)__double_as_longlong(v));
}

// One thread per column: the surface cells, set_dz (tracers.c:5731-5848), the
// scheme work arrays w5/w9 (:561-567) and their 2/(w9+w9) factors, the
// sub-step search (:591-668) as a min-reduction, the column flags and the
// tracer-independent LU factors of vert_diffuse_3d / implicit_vdiff_tr
// (:3841-3889, :4185-4195).  Layer j of the column (j = 0 the sediment cell,
// j = 1..nk the wet layers from the bottom up) comes from the layer-by-column
// table; the thickness of a layer is a function of the surface cells and two
// layer faces, so the column is streamed twice without per-layer arrays: top
// down for the thicknesses, work arrays and sub-step search (a window of the
// layers around j in registers), bottom up for the LU recurrence.  Every
// value is the reference's expression on the reference's operands, and the
// sub-step minimum does not depend on the order the cells are visited in.
// list_all: put every column the tile kernels do not handle on the
// general-path list (else only the tracer-coupled thin-surface columns).
// fp32: also write the FP32 thickness and LU factors.
// own (or null): 1 for the columns whose cells count in the sub-step minimum
// (a strip of a decomposed basin counts its own columns, not its halo).
// probe: compute the minimum only and leave the surface vectors as they are.
// Reads of arrays no kernel of the step writes go through the read-only
// path (__ldg), so the compiler may issue them ahead of this thread's stores
// to the work arrays.  The walk down a column waits on dependent loads, so
// the kernel is held to 64 registers for 8 blocks (32 warps) per SM: 2.26
// against 2.67 ms outside the transport kernels at stiff2048 (80 registers,
// 6 blocks); tighter bounds spill.
__global__ void __launch_bounds__(128, 8) k_set_dz(Geo G, Flow F, Work W, Opt O, Tile Tl,
                                                int any_vdiff, int *counts, int list_all,
                                                int fp32, const int *own, int probe) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  double dtmin = __longlong_as_double(0x7ff0000000000000ll);
  int nwetcol = 0, ncells = 0;  // this column's share of counts[0], counts[1]
  if (col < G.ncol) {
    const int top = G.col_top[col], bot = G.col_bot[col], kb = G.col_kb[col];
    const int nk = G.nz - kb;  // wet layers of the column
    const int sed = G.zm1[bot];
    // cell of layer j and the layer of a cell of this column
    auto cell = [&](int j) {
      return j == 0 ? sed : __ldg(&Tl.cellk[(size_t)(kb + j - 1) * Tl.ncolp + col]);
    };
    auto jof = [&](int c) { return c == sed ? 0 : __ldg(&G.kof[c]) - kb + 1; };

    // new and old surface cells (tracers.c:5739-5755): down from the top
    // while the cell's bottom is at or above eta, at most to the sediment
    int sur = W.nsur_t[col];
    int jn = nk;
    const double etat = F.eta[top];
    while (jn > 0 && __ldg(&G.gridz[cell(jn)]) >= etat) --jn;
    int nsur = cell(jn);
    if (!probe) {
      W.sur_t[col] = sur;
      W.nsur_t[col] = nsur;
    }
    const bool counts_min = !own || own[col];
    const int js0 = jof(sur);
    // cells-to-process membership (:5778-5800): s is the lower of the two
    int s = sur > nsur ? sur : nsur;
    const int js = js0 < jn ? js0 : jn;
    int c2 = G.m2d[s];
    double tz = F.eta[c2] < F.oldeta[c2] ? F.eta[c2] : F.oldeta[c2];
    double bz = SHOC_TR_DRY_FRAC * O.hmin + G.botz[c2];
    bool wet = (tz > bz && js > 0);
    // thickness of layer j (:5824-5846): from the old surface down to the
    // bottom, the layers above the old surface copy the old surface cell's
    // (with the old surface in the sediment, every layer copies the
    // sediment's)
    const int t2 = G.m2d[sur];
    const double oet = F.oldeta[t2], bott = G.botz[t2], dzsed = W.dz[sed];
    auto dzof = [&](int j) -> double {
      const int jj = j < js0 ? j : js0;
      if (jj == 0) return dzsed;
      const double tp = (jj == js0) ? oet : __ldg(&G.gridz[cell(jj + 1)]);
      return tp - ((jj > 1) ? __ldg(&G.gridz[cell(jj)]) : bott);
    };
    // top-down pass: dz, dz32, w5, w9, dbz, dfz (:530-567), the sub-step
    // search over the cells to process (:591-661) and what the flags need
    const bool substep = O.substep != 0, quick = O.trasc == SHOC_TR_QUICKEST;
    int nc = 0;
    int ja = -1;             // highest layer <= jn of zero thickness
    double dz_js0 = dzsed, dz_jn = 0.0, dz_jn1 = 0.0;
    double dzc = dzof(nk);                         // dz(j)
    double dzm = nk >= 1 ? dzof(nk - 1) : dzsed;   // dz(j - 1)
    double w9c = 0.5 * (dzc + dzm), w9p = w9c;     // w9(j), w9(j + 1)
    for (int j = nk; j >= 1; --j) {
      const int cc = cell(j);
      const double dzmm = j >= 2 ? dzof(j - 2) : 0.0;
      const double w9m = j >= 2 ? 0.5 * (dzm + dzmm) : 0.0;  // w9(j - 1)
      W.dz[cc] = dzc;
      if (fp32) W.dz32[cc] = (float)dzc;
      if (quick || O.trasc == SHOC_TR_ORDER2) W.w5[cc] = dzm / (dzm + dzc);
      W.w9[cc] = w9c;
      W.dbz[cc] = 2.0 / (w9m + w9c);
      W.dfz[cc] = 2.0 / (w9c + w9p);
      if (j == js0) dz_js0 = dzc;
      if (j == jn) dz_jn = dzc;
      if (j == jn - 1) dz_jn1 = dzc;
      if (j <= jn && ja < 0 && !dzc) ja = j;
      if (wet && j <= js) {
        nc++;
        if (substep && counts_min) {
          const int xp = __ldg(&G.xp1[cc]), yp = __ldg(&G.yp1[cc]), zp = cell(j < nk ? j + 1 : nk);
          double d4 = 0.5 * (__ldg(&F.u1[cc]) + __ldg(&F.u1[xp]));
          if (fabs(d4) < kMinVal) d4 = kMinVal;
          double d1 = kSF * fabs(G.h1acell[c2] / d4);
          if (d1 < dtmin) dtmin = d1;
          d4 = 0.5 * (__ldg(&F.u2[cc]) + __ldg(&F.u2[yp]));
          if (fabs(d4) < kMinVal) d4 = kMinVal;
          double d2 = kSF * fabs(G.h2acell[c2] / d4);
          if (d2 < dtmin) dtmin = d2;
          if (j != js) {
            d4 = 0.5 * (__ldg(&F.w[cc]) + __ldg(&F.w[zp]));
            if (fabs(d4) < kMinVal) d4 = kMinVal;
            double d3 = kSF * fabs(dzc * 1.0 / d4);
            if (d3 > 0.0 && d3 < dtmin) dtmin = d3;
          }
        }
      }
      w9p = w9c;
      w9c = w9m;
      dzc = dzm;
      dzm = dzmm;
    }
    if (jn == 0) dz_jn = dzsed;
    if (ja < 0) ja = 0;
    int flags = 0;
    int cbs = 0;
    if (wet) {
      flags |= COL_WET;
      nwetcol = 1;
      ncells = nc;
      // tr_bounds thin-surface test (:3250-3252)
      if (js > 1 && dz_js0 < O.hmin) {
        flags |= COL_THIN;
        if (s != top) flags |= COL_SERIAL;
      }
      // implicit vertical diffusion set-up (:3841-3889) and LU (:4185-4195),
      // bottom up from the lowest layer of the solve
      int cs = nsur;
      if (jn <= 1 || !dz_jn1) {
        flags |= COL_SINGLE;
      } else if (any_vdiff && !dz_jn) {
        // zero-thickness surface cell: the reference solves over an empty
        // range and reads stale work memory; report instead of guessing
        flags |= COL_NOSOLVE;
        atomicOr(W.status, ST_GEOM);
      } else if (any_vdiff) {
        const int jb = ja + 1;  // bottom of the solve
        cbs = cell(jb);
        // dzface(c) = 0.5 (dz[zm1] + dz[c]) for c in [cbs, cs]
        double dt = F.dt;
        int cb = cbs;
        int zpb = cell(jb + 1);
        double dzj = W.dz[cb], dzj1 = W.dz[zpb];
        double dzf_p = 0.5 * (dzj + dzj1);
        double dzdt = dzj / dt;
        double cp1 = -__ldg(&F.Kz[zpb]) / dzf_p;
        double C = dzdt - cp1;
        double div = C;
        W.vd_cm1[cb] = 0.0;
        W.vd_div[cb] = div;
        W.vd_ud[cb] = 0.0;
        W.vd_dzdt[cb] = dzdt;
        if (fp32) W.lu32[cb] = make_float4((float)dzdt, 0.f, (float)(1.0 / div), 0.f);
        double bp1 = cp1;
        int cc2 = zpb;
        for (int j = jb + 1; j < jn; ++j) {
          const int zp = cell(j + 1);
          const double dzn = W.dz[zp];
          double dzf_c = dzf_p;
          dzf_p = 0.5 * (dzj1 + dzn);
          dzdt = dzj1 / dt;
          double cm1 = -__ldg(&F.Kz[cc2]) / dzf_c;
          cp1 = -__ldg(&F.Kz[zp]) / dzf_p;
          C = dzdt - cm1 - cp1;
          double ud = bp1 / div;
          div = C - cm1 * ud;
          if (div == 0.0) atomicOr(W.status, ST_PIVOT);
          W.vd_cm1[cc2] = cm1;
          W.vd_div[cc2] = div;
          W.vd_ud[cc2] = ud;
          W.vd_dzdt[cc2] = dzdt;
          if (fp32)
            W.lu32[cc2] = make_float4((float)dzdt, (float)cm1, (float)(1.0 / div), (float)ud);
          bp1 = cp1;
          cc2 = zp;
          dzj1 = dzn;
        }
        {
          double dzf_c = dzf_p;
          dzdt = dz_jn / dt;
          double cm1 = -__ldg(&F.Kz[cs]) / dzf_c;
          C = dzdt - cm1;
          double ud = bp1 / div;
          div = C - cm1 * ud;
          if (div == 0.0) atomicOr(W.status, ST_PIVOT);
          W.vd_cm1[cs] = cm1;
          W.vd_div[cs] = div;
          W.vd_ud[cs] = ud;
          W.vd_dzdt[cs] = dzdt;
          if (fp32)
            W.lu32[cs] = make_float4((float)dzdt, (float)cm1, (float)(1.0 / div), (float)ud);
        }
      }
    } else if (col == G.v2col) {
      atomicOr(W.status, ST_LASTDRY);
    }
    ColInfo ci;
    ci.s = wet ? s : 0;
    ci.co = sur;
    ci.cs = nsur;
    ci.cbs = cbs;
    ci.flags = flags;
    ci.ks = kb + js - 1;
    if (O.tiled && staged_column(ci, bot)) ci.flags |= COL_STAGED;
    W.col[col] = ci;
    if ((flags & COL_SERIAL) || (list_all && !(ci.flags & COL_STAGED))) {
      int i = atomicAdd(W.serial_count, 1);
      W.serial_list[i] = col;
    }
  }
  // warp-reduce the counts and the sub-step minimum: one atomic per warp
  const int wc = __reduce_add_sync(0xffffffffu, nwetcol);
  const int wn = __reduce_add_sync(0xffffffffu, ncells);
  double v = dtmin;
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) {
    if (wc) atomicAdd(&counts[0], wc);
    if (wn) atomicAdd(&counts[1], wn);
    if (v < __longlong_as_double(0x7ff0000000000000ll)) atomic_min_pos(W.dtm_bits, v);
  }
}

// Courant numbers of one sub-step over every wet cell (tracers.c:730-736).
// only_listed: skip when the general-path list is empty (the staged kernels
// compute their own Courant numbers).
__global__ void k_courant(Geo G, Flow F, Work W, double dtu, int only_listed) {
  if (only_listed && *W.serial_count == 0) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < G.S; c += gridDim.x * blockDim.x) {
    if (!(G.cflag[c] & CF_WET)) continue;
    int c2 = G.m2d[c];
    W.w6[c] = F.u1[c] * dtu / G.h1au1[c2];
    W.w7[c] = F.u2[c] * dtu / G.h2au2[c2];
    W.w8[c] = F.w[c] * dtu / (W.w9[c] * 1.0);
  }
}

// Columns where tr_bounds' thin-surface cursor can move between tracers:
// one thread per column, tracers in tbdy order, as the reference loops.
// When the tracers go through in chunks of slots (the drop-in step's
// pipeline), c3s holds each listed column's cursor state between the chunks
// of one sub-step: read when c3_load, written back always.  lo_out
// (FP32_COMP): these columns step their FP32 values as stored, and their
// compensations, from the sediment ghost to the top cell, are set to 0.
template <bool LAST, class TR>
__global__ void k_serial(Geo G, Flow F, Work W, Opt O, TrSet T, SubStep ss,
                         const TR *__restrict__ tr_in, TR *__restrict__ tr_out,
                         uint8_t *__restrict__ c3s, int c3_load,
                         int16_t *__restrict__ lo_out = nullptr) {
  int cnt = *W.serial_count;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    int col = W.serial_list[i];
    LocalSol sol;
    bool c3 = (c3s && c3_load) ? c3s[i] != 0 : false;
    unsigned long long warn = 0;
    int stat = 0;
    for (int sl = 0; sl < T.nslot; ++sl) {
      int n = T.slot_tr[sl];
      if (n >= G.colntr[col]) continue;  // not carried in this column
      column_pass<LAST>(G, F, W, O, T, ss, tr_in + (size_t)n * G.S, tr_out + (size_t)n * G.S,
                        col, n, G.col_kb[col], true, sol, c3, warn, stat);
      if (lo_out) {
        int16_t *lo = lo_out + (size_t)n * G.S;
        int c = G.zm1[G.col_bot[col]];
        lo[c] = 0;
        do {
          c = G.zp1[c];
          lo[c] = 0;
        } while (c != G.col_top[col]);
      }
    }
    if (c3s) c3s[i] = c3 ? 1 : 0;
    if (warn) atomicAdd(W.nwarn, warn);
    if (stat) atomicOr(W.status, stat);
  }
}

// Compensated (Neumaier) FP64 mass sum per tracer: sum of tr * dz * area
// over each column from its current surface cell (nsur_t, top at eta) down
// to the bottom (botz), the water the column holds now.  One thread per
// (column, tracer); block partials are summed on the host.
__device__ __forceinline__ void neumaier(double &s, double &comp, double v) {
  double u = s + v;
  comp += (fabs(s) >= fabs(v)) ? (s - u) + v : (v - u) + s;
  s = u;
}

// ---------------------------------------------------------------------------
// Transport-mode flow preamble (transport_step, model/hd/tracers/
// transport.c:436-462): what SHOC's transport mode computes from the
// velocities and the surface before the tracer step, on the device.  A z-level
// window, linear free surface (wtop = detadt), no point sources (waterss = 0),
// conserve = CONS_W, mdx = mdy = 1 and no one-cell-deep face list (the
// momentum step builds that list; transport mode does not run it).

// set_dz_at_u1 / set_dz_at_u2 (model/hd/momentum/vel3d.c:720-853, :2718-2850,
// z coordinates) and set_flux_3d (vel3d.c:4041-4175, VEL3D) of one face
// column per thread, e1 faces first: the face's surface is the higher of the
// two elevations beside it (at least the face's floor botzu), its surface cell
// the first cell down from the surface layer whose bottom is at or below it,
// its thicknesses from there to the bottom face cell (the layers above copy
// the surface cell's), the volume flux u dzu h2au1 (h1au2) at and below the
// surface and zero above.  The arrays start zeroed (the reference's memsets).
// fc: {2D cell, bottom face cell} per face column, bz: its floor.
__global__ void k_faces(Geo G, Flow F, int n1, int n, const int2 *fc, const double *bz,
                        double *dzu1, double *dzu2, double *f1, double *f2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool e1 = i < n1;
  const int c2 = fc[i].x, cb = fc[i].y;
  const int nb = e1 ? G.xm1[c2] : G.ym1[c2];
  const double *u = e1 ? F.u1 : F.u2;
  const double hf = e1 ? G.h2au1[c2] : G.h1au2[c2];
  double *dzu = e1 ? dzu1 : dzu2, *flux = e1 ? f1 : f2;
  const double floor = bz[i];
  double top = F.eta[c2] > F.eta[nb] ? F.eta[c2] : F.eta[nb];
  top = top > floor ? top : floor;
  int c = c2, zm = G.zm1[c];
  while (c != zm && G.gridz[c] > top) {
    c = zm;
    zm = G.zm1[c];
  }
  const int sur = c;
  double t = top;
  while (c != cb) {
    const double bot = G.gridz[c];
    const double d = t - bot;
    dzu[c] = d;
    flux[c] = u[c] * d * hf;
    t = bot;
    c = G.zm1[c];
  }
  {
    const double d = t - floor;
    dzu[cb] = d;
    flux[cb] = u[cb] * d * hf;
  }
  const double ds = dzu[sur];
  c = sur;
  while (c != c2) {
    c = G.zp1[c];
    dzu[c] = ds;
  }
}

// vel_w_update (vel3d.c:4609-4760, z coordinates, CONS_W) of one water column
// per thread, before k_set_dz: the column's old surface cell (the previous
// step's new one) and new surface cell, and whether the column is processed,
// as set_dz decides them (tracers.c:5739-5800); then w from continuity from
// the bottom (wbot = 0) up to the old surface, wtop = detadt in the cells the
// surface moved through, and set_w_dry (vel3d.c:5116-5135): wtop in every
// cell above the new surface cell, in every column.  w starts zeroed (the
// reference's memset).
__global__ void k_wvel(Geo G, Flow F, Work W, Opt O, const double *detadt, double *w) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= G.ncol) return;
  const int top = G.col_top[col], bot = G.col_bot[col];
  const int sur = W.nsur_t[col];
  int nsur = top, zm = G.zm1[nsur];
  const double etat = F.eta[top];
  while (nsur != zm && G.gridz[nsur] >= etat) {
    nsur = zm;
    zm = G.zm1[nsur];
  }
  const int s = sur > nsur ? sur : nsur;
  const int c2 = G.m2d[s];
  const double tz = F.eta[c2] < F.oldeta[c2] ? F.eta[c2] : F.oldeta[c2];
  const double bz = SHOC_TR_DRY_FRAC * O.hmin + G.botz[c2];
  if (tz > bz && s != G.zm1[s]) {
    const int cs = G.m2d[bot];
    const double area = G.cellarea[cs];
    int c = bot;
    const double wb = 0.0;  // wbot (vel_w_bounds, z coordinates)
    w[c] = wb;
    double fcbot = wb * area;
    while (c > sur) {
      const int xp = G.xp1[c], yp = G.yp1[c], zp = G.zp1[c];
      const double fctop = fcbot + F.u1flux3d[c] - F.u1flux3d[xp] + F.u2flux3d[c] -
                           F.u2flux3d[yp] + 0.0;  // + waterss
      w[zp] = fctop / area;
      fcbot = fctop;
      c = zp;
    }
    while (c > nsur) {
      const int zp = G.zp1[c];
      w[zp] = detadt[cs];  // wtop (vel_w_bounds, linear surface)
      c = zp;
    }
  }
  // set_w_dry
  const int cs = G.m2d[nsur];
  int c = nsur, zp = G.zp1[c];
  while (c != zp) {
    w[zp] = detadt[cs];
    c = zp;
    zp = G.zp1[c];
  }
}

__global__ void k_to_f32(const double *a, float *b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
// one uploaded tracer into both ping-pong buffers (and, SHOC_TR_FP32_COMP,
// the compensation of both: lb / lc non-null)
__global__ void k_to_f32x2(const double *a, float *b, float *c, size_t n, int16_t *lb = nullptr,
                           int16_t *lc = nullptr) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float v = (float)a[i];
    b[i] = v;
    c[i] = v;
    if (lb) {
      const int16_t q = lo_enc(a[i], v);
      lb[i] = q;
      lc[i] = q;
    }
  }
}
// a tracer back to FP64 (with its compensation where l is non-null)
__global__ void k_to_f64(const float *a, double *b, size_t n, const int16_t *l = nullptr) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = l ? (double)a[i] + lo_dec(l[i], a[i]) : (double)a[i];
}
// K = dzu h2au1 u1kh / h1au1 (e1) or dzu2 h1au2 u2kh / h2au2 (e2): the
// tracer-independent factor of hor_diffuse (tracers.c:3660-3666)
__global__ void k_khfac(Geo G, Flow F, float *khx, float *khy) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < G.S; c += gridDim.x * blockDim.x) {
    if (!(G.cflag[c] & CF_WET)) continue;
    int c2 = G.m2d[c];
    khx[c] = (float)(F.dzu1[c] * G.h2au1[c2] * F.u1kh[c] / G.h1au1[c2]);
    khy[c] = (float)(F.dzu2[c] * G.h1au2[c2] * F.u2kh[c] / G.h2au2[c2]);
  }
}

// carry (FP32-mixed path, else null): [ntr][ncol] mass the stored
// values owe each column, part of the state's mass.
// colreg (or null): the region of each column; only region `reg` is summed.
template <class TR>
__global__ void k_mass(Geo G, Flow F, Work W, const TR *tr, const double *carry, double *out,
                       const int *colreg = nullptr, int reg = 0, const int16_t *lo = nullptr) {
  const int n = blockIdx.y;
  const TR *t = tr + (size_t)n * G.S;
  const int16_t *l = lo ? lo + (size_t)n * G.S : nullptr;  // compensation (FP32_COMP)
  double s = 0.0, comp = 0.0;
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < G.ncol;
       col += gridDim.x * blockDim.x) {
    if (colreg && colreg[col] != reg) continue;
    const int top = G.col_top[col], bot = G.col_bot[col];
    int c = W.nsur_t[col];
    if (n >= G.colntr[col]) continue;  // tracer not carried in this column
    if (carry) neumaier(s, comp, carry[(size_t)n * G.ncol + col]);
    if (c == G.zm1[c]) continue;  // surface below the bottom: dry
    const double area = G.cellarea[top];
    double tz = F.eta[top];
    for (int it = 0; it <= G.nz; ++it) {
      double bz = (c == bot) ? G.botz[top] : G.gridz[c];
      double h = tz - bz;
      if (h > 0.0) {
        const double v = l ? (double)t[c] + lo_dec(l[c], (float)t[c]) : (double)t[c];
        neumaier(s, comp, v * h * area);
      }
      if (c == bot) break;
      tz = bz;
      c = G.zm1[c];
    }
  }
  s += comp;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0, bc = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) neumaier(b, bc, part[i]);
    out[(size_t)n * gridDim.x + blockIdx.x] = b + bc;
  }
}

// Differences between the tracers of two handles of one window: one thread
// per (column, tracer) over the column's wet cells (bottom to top layer), for
// the tracers both handles carry in the column.  Per (region, tracer): the
// largest |a - b| and |b| (atomicMax on the bits of a non-negative double,
// which order as unsigned integers) and the sums of (a - b)^2 and b^2.
template <class TA, class TB>
__global__ void k_compare(Geo G, Tile Tl, const int *colntr_b, const TA *ta, const TB *tb,
                          const int *region, int nreg, unsigned long long *maxabs,
                          unsigned long long *maxref, double *ssd, double *ssr,
                          const int16_t *la, const int16_t *lb) {
  const int n = blockIdx.y;
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < G.ncol;
       col += gridDim.x * blockDim.x) {
    if (n >= G.colntr[col] || n >= colntr_b[col]) continue;
    const int r = region ? region[col] : 0;
    if (r < 0 || r >= nreg) continue;
    double ma = 0.0, mr = 0.0, sd = 0.0, sr = 0.0;
    for (int k = G.col_kb[col]; k < G.nz; ++k) {
      const int c = Tl.cellk[(size_t)k * Tl.ncolp + col];
      if (!c) continue;
      const size_t i = (size_t)n * G.S + c;
      double a = (double)ta[i], b = (double)tb[i];
      if (la) a += lo_dec(la[i], (float)ta[i]);  // FP32_COMP: value + compensation
      if (lb) b += lo_dec(lb[i], (float)tb[i]);
      const double d = a - b;
      ma = fmax(ma, fabs(d));
      mr = fmax(mr, fabs(b));
      sd += d * d;
      sr += b * b;
    }
    const size_t o = (size_t)r * gridDim.y + n;
    atomicMax(&maxabs[o], (unsigned long long)__double_as_longlong(ma));
    atomicMax(&maxref[o], (unsigned long long)__double_as_longlong(mr));
    atomicAdd(&ssd[o], sd);
    atomicAdd(&ssr[o], sr);
  }
}

// ---------------------------------------------------------------------------
// The other per-column tridiagonal solves, one thread per water column (from
// its bottom cell up to its surface cell, the handle's current nsur_t; a
// column whose surface is its sediment cell is dry).  The arithmetic is the
// reference's, operation by operation (this file is compiled without FMA
// contraction, with IEEE division), so the results are bitwise its own.  The
// reference keeps the rows in layer-indexed work vectors; here every array is
// indexed by SHOC cell (a cell carries the row of its layer).

// tridiagonal (model/hd/closure/MY2-5.c:499-536): the closures' solve
__global__ void k_tridiag(Geo G, Work W, const double *C, const double *Cm1, const double *Cp1,
                          const double *rhs, double *var, double *sol, double *ud,
                          double minvar) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= G.ncol) return;
  const int cs = W.nsur_t[col], cb = G.col_bot[col];
  if (cs == G.zm1[cs]) return;
  int stat = 0;
  double div = C[cb];
  sol[cb] = rhs[cb] / div;
  int c = cb;
  for (int it = 0; c != cs && it < G.nz; ++it) {
    const int cn = G.zp1[c];
    ud[cn] = Cp1[c] / div;
    div = C[cn] - Cm1[cn] * ud[cn];
    if (div == 0.0) stat |= ST_PIVOT;
    sol[cn] = (rhs[cn] - Cm1[cn] * sol[c]) / div;
    c = cn;
  }
  if (c != cs) stat |= ST_GEOM;
  for (int it = 0; c != cb && it < G.nz; ++it) {
    const int cd = G.zm1[c];
    sol[cd] -= ud[c] * sol[c];
    c = cd;
  }
  for (int it = 0; it <= G.nz; ++it) {
    var[c] = sol[c] > minvar ? sol[c] : minvar;
    if (c == cs) break;
    c = G.zp1[c];
  }
  if (stat) atomicOr(W.status, stat);
}

// implicit_vdiff_at_cc (model/hd/tracers/tracers.c:7407-7545): implicit
// vertical diffusion of var with bottom / top fluxes fb, ft, sources Splus,
// Sminus (may be null) and the scale factor, with no thin layers
__global__ void k_vdiff_cols(Geo G, Work W, double *var, const double *dzcell, const double *C,
                             const double *Cm1, const double *Cp1, const double *fb,
                             const double *ft, const double *Splus, const double *Sminus,
                             const double *scale, double *sol, double *ud, double dt,
                             double dt_win, double hmin) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= G.ncol) return;
  const int cs = W.nsur_t[col], cb = G.col_bot[col];
  if (cs == G.zm1[cs]) return;
  const int c2 = G.m2d[cs];
  const int zm1 = G.zm1[cs];
  int stat = 0;
  // single layer (the surface in the bottom layer, :7459-7467)
  if (zm1 == G.zm1[zm1] || !dzcell[zm1]) {
    const double h = dzcell[cs] > hmin ? dzcell[cs] : hmin;
    var[cs] += dt_win * (fb[c2] - ft[c2]) / h;
    return;
  }
  // right-hand side (:7479-7508) into sol, the main diagonal with the
  // negative sources into ud (both are rewritten by the sweep below)
  int c = cb;
  for (int it = 0; it <= G.nz; ++it) {
    const double dzdt = dzcell[c] / dt;
    double r = dzdt * var[c];
    if (c == cb) r = r + fb[c2];
    if (c == cs) r = r - ft[c2];
    sol[c] = r;
    ud[c] = C[c];
    if (c == cs) break;
    c = G.zp1[c];
  }
  if (c != cs) stat |= ST_GEOM;
  if (Splus) {
    for (int cc = cb, it = 0; it <= G.nz; cc = G.zp1[cc], ++it) {
      sol[cc] += dzcell[cc] * Splus[cc];
      if (cc == cs) break;
    }
  }
  if (Sminus) {
    for (int cc = cb, it = 0; it <= G.nz; cc = G.zp1[cc], ++it) {
      ud[cc] += dzcell[cc] * Sminus[cc] / var[cc];
      if (cc == cs) break;
    }
  }
  // Thomas sweep (:7517-7526): the main diagonal B sits in ud until the row
  // is eliminated, then ud holds the elimination factor
  double div = ud[cb];
  sol[cb] = sol[cb] / div;
  c = cb;
  for (int it = 0; c != cs && it < G.nz; ++it) {
    const int cn = G.zp1[c];
    const double B = ud[cn];
    ud[cn] = Cp1[c] / div;
    div = B - Cm1[cn] * ud[cn];
    if (div == 0.0) stat |= ST_PIVOT;
    sol[cn] = (sol[cn] - Cm1[cn] * sol[c]) / div;
    c = cn;
  }
  // update (:7530-7536)
  const double sc = scale[c2];
  var[cs] += (sol[cs] - var[cs]) * sc;
  for (int it = 0; c != cb && it < G.nz; ++it) {
    const int cd = G.zm1[c];
    sol[cd] -= ud[c] * sol[c];
    var[cd] += (sol[cd] - var[cd]) * sc;
    c = cd;
  }
  if (stat) atomicOr(W.status, stat);
}

// Halo exchange of a strip of a decomposed basin: gather the send cells of
// every tracer into a contiguous buffer, or scatter a buffer into the
// receive cells of both tracer buffers.
template <class TR>
__global__ void k_halo_pack(const TR *tr, int S, int ntr, const int *cells, int n, TR *buf) {
  const long long tot = (long long)ntr * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / n), j = (int)(i % n);
    buf[i] = tr[(size_t)t * S + cells[j]];
  }
}
template <class TR>
__global__ void k_halo_unpack(TR *tra, TR *trb, int S, int ntr, const int *cells, int n,
                              const TR *buf) {
  const long long tot = (long long)ntr * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / n), j = (int)(i % n);
    const size_t o = (size_t)t * S + cells[j];
    tra[o] = buf[i];
    trb[o] = buf[i];
  }
}

// shared memory of the column kernel of the handle's precision
size_t vd_smem(const shoc_tr_gpu *h, int nd, int nw) {
  return h->esize == sizeof(float) ? vd32_smem(nd, nw, h->vd_pf, h->comp) : vd64_smem(nd, nw);
}

// Static tables of the column-tile kernel: the cell of every column at every
// layer (cells are numbered layer by layer, so a column's cells are found by
// walking zp1 up from its bottom cell), the first and second horizontal
// neighbours of every cell, the 2D cells of its east and north neighbours and
// their flags.
int build_tile_tables(shoc_tr_gpu *h, const shoc_tr_geom *g, const std::vector<uint8_t> &cflag,
                      const std::vector<int> &col_bot, const std::vector<int> &col_kb) {
  const int S = h->S, nz = h->nz, ncol = h->ncol;
  const int ncolp = (ncol + 31) / 32 * 32;
  std::vector<int> cellk((size_t)nz * ncolp, 0);
  for (int col = 0; col < ncol; col++) {
    int c = col_bot[col];
    for (int k = col_kb[col]; k < nz; k++) {
      if (c <= 0 || c >= S) break;
      cellk[(size_t)k * ncolp + col] = c;
      c = g->zp1[c];
    }
  }
  auto in = [S](int c) { return c >= 0 && c < S ? c : 0; };
  const int S2 = h->S2;
  auto in2 = [S2](int c) { return c >= 0 && c < S2 ? c : 0; };
  std::vector<int4> nb1(S), nb2(S);
  std::vector<int2> m2e(S);
  std::vector<uint8_t> fl(S);
  for (int c = 0; c < S; c++) {
    const int xm = in(g->xm1[c]), xp = in(g->xp1[c]), ym = in(g->ym1[c]), yp = in(g->yp1[c]);
    nb1[c] = make_int4(xm, xp, ym, yp);
    nb2[c] = make_int4(in(g->xm1[xm]), in(g->xp1[xp]), in(g->ym1[ym]), in(g->yp1[yp]));
    m2e[c] = make_int2(in2(g->m2d[xp]), in2(g->m2d[yp]));
    uint8_t f = cflag[c] & (CF_WET | CF_E1 | CF_E2);
    if (cflag[xp] & CF_WET) f |= FL_XP_WET;
    if (cflag[xp] & CF_E1) f |= FL_XP_E1;
    if (cflag[yp] & CF_WET) f |= FL_YP_WET;
    if (cflag[yp] & CF_E2) f |= FL_YP_E2;
    fl[c] = f;
  }
  // vertical neighbours and the column of each wet cell
  std::vector<int4> nbz(S);
  for (int c = 0; c < S; c++) {
    const int zm = in(g->zm1[c]), zp = in(g->zp1[c]);
    nbz[c] = make_int4(zm, in(g->zm1[zm]), zp, in(g->zp1[zp]));
  }
  std::vector<int> colof(S, 0);
  for (int col = 0; col < ncol; col++)
    for (int k = col_kb[col]; k < nz; k++) {
      const int c = cellk[(size_t)k * ncolp + col];
      if (c) colof[c] = col;
    }
  // k_adv32 cell order: tile by tile (32 adjacent columns), layer by layer
  // within a tile, so the vertical and y-neighbours a block reads were read
  // by blocks shortly before it (cache reuse) and a warp's cells are mostly
  // adjacent cells of one layer
  std::vector<uint8_t> is_wet(S, 0);
  for (int i = 1; i <= g->a3_t; i++) {
    const int c = g->w3_t[i];
    if (c > 0 && c < S) is_wet[c] = 1;
  }
  std::vector<int> wet;
  wet.reserve(g->a3_t);
  for (int t = 0; t < ncolp / 32; t++)
    for (int k = nz - 1; k >= 0; k--)
      for (int l = 0; l < 32; l++) {
        const int col = t * 32 + l;
        if (col >= ncol) break;
        const int c = cellk[(size_t)k * ncolp + col];
        if (c && is_wet[c]) wet.push_back(c);
      }
  // k_vd32 column order: tiles of 32 adjacent columns (a warp's lanes at one
  // layer are adjacent cells: coalesced loads and stores), the tiles sorted
  // by depth so launches per depth class size shared memory to their tiles
  const int ntile = ncolp / 32;
  std::vector<int> tdepth(ntile, 0), tord(ntile);
  for (int t = 0; t < ntile; t++) {
    int kmin = nz;
    for (int l = 0; l < 32 && t * 32 + l < ncol; l++) kmin = std::min(kmin, col_kb[t * 32 + l]);
    tdepth[t] = nz - kmin;
    tord[t] = t;
  }
  std::stable_sort(tord.begin(), tord.end(), [&](int a, int b) { return tdepth[a] < tdepth[b]; });
  std::vector<int> vdcol(ncolp, -1);
  h->vd_depth.resize(ntile);
  for (int i = 0; i < ntile; i++) {
    const int t = tord[i];
    h->vd_depth[i] = tdepth[t];
    for (int l = 0; l < 32; l++) vdcol[i * 32 + l] = (t * 32 + l < ncol) ? t * 32 + l : -1;
  }
  std::vector<int4> colrec(ncolp, make_int4(0, 0, nz, 0));
  for (int col = 0; col < ncol; col++)
    colrec[col] = make_int4(col_bot[col], g->w2_t[col + 1], col_kb[col], 0);
  Tile &T = h->tl;
  T.ncolp = ncolp;
  T.nwet = (int)wet.size();
  int *ip;
  int rc;
  if ((rc = dupload(h, &ip, cellk.data(), cellk.size()))) return rc;
  T.cellk = ip;
  int4 *i4;
  if ((rc = dupload(h, &i4, nb1.data(), S))) return rc;
  T.nb1 = i4;
  if ((rc = dupload(h, &i4, nb2.data(), S))) return rc;
  T.nb2 = i4;
  int2 *i2;
  if ((rc = dupload(h, &i2, m2e.data(), S))) return rc;
  T.m2e = i2;
  uint8_t *u8;
  if ((rc = dupload(h, &u8, fl.data(), S))) return rc;
  T.fl = u8;
  T.kof = h->G.kof;
  if ((rc = dupload(h, &i4, nbz.data(), S))) return rc;
  T.nbz = i4;
  if ((rc = dupload(h, &i4, colrec.data(), colrec.size()))) return rc;
  T.colrec = i4;
  if ((rc = dupload(h, &ip, colof.data(), S))) return rc;
  T.colof = ip;
  if ((rc = dupload(h, &ip, wet.data(), wet.size()))) return rc;
  T.wet = ip;
  if ((rc = dupload(h, &ip, vdcol.data(), vdcol.size()))) return rc;
  T.vdcol = ip;
  return 0;
}

// Tiles of the fused FP32-mixed kernel: tx x ty water columns, ty = 32 / tx
// (lane = tx * iy + ix for the column at (tx * ti + ix, ty * tj + iy)), in
// row-major tile order so that blocks running at the same time hold
// neighbouring tiles; a tile's lowest layer bounds its layer loop.
int build_fused_tiles(shoc_tr_gpu *h, const shoc_tr_geom *g, const std::vector<int> &col_kb,
                      int tx, shoc_tr_gpu::FusedTiles &out) {
  const int ty = 32 / tx;
  const int ncol = h->ncol;
  int imax = 0, jmax = 0;
  for (int col = 0; col < ncol; col++) {
    const int top = g->w2_t[col + 1];
    if (g->s2i[top] < 0 || g->s2j[top] < 0) return SHOC_TR_EGEOM;
    imax = std::max(imax, g->s2i[top]);
    jmax = std::max(jmax, g->s2j[top]);
  }
  const long long nti = imax / tx + 1, ntj = jmax / ty + 1;
  std::vector<int> tid((size_t)(nti * ntj), -1);
  std::vector<int> tcol, tkmin;
  std::vector<int> order(ncol);
  for (int col = 0; col < ncol; col++) order[col] = col;
  auto key = [&](int col) {
    const int top = g->w2_t[col + 1];
    return (long long)(g->s2j[top] / ty) * nti + g->s2i[top] / tx;
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key(a) < key(b); });
  for (int col : order) {
    const int top = g->w2_t[col + 1];
    const int i = g->s2i[top], j = g->s2j[top];
    int &t = tid[(size_t)key(col)];
    if (t < 0) {
      t = (int)tkmin.size();
      tkmin.push_back(h->nz);
      tcol.insert(tcol.end(), 32, -1);
    }
    const int lane = (j % ty) * tx + i % tx;
    if (tcol[(size_t)t * 32 + lane] >= 0) return SHOC_TR_EGEOM;  // two columns at one (i, j)
    tcol[(size_t)t * 32 + lane] = col;
    tkmin[t] = std::min(tkmin[t], col_kb[col]);
  }
  out.ntile = (int)tkmin.size();
  int *ip;
  int rc;
  if ((rc = dupload(h, &ip, tcol.data(), tcol.size()))) return rc;
  out.tcol = ip;
  if ((rc = dupload(h, &ip, tkmin.data(), tkmin.size()))) return rc;
  out.tkmin = ip;
  return 0;
}

// k_step32's shared memory with nwb phase-B warps, and its reduction group:
// as many advected tracers per phase-A reduction pass as fit the space the
// phase-B arrays leave.
size_t fused_config(const shoc_tr_gpu *h, int nwb, int *ngrp) {
  const int ntb = h->T.ntb;
  const size_t room = (size_t)2 * nwb * h->nz * 32 * 4;
  const size_t buf = (size_t)2 * kStencil * kFusedThreads * 4;
  const int gmax = room > buf ? (int)((room - buf) / fused_red(1)) : 1;
  *ngrp = std::max(1, std::min(std::max(ntb, 1), gmax));
  return fused_smem(h->nz, nwb, ntb, *ngrp);
}

int tile_index(int tx) { return tx == 8 ? 0 : tx == 16 ? 1 : tx == 32 ? 2 : -1; }

void drop_graphs(shoc_tr_gpu *h) {
  for (int i = 0; i < 2; i++)
    if (h->graph[i]) {
      cudaGraphExecDestroy(h->graph[i]);
      h->graph[i] = nullptr;
    }
}

// The launch configuration of the transport kernels (validated; takes
// effect at the next step).
int apply_tuning(shoc_tr_gpu *h, const shoc_tr_tuning &t) {
  const bool f32 = h->esize == sizeof(float);
  if (t.tracers_per_block < 1 || t.tracers_per_block > (f32 ? kVd32MaxWarps : 8))
    return SHOC_TR_EUNSUPPORTED;
  if (t.prefetch && !f32) return SHOC_TR_EUNSUPPORTED;
  const size_t vb = f32 ? vd32_smem(h->nz, t.tracers_per_block, t.prefetch != 0, h->comp)
                        : vd64_smem(h->nz, t.tracers_per_block);
  if (vb > 227 * 1024) return SHOC_TR_EUNSUPPORTED;
  if (t.fused) {
    const int ti = tile_index(t.tile_x);
    if (!f32 || h->comp || !h->fnwb_max || ti < 0 || !h->ftile[ti].tcol) return SHOC_TR_EUNSUPPORTED;
    if (t.phase_b_warps < 1 || t.phase_b_warps > h->fnwb_max) return SHOC_TR_EUNSUPPORTED;
  } else if (f32 && !h->rnd) {
    const int rc = dalloc(h, &h->rnd, (size_t)h->ntr * h->S);
    if (rc) return rc;
  }
  h->tw = t.tracers_per_block;
  h->vd_pf = t.prefetch != 0;
  h->fused = t.fused != 0;
  if (h->fused) {
    const auto &ft = h->ftile[tile_index(t.tile_x)];
    h->fu.tcol = ft.tcol;
    h->fu.tkmin = ft.tkmin;
    h->fu.ntile = ft.ntile;
    h->fu.tx = t.tile_x;
    h->fu.nwb = t.phase_b_warps;
    h->fused_bytes = fused_config(h, t.phase_b_warps, &h->fu.ngrp);
  }
  drop_graphs(h);
  return SHOC_TR_OK;
}

shoc_tr_tuning current_tuning(const shoc_tr_gpu *h) {
  shoc_tr_tuning t;
  t.fused = h->fused ? 1 : 0;
  t.tracers_per_block = h->tw;
  t.tile_x = h->fused ? h->fu.tx : 8;
  t.phase_b_warps = h->fused ? h->fu.nwb : h->fnwb_max;
  t.prefetch = h->vd_pf ? 1 : 0;
  return t;
}

int map_status(int st) {
  if (st & ST_GEOM) return SHOC_TR_EGEOM;
  if (st & ST_PIVOT) return SHOC_TR_EPIVOT;
  if (st & ST_NAN) return SHOC_TR_ENAN;
  if (st & ST_LASTDRY) return SHOC_TR_EUNSUPPORTED;
  if (st & ST_SCRATCH) return SHOC_TR_ESCRATCH;
  return SHOC_TR_OK;
}

int check_geom(const shoc_tr_geom *g, const shoc_tr_opts *o, int ntr) {
  if (!g || !o || ntr < 0) return SHOC_TR_EARG;
  switch (o->trasc) {  // FFSL and LAGRANGE are not built
    case SHOC_TR_QUICKEST: case SHOC_TR_VANLEER: case SHOC_TR_ORDER1: case SHOC_TR_ORDER2:
    case SHOC_TR_ORDER4: case SHOC_TR_QUICKEST_CO: case SHOC_TR_ORDER2_UW: break;
    default: return SHOC_TR_EUNSUPPORTED;
  }
  if (g->v3_t != g->b3_t || g->b3_t != g->a3_t) return SHOC_TR_EUNSUPPORTED;  // OBC / aux cells
  if (g->v2_t != g->b2_t || g->b2_t != g->a2_t) return SHOC_TR_EUNSUPPORTED;
  if (g->nz < 1 || g->nz > kSerialMaxLayers) return SHOC_TR_EUNSUPPORTED;
  if (o->ntr2d) {  // per-column tracer counts: the advected tracers in ascending order
    for (int i = 1; i < o->ntbdy; i++)
      if (o->tbdy[i] <= o->tbdy[i - 1]) return SHOC_TR_EARG;
  }
  if (g->sgsiz < 2 || g->sgsizS < 2 || g->b2_t < 1) return SHOC_TR_EGEOM;
  const int S = g->sgsiz;
  std::vector<uint8_t> wet(S, 0);
  for (int i = 1; i <= g->a3_t; i++) {
    int c = g->w3_t[i];
    if (c < 1 || c >= S) return SHOC_TR_EGEOM;
    wet[c] = 1;
  }
  for (int c = 1; c < S; c++) {
    const int *mp[6] = {g->xp1, g->xm1, g->yp1, g->ym1, g->zp1, g->zm1};
    for (int q = 0; q < 6; q++)
      if (mp[q][c] < 0 || mp[q][c] >= S) return SHOC_TR_EGEOM;
    if (!wet[c]) continue;
    if (g->m2d[c] < 1 || g->m2d[c] >= g->sgsizS) return SHOC_TR_EGEOM;
    // the stencil of the neighbouring face reuses this cell's values
    if (wet[g->xp1[c]] && g->xm1[g->xp1[c]] != c) return SHOC_TR_EGEOM;
    if (wet[g->yp1[c]] && g->ym1[g->yp1[c]] != c) return SHOC_TR_EGEOM;
    if (g->zp1[c] != c && g->zm1[g->zp1[c]] != c) return SHOC_TR_EGEOM;
  }
  for (int cc = 1; cc <= g->b2_t; cc++) {
    int top = g->w2_t[cc], bot = g->bot_t[cc];
    if (top < 1 || top >= g->sgsizS || !wet[top] || bot < 1 || bot >= S || !wet[bot])
      return SHOC_TR_EGEOM;
    if (g->zp1[top] != top || g->s2k[top] != g->nz - 1) return SHOC_TR_EGEOM;
    // bottom reaches the top through zp1 and sits on a self-mapping sediment
    int sed = g->zm1[bot];
    if (sed == bot || wet[sed] || g->zm1[sed] != sed || g->zp1[sed] != bot) return SHOC_TR_EGEOM;
    // and every cell on the way sits one layer above the previous one
    int c = bot, steps = 0;
    const int kb = g->s2k[bot];
    if (kb < 0 || kb >= g->nz) return SHOC_TR_EGEOM;
    while (c != top && steps <= g->nz) {
      if (g->s2k[c] != kb + steps) return SHOC_TR_EGEOM;
      c = g->zp1[c];
      steps++;
    }
    if (c != top || kb + steps != g->nz - 1) return SHOC_TR_EGEOM;
  }
  for (int i = 1; i <= g->nbpt; i++)
    if (g->bpt[i] < 1 || g->bpt[i] >= S || g->bin[i] < 1 || g->bin[i] >= S) return SHOC_TR_EGEOM;
  return SHOC_TR_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C-ABI

// The e1 (e2) face columns of a window as SHOC lists them in w2_e1, bot_e1
// and botzu1 (w2_e2, bot_e2, botzu2): the surface-layer cells of w3_e1, each
// column's deepest w3_e1 cell (the faces are wet from the surface layer
// down to it) and the higher of the floors on the two sides of the face
// (hd_init.c:1443).  bm: the backward map (xm1 or ym1).  False where w3_e1 is
// not one run from the surface layer down in every face column.
bool face_columns(const shoc_tr_geom *g, int ne, const int *w3, const int *bm,
                  std::vector<int2> &fc, std::vector<double> &bz) {
  const int S = g->sgsiz;
  if (ne > 0 && !w3) return false;
  std::vector<uint8_t> in(S, 0);
  for (int i = 1; i <= ne; i++) {
    const int c = w3[i];
    if (c <= 0 || c >= S || in[c]) return false;
    in[c] = 1;
  }
  long long covered = 0;
  for (int i = 1; i <= ne; i++) {
    const int c2 = w3[i];
    if (g->zp1[c2] != c2) continue;  // below the surface layer
    int c = c2, cb = c2;
    while (g->zm1[c] != c && in[c]) {
      cb = c;
      covered++;
      c = g->zm1[c];
    }
    fc.push_back(make_int2(c2, cb));
    const double a = g->botz[bm[c2]], b = g->botz[c2];
    bz.push_back(a > b ? a : b);
  }
  return covered == ne;
}

extern "C" {

const char *shoc_tr_gpu_strerror(int st) {
  switch (st) {
    case SHOC_TR_OK: return "ok";
    case SHOC_TR_ESUBSTEP: return "maximum number of tracer sub-steps exceeded";
    case SHOC_TR_EPIVOT: return "zero pivot in the implicit vertical diffusion solve";
    case SHOC_TR_ENAN: return "NaN in a tracer after the step";
    case SHOC_TR_EGEOM: return "geometry fails the layout checks";
    case SHOC_TR_EUNSUPPORTED: return "unsupported option";
    case SHOC_TR_ECUDA: return "CUDA runtime error";
    case SHOC_TR_EARG: return "bad argument";
    case SHOC_TR_ENOMEM: return "allocation failed";
    case SHOC_TR_ESCRATCH: return "problem larger than the fixed scratch area";
  }
  return "unknown status";
}

void shoc_tr_gpu_destroy(shoc_tr_gpu *h) {
  if (!h) return;
  DeviceScope dev_(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int i = 0; i < 2; i++)
    if (h->graph[i]) cudaGraphExecDestroy(h->graph[i]);
  {
    std::vector<cudaEvent_t> done;  // pairs may share events
    for (auto &e : h->ev)
      for (cudaEvent_t x : {e.a, e.b})
        if (std::find(done.begin(), done.end(), x) == done.end()) done.push_back(x);
    for (cudaEvent_t x : done) cudaEventDestroy(x);
  }
  for (cudaStream_t x : {h->s_up, h->s_dn})
    if (x) cudaStreamSynchronize(x);
  for (cudaEvent_t x : h->pev) cudaEventDestroy(x);
  for (void *p : h->allocs) cudaFree(p);
  if (h->h_dtm) cudaFreeHost(h->h_dtm);
  for (cudaStream_t x : {h->s_up, h->s_dn})
    if (x) cudaStreamDestroy(x);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int shoc_tr_gpu_create(const shoc_tr_geom *g, const shoc_tr_opts *o, int ntr, int precision,
                       int device, shoc_tr_gpu **out) {
  if (!out) return SHOC_TR_EARG;
  *out = nullptr;
  int rc = check_geom(g, o, ntr);
  if (rc) return rc;
  if (precision != SHOC_TR_FP64 && precision != SHOC_TR_FP32_MIXED &&
      precision != SHOC_TR_FP32_COMP)
    return SHOC_TR_EUNSUPPORTED;
  if (precision == SHOC_TR_FP32_MIXED && ntr > kMaxTracers) return SHOC_TR_EUNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || device < 0 || device >= ndev)
    return SHOC_TR_ECUDA;
  shoc_tr_gpu *h = new shoc_tr_gpu();
  h->device = device;
  h->precision = precision;
  h->ntr = ntr;
  h->S = g->sgsiz;
  h->S2 = g->sgsizS;
  h->nz = g->nz;
  h->ncol = g->b2_t;
  h->nbpt = g->nbpt;
#define TRY(x)                \
  do {                        \
    int r_ = (x);             \
    if (r_) {                 \
      shoc_tr_gpu_destroy(h); \
      return r_;              \
    }                         \
  } while (0)
  DeviceScope dev_(device);
  if (!dev_.ok) TRY(SHOC_TR_ECUDA);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    TRY(SHOC_TR_ECUDA);
  const int S = h->S, S2 = h->S2, ncol = h->ncol;

  // ---- host precomputation ----
  std::vector<uint8_t> cflag(S, 0);
  for (int i = 1; i <= g->a3_t; i++) cflag[g->w3_t[i]] |= CF_WET;
  for (int i = 1; i <= g->v3_e1; i++) cflag[g->w3_e1[i]] |= CF_E1;
  for (int i = 1; i <= g->v3_e2; i++) cflag[g->w3_e2[i]] |= CF_E2;
  std::vector<Face2D> fx(S2), fy(S2);
  for (int c2 = 1; c2 < S2; c2++) {
    int xm = g->xm1[c2], xp = g->xp1[c2], ym = g->ym1[c2], yp = g->yp1[c2];
    if (xm >= S2 || xp >= S2 || ym >= S2 || yp >= S2) continue;  // not a 2D cell
    Face2D a, b;
    // d3 / d4 (tracers.c:568-577) and the QUICKEST metric factors (:1862-1864)
    a.d = g->h1acell[xm] / (g->h1acell[xm] + g->h1acell[c2]);
    a.db = 2.0 / (g->h1au1[xm] + g->h1au1[c2]);
    a.df = 2.0 / (g->h1au1[c2] + g->h1au1[xp]);
    a.hm = g->h1au1[xm];
    a.h0 = g->h1au1[c2];
    a.hp = g->h1au1[xp];
    b.d = g->h2acell[ym] / (g->h2acell[ym] + g->h2acell[c2]);
    b.db = 2.0 / (g->h2au2[ym] + g->h2au2[c2]);
    b.df = 2.0 / (g->h2au2[c2] + g->h2au2[yp]);
    b.hm = g->h2au2[ym];
    b.h0 = g->h2au2[c2];
    b.hp = g->h2au2[yp];
    fx[c2] = a;
    fy[c2] = b;
  }
  std::vector<int> col_top(ncol), col_bot(ncol), col_kb(ncol), sur0(ncol, 0);
  for (int cc = 1; cc <= ncol; cc++) {
    col_top[cc - 1] = g->w2_t[cc];
    col_bot[cc - 1] = g->bot_t[cc];
    col_kb[cc - 1] = g->s2k[g->bot_t[cc]];
  }

  // ---- device geometry ----
  Geo &G = h->G;
  G.S = S;
  G.S2 = S2;
  G.nz = g->nz;
  G.ncol = ncol;
  G.v2col = g->v2_t - 1;
  int *ip;
  TRY(dupload(h, &ip, g->xp1, S)); G.xp1 = ip;
  TRY(dupload(h, &ip, g->xm1, S)); G.xm1 = ip;
  TRY(dupload(h, &ip, g->yp1, S)); G.yp1 = ip;
  TRY(dupload(h, &ip, g->ym1, S)); G.ym1 = ip;
  TRY(dupload(h, &ip, g->zp1, S)); G.zp1 = ip;
  TRY(dupload(h, &ip, g->zm1, S)); G.zm1 = ip;
  TRY(dupload(h, &ip, g->m2d, S)); G.m2d = ip;
  uint8_t *u8;
  TRY(dupload(h, &u8, cflag.data(), S)); G.cflag = u8;
  TRY(dupload(h, &ip, col_top.data(), ncol)); G.col_top = ip;
  TRY(dupload(h, &ip, col_bot.data(), ncol)); G.col_bot = ip;
  TRY(dupload(h, &ip, col_kb.data(), ncol)); G.col_kb = ip;
  TRY(dupload(h, &ip, g->s2k, S)); G.kof = ip;
  {
    std::vector<int> colntr(ncol, ntr);
    if (o->ntr2d)
      for (int col = 0; col < ncol; col++)
        colntr[col] = std::max(0, std::min(ntr, o->ntr2d[col_top[col]]));
    TRY(dupload(h, &ip, colntr.data(), ncol)); G.colntr = ip;
  }
  double *dp;
  TRY(dupload(h, &dp, g->h1au1, S2)); G.h1au1 = dp;
  TRY(dupload(h, &dp, g->h2au2, S2)); G.h2au2 = dp;
  TRY(dupload(h, &dp, g->h1au2, S2)); G.h1au2 = dp;
  TRY(dupload(h, &dp, g->h2au1, S2)); G.h2au1 = dp;
  TRY(dupload(h, &dp, g->h1acell, S2)); G.h1acell = dp;
  TRY(dupload(h, &dp, g->h2acell, S2)); G.h2acell = dp;
  TRY(dupload(h, &dp, g->cellarea, S2)); G.cellarea = dp;
  TRY(dupload(h, &dp, g->botz, S2)); G.botz = dp;
  TRY(dupload(h, &dp, g->gridz, S)); G.gridz = dp;
  Face2D *fp;
  TRY(dupload(h, &fp, fx.data(), S2)); G.fx = fp;
  TRY(dupload(h, &fp, fy.data(), S2)); G.fy = fp;
  if (g->nbpt > 0) {
    TRY(dupload(h, &h->bpt, g->bpt + 1, g->nbpt));
    TRY(dupload(h, &h->bin, g->bin + 1, g->nbpt));
  }

  // ---- options and tracers ----
  h->O.trasc = o->trasc;
  // order1 is monotonic and switches the limiter off (tracers.c:497-503)
  h->O.ultimate = o->trasc == SHOC_TR_ORDER1 ? 0 : o->ultimate;
  h->O.tiled = (o->trasc == SHOC_TR_QUICKEST || o->trasc == SHOC_TR_VANLEER) ? 1 : 0;
  h->O.substep =
      (o->stab & (SHOC_TR_SUB_STEP | SHOC_TR_SUB_STEP_NOSURF | SHOC_TR_SUB_STEP_TRACER)) ? 1 : 0;
  h->O.hmin = o->hmin;
  h->trf.assign(ntr, 0);
  std::vector<int> slot;
  for (int i = 0; i < o->ntbdy; i++) {
    int n = o->tbdy[i];
    if (n < 0 || n >= ntr) TRY(SHOC_TR_EARG);
    h->trf[n] |= TR_TBDY;
    if (o->advect[n]) h->trf[n] |= TR_ADV;
    if (o->diffuse[n]) {
      h->trf[n] |= TR_HDIFF;
      h->any_hdiff = true;
    }
    slot.push_back(n);
  }
  for (int i = 0; i < o->ntdif_v; i++) {
    int n = o->tdif_v[i];
    if (n < 0 || n >= ntr) TRY(SHOC_TR_EARG);
    h->trf[n] |= TR_VDIFF;
    h->any_vdiff = true;
  }
  for (int n = 0; n < ntr; n++)
    if (!(h->trf[n] & TR_TBDY)) slot.push_back(n);
  {
    bool all_a = true, all_h = true, no_h = true;
    for (int i = 0; i < o->ntbdy; i++) {
      const uint8_t f = h->trf[o->tbdy[i]];
      all_a = all_a && (f & TR_ADV);
      all_h = all_h && (f & TR_HDIFF);
      no_h = no_h && !(f & TR_HDIFF);
    }
    h->adv_flags = !all_a ? 0 : (no_h ? 1 : (all_h ? 2 : 0));
  }
  h->nslot = (int)slot.size();
  h->slot_host = slot;
  TrSet &T = h->T;
  T.ntr = ntr;
  T.nslot = h->nslot;
  T.ntb = o->ntbdy;
  TRY(dupload(h, &ip, slot.data(), slot.size())); T.slot_tr = ip;
  TRY(dupload(h, &u8, h->trf.data(), ntr)); T.trf = u8;
  TRY(dupload(h, &dp, o->mintr, ntr)); T.mintr = dp;
  TRY(dupload(h, &dp, o->maxtr, ntr)); T.maxtr = dp;

  // ---- work arrays ----
  Work &W = h->W;
  TRY(dupload<double>(h, &W.dz, nullptr, S));
  TRY(dupload<double>(h, &W.w5, nullptr, S));
  TRY(dupload<double>(h, &W.w9, nullptr, S));
  TRY(dupload<double>(h, &W.dbz, nullptr, S));
  TRY(dupload<double>(h, &W.dfz, nullptr, S));
  TRY(dupload<double>(h, &W.w6, nullptr, S));
  TRY(dupload<double>(h, &W.w7, nullptr, S));
  TRY(dupload<double>(h, &W.w8, nullptr, S));
  TRY(dupload<double>(h, &W.vd_cm1, nullptr, S));
  TRY(dupload<double>(h, &W.vd_div, nullptr, S));
  TRY(dupload<double>(h, &W.vd_ud, nullptr, S));
  TRY(dupload<double>(h, &W.vd_dzdt, nullptr, S));
  TRY(dupload<int>(h, &W.sur_t, nullptr, ncol));
  TRY(dupload<int>(h, &W.nsur_t, nullptr, ncol));
  TRY(dupload<ColInfo>(h, &W.col, nullptr, ncol));
  TRY(dupload<int>(h, &W.status, nullptr, 1));
  TRY(dupload<unsigned long long>(h, &W.dtm_bits, nullptr, 1));
  TRY(dupload<unsigned long long>(h, &W.nwarn, nullptr, 1));
  TRY(dupload<int>(h, &W.serial_list, nullptr, ncol));
  TRY(dupload<int>(h, &W.serial_count, nullptr, 1));
  TRY(dupload<int>(h, &h->d_counts, nullptr, 2));
  const bool f32p = precision != SHOC_TR_FP64;
  h->esize = f32p ? sizeof(float) : sizeof(double);
  h->comp = precision == SHOC_TR_FP32_COMP;
  h->staged = true;
  for (int b = 0; b < 2; b++) {
    if (f32p) {
      float *fp = nullptr;
      TRY(dupload<float>(h, &fp, nullptr, (size_t)ntr * S));
      h->tr[b] = fp;
      if (h->comp) TRY(dupload<int16_t>(h, &h->lo[b], nullptr, (size_t)ntr * S));
    } else {
      double *dp2 = nullptr;
      TRY(dupload<double>(h, &dp2, nullptr, (size_t)ntr * S));
      h->tr[b] = dp2;
    }
  }
  if (f32p) {
    TRY(dupload<double>(h, &h->xfer, nullptr, S));
    TRY(dupload<float>(h, &W.dz32, nullptr, S));
    TRY(dupload<float4>(h, &W.lu32, nullptr, S));
    float *fp;
    TRY(dupload<float>(h, &fp, nullptr, S)); h->F3.u1 = fp;
    TRY(dupload<float>(h, &fp, nullptr, S)); h->F3.u2 = fp;
    TRY(dupload<float>(h, &fp, nullptr, S)); h->F3.w = fp;
    if (h->any_hdiff) {
      TRY(dupload<float>(h, &fp, nullptr, S)); h->F3.khx = fp;
      TRY(dupload<float>(h, &fp, nullptr, S)); h->F3.khy = fp;
    }
    // per-column metric factors of the FP32 face values
    std::vector<f32::Face2> ax(S2), ay(S2);
    for (int c2 = 1; c2 < S2; c2++) {
      const Face2D &a = fx[c2], &b = fy[c2];
      ax[c2] = {(float)a.d, (float)(a.db * a.hm), (float)(a.db * a.h0), (float)(a.df * a.h0),
                (float)(a.df * a.hp), a.h0 != 0.0 ? (float)(1.0 / a.h0) : 0.f};
      ay[c2] = {(float)b.d, (float)(b.db * b.hm), (float)(b.db * b.h0), (float)(b.df * b.h0),
                (float)(b.df * b.hp), b.h0 != 0.0 ? (float)(1.0 / b.h0) : 0.f};
    }
    TRY(dupload(h, &h->fx2, ax.data(), S2));
    TRY(dupload(h, &h->fy2, ay.data(), S2));
    // the FP64 mass each column's stored values owe it
    TRY(dupload<double>(h, &h->fu.carry, nullptr, (size_t)ntr * ncol));
  }
  TRY(dupload<double>(h, &h->fzs64, nullptr, (size_t)ntr * ncol));
  // tiling: tracers per block
  int tw = 8;
  {
    // tracers (k_vd64) or warps (k_vd32) per column-kernel block: two
    // blocks per SM at full depth, balanced rounds over the tracers (on
    // stiff2048 two blocks of 4 warps beat one block of 12: 9.4 against
    // 11.5 ms for k_vd32)
    while (tw > 1 && vd_smem(h, g->nz, tw) > 113 * 1024) tw--;
    int nch = (h->nslot + tw - 1) / std::max(tw, 1);
    if (nch > 0) tw = (h->nslot + nch - 1) / nch;
    if (tw < 1) tw = 1;
  }
  h->tw = tw;
  TRY(build_tile_tables(h, g, cflag, col_bot, col_kb));
  {  // face columns of the transport-mode preamble
    std::vector<int2> fc;
    std::vector<double> bz;
    bool ok = face_columns(g, g->v3_e1, g->w3_e1, g->xm1, fc, bz);
    const int n1 = (int)fc.size();
    ok = ok && face_columns(g, g->v3_e2, g->w3_e2, g->ym1, fc, bz);
    h->pre.ok = ok;
    if (ok && !fc.empty()) {
      h->pre.n1 = n1;
      h->pre.n2 = (int)fc.size() - n1;
      TRY(dupload(h, &h->pre.fc, fc.data(), fc.size()));
      TRY(dupload(h, &h->pre.bz, bz.data(), bz.size()));
    }
  }
  if (f32p) {
    // the fused sub-step kernel k_step32: every advected tracer's
    // accumulators and the column arrays of up to as many phase-B warps as
    // keep two blocks per SM; tiles of every width the autotuner may choose
    // (not with FP32_COMP: k_step32 keeps no compensation)
    if (o->ntbdy <= kFusedMaxTracers && !h->comp) {
      for (int c = kFusedWarps; c >= 1 && !h->fnwb_max; c--) {
        int gq;
        if (fused_config(h, c, &gq) <= 113 * 1024) h->fnwb_max = c;
      }
    }
    if (h->fnwb_max) {
      int gq;
      if (fused32_set_smem_attr((int)fused_config(h, h->fnwb_max, &gq)) != cudaSuccess)
        TRY(SHOC_TR_ECUDA);
      for (int tx : {8, 16, 32}) TRY(build_fused_tiles(h, g, col_kb, tx, h->ftile[tile_index(tx)]));
    }
    // the two-kernel sub-step is the default (measured faster);
    // SHOC_TR_GPU_KERNELS=fused starts with k_step32 (8 x 4 tiles)
    const char *env = getenv("SHOC_TR_GPU_KERNELS");
    shoc_tr_tuning t0 = current_tuning(h);
    if (env && strcmp(env, "fused") == 0 && h->fnwb_max && !h->comp) {
      t0.fused = 1;
      t0.tile_x = 8;
      t0.phase_b_warps = h->fnwb_max;
    }
    TRY(apply_tuning(h, t0));
  }
  // flow fields
  Flow &F = h->F;
  TRY(dupload<double>(h, (double **)&F.u1, nullptr, S));
  TRY(dupload<double>(h, (double **)&F.u2, nullptr, S));
  TRY(dupload<double>(h, (double **)&F.w, nullptr, S));
  TRY(dupload<double>(h, (double **)&F.u1flux3d, nullptr, S));
  TRY(dupload<double>(h, (double **)&F.u2flux3d, nullptr, S));
  TRY(dupload<double>(h, (double **)&F.Kz, nullptr, S));
  if (f32p) {  // the FP32-mixed kernels take the FP64 volume fluxes
    h->F3.u1flux3d = F.u1flux3d;
    h->F3.u1_64 = F.u1;
    h->F3.u2_64 = F.u2;
    h->F3.u2flux3d = F.u2flux3d;
    h->F3.w64 = F.w;
  }
  if (h->any_hdiff) {
    TRY(dupload<double>(h, (double **)&F.dzu1, nullptr, S));
    TRY(dupload<double>(h, (double **)&F.dzu2, nullptr, S));
    TRY(dupload<double>(h, (double **)&F.u1kh, nullptr, S));
    TRY(dupload<double>(h, (double **)&F.u2kh, nullptr, S));
  }
  TRY(dupload<double>(h, (double **)&F.eta, nullptr, S2));
  TRY(dupload<double>(h, (double **)&F.oldeta, nullptr, S2));
  // pinned readback words
  void *pin = nullptr;
  if (cudaHostAlloc(&pin, 64, cudaHostAllocDefault) != cudaSuccess) TRY(SHOC_TR_ENOMEM);
  h->h_dtm = (unsigned long long *)pin;
  h->h_status = (int *)((char *)pin + 8);
  h->h_nwarn = (unsigned long long *)((char *)pin + 16);
  h->h_counts = (int *)((char *)pin + 24);
  if (cudaFuncSetAttribute(k_vd64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           227 * 1024) != cudaSuccess ||
      cudaFuncSetAttribute(k_vd64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           227 * 1024) != cudaSuccess ||
      tile32_set_smem_attr() != cudaSuccess)
    TRY(SHOC_TR_ECUDA);
#undef TRY
  *out = h;
  return SHOC_TR_OK;
}

}  // extern "C"

namespace {

// Sub-step schedule from the device minimum (tracers.c:591-668, :715-720).
int make_schedule(shoc_tr_gpu *h, double dmin, Sched &s) {
  double dt = h->dt, dtm = dt;
  if (h->O.substep) {
    if (dmin < dtm) dtm = dmin;
    if (dtm != dt) dtm = floor(dtm);
  }
  s.dtm = dtm;
  s.sub.clear();
  if (dtm == 0.0 || (int)(dt / dtm) > kItermax) return SHOC_TR_ESUBSTEP;
  double trem = dt, prev_f = 0.0;
  bool first = true;
  while (trem > 0) {
    double dtu = dtm;
    if (trem < dtu) dtu = trem;
    if (dtu > 0.0) {
      SubStep ss;
      ss.dtu = dtu;
      ss.trem = trem;
      ss.subeta_f = 1.0 + (dtu - trem) / dt;
      ss.osub_f = prev_f;
      ss.first = first ? 1 : 0;
      prev_f = ss.subeta_f;
      first = false;
      s.sub.push_back(ss);
    }
    trem -= dtu;
  }
  return SHOC_TR_OK;
}

// set_lateral_BC_tr for the tracers of T (every tracer, or one chunk of the
// drop-in step's pipeline) into both buffers
void launch_lateral(shoc_tr_gpu *h, int cur, const TrSet &T) {
  if (h->nbpt <= 0 || T.nslot <= 0) return;
  cudaStream_t st = h->stream;
  long long tot = (long long)h->nbpt * T.nslot;
  int blocks = (int)std::min<long long>((tot + 255) / 256, 148 * 16);
  if (h->esize == sizeof(float))
    k_lateral<float><<<blocks, 256, 0, st>>>(h->nbpt, h->bpt, h->bin, T.slot_tr, T.nslot, h->S,
                                             (float *)h->tr[cur], (float *)h->tr[cur ^ 1],
                                             h->comp ? h->lo[cur] : nullptr,
                                             h->comp ? h->lo[cur ^ 1] : nullptr);
  else
    k_lateral<double><<<blocks, 256, 0, st>>>(h->nbpt, h->bpt, h->bin, T.slot_tr, T.nslot,
                                              h->S, (double *)h->tr[cur],
                                              (double *)h->tr[cur ^ 1]);
  h->launches++;
}

// The transport-mode flow preamble: dzu1, dzu2, u1flux3d, u2flux3d and w
// from the velocities, the surface and detadt (k_faces, k_wvel), and the
// FP32-mixed path's copies of what changed.
int launch_preamble(shoc_tr_gpu *h) {
  cudaStream_t st = h->stream;
  const size_t S = (size_t)h->S;
  double *f1 = (double *)h->F.u1flux3d, *f2 = (double *)h->F.u2flux3d, *w = (double *)h->F.w;
  double *d1 = (double *)h->F.dzu1, *d2 = (double *)h->F.dzu2;
  for (double *p : {f1, f2, w, d1, d2}) CK(cudaMemsetAsync(p, 0, S * sizeof(double), st));
  const int n = h->pre.n1 + h->pre.n2;
  if (n > 0) {
    k_faces<<<(n + 127) / 128, 128, 0, st>>>(h->G, h->F, h->pre.n1, n, h->pre.fc, h->pre.bz, d1,
                                             d2, f1, f2);
    h->launches++;
  }
  k_wvel<<<(h->ncol + 127) / 128, 128, 0, st>>>(h->G, h->F, h->W, h->O, h->pre.detadt, w);
  h->launches++;
  if (h->esize == sizeof(float)) {
    k_to_f32<<<592, 256, 0, st>>>(h->F.w, (float *)h->F3.w, S);
    h->launches++;
    if (h->any_hdiff) {
      k_khfac<<<592, 256, 0, st>>>(h->G, h->F, (float *)h->F3.khx, (float *)h->F3.khy);
      h->launches++;
    }
  }
  CK(cudaGetLastError());
  return 0;
}

// Step set-up: counters, lateral boundaries (when `lateral`), the flow
// preamble (when on) and k_set_dz.  k_set_dz reads no tracer, so the lateral
// copies may follow it instead.
int launch_part_a(shoc_tr_gpu *h, int cur, bool lateral = true) {
  cudaStream_t st = h->stream;
  k_reset<<<1, 32, 0, st>>>(h->W, h->d_counts);
  h->launches++;
  if (lateral) launch_lateral(h, cur, h->T);
  if (h->pre.on) {
    const int rc = launch_preamble(h);
    if (rc) return rc;
  }
  int nb = (h->ncol + 127) / 128;
  k_set_dz<<<nb, 128, 0, st>>>(h->G, h->F, h->W, h->O, h->tl, h->any_vdiff ? 1 : 0, h->d_counts,
                               h->staged ? 1 : 0, h->esize == sizeof(float) ? 1 : 0, h->colown,
                               0);
  h->launches++;
  CK(cudaGetLastError());
  return 0;
}

// One FP64 transport sub-step over the staged columns: k_adv64, then one
// k_vd64 launch per depth class.  Returns the kernels launched.
template <bool Q, bool U, int M>
void adv64(const shoc_tr_gpu *h, int grid, const SubStep &ss, const Tile &tl, const TrSet &T,
           const double *tin, double *tout) {
  k_adv64<Q, U, M><<<grid, kAdvBlock, 0, h->stream>>>(h->G, h->F, h->W, T, ss, tl, tin, tout,
                                                      h->fzs64, h->any_hdiff ? 1 : 0);
}
template <bool Q, bool U>
void adv64_mode(const shoc_tr_gpu *h, int grid, const SubStep &ss, const Tile &tl,
                const TrSet &T, const double *tin, double *tout) {
  if (h->adv_flags == 1)
    adv64<Q, U, 1>(h, grid, ss, tl, T, tin, tout);
  else if (h->adv_flags == 2)
    adv64<Q, U, 2>(h, grid, ss, tl, T, tin, tout);
  else
    adv64<Q, U, 0>(h, grid, ss, tl, T, tin, tout);
}
int tile64_substep(const shoc_tr_gpu *h, bool last, const SubStep &ss, const Tile &tl,
                   const TrSet &T, const double *tin, double *tout, int nw, cudaEvent_t *ev) {
  cudaStream_t st = h->stream;
  int nl = 0;
  if (ev) cudaEventRecord(ev[0], st);
  if (T.ntb > 0 && tl.nwet > 0) {
    const int grid = (tl.nwet + kAdvBlock - 1) / kAdvBlock;
    const bool q = h->O.trasc == SHOC_TR_QUICKEST, u = h->O.ultimate != 0;
    if (q && u)
      adv64_mode<true, true>(h, grid, ss, tl, T, tin, tout);
    else if (q)
      adv64_mode<true, false>(h, grid, ss, tl, T, tin, tout);
    else if (u)
      adv64_mode<false, true>(h, grid, ss, tl, T, tin, tout);
    else
      adv64_mode<false, false>(h, grid, ss, tl, T, tin, tout);
    nl++;
  }
  if (ev) cudaEventRecord(ev[1], st);
  const int nchunk = (T.nslot + nw - 1) / nw;
  const dim3 blk(32, nw);
  for (int i = 0; i < tl.nclass; i++) {
    const int t0 = tl.ctile[i], nt = tl.ctile[i + 1] - t0, kbase = tl.cbase[i];
    if (nt <= 0) continue;
    const size_t smem = vd64_smem(h->nz - kbase, nw);
    if (last)
      k_vd64<true><<<nt * nchunk, blk, smem, st>>>(
          h->G, h->F, h->W, h->O, T, ss, tl, tin, tout, h->fzs64, h->W.vd_dzdt, h->W.vd_cm1,
          h->W.vd_div, h->W.vd_ud, nw, nchunk, t0, kbase);
    else
      k_vd64<false><<<nt * nchunk, blk, smem, st>>>(
          h->G, h->F, h->W, h->O, T, ss, tl, tin, tout, h->fzs64, h->W.vd_dzdt, h->W.vd_cm1,
          h->W.vd_div, h->W.vd_ud, nw, nchunk, t0, kbase);
    nl++;
  }
  if (ev) cudaEventRecord(ev[2], st);
  return nl;
}

// Depth classes of the k_vd32 launches for nw tracers per block: the deepest
// tile that still lets 4, 3 and 2 blocks share an SM's shared memory bounds
// a class; each class is launched with shared memory for its own depth.
Tile vd_classes(const shoc_tr_gpu *h, int nw) {
  Tile t = h->tl;
  const int ntile = (int)h->vd_depth.size();
  const size_t per_layer = vd_smem(h, 1, nw);
  const size_t sm = 233472, rsv = 1024;
  t.nclass = 0;
  t.ctile[0] = 0;
  int start = 0;
  for (int blocks = 4; blocks >= 1 && start < ntile; blocks--) {
    int dmax = (int)((sm / blocks - rsv) / per_layer);
    if (blocks == 1 || dmax >= h->nz) dmax = h->nz;
    int end = start;
    while (end < ntile && h->vd_depth[end] <= dmax) end++;
    if (end == start) continue;
    t.cbase[t.nclass] = h->nz - h->vd_depth[end - 1];
    t.ctile[++t.nclass] = end;
    start = end;
    if (dmax == h->nz) break;
  }
  return t;
}

// The transport sub-steps of one step for the tracers of T (every tracer, or
// one chunk of the drop-in step's pipeline; c3s/c3_load as k_serial takes
// them, one row of ncol bytes per sub-step).
int launch_part_b(shoc_tr_gpu *h, const Sched &s, int cur0, const TrSet &T,
                  uint8_t *c3s = nullptr, bool c3_load = false) {
  cudaStream_t st = h->stream;
  int cur = cur0;
  const int nsub = (int)s.sub.size();
  const int tw = std::max(1, std::min(h->tw, T.nslot));  // no idle tracer rows
  int cblocks = std::min((h->S + 255) / 256, 148 * 32);
  for (int i = 0; i < nsub; i++) {
    const SubStep &ss = s.sub[i];
    bool last = (i == nsub - 1);
    uint8_t *c3row = c3s ? c3s + (size_t)i * h->ncol : nullptr;
    k_courant<<<cblocks, 256, 0, st>>>(h->G, h->F, h->W, ss.dtu, h->staged ? 1 : 0);
    h->launches++;
    if (h->esize == sizeof(float) && T.nslot > 0) {  // FP32-mixed
      const float *tin = (const float *)h->tr[cur];
      float *tout = (float *)h->tr[cur ^ 1];
      bool prof = h->profile && last;
      cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
      if (prof)
        for (auto &e : ev) cudaEventCreate(&e);
      if (h->fused) {
        if (prof) cudaEventRecord(ev[0], st);
        fused32_substep(last, h->O.trasc == SHOC_TR_QUICKEST, h->O.ultimate != 0, st, h->G, h->F,
                        h->F3, h->W, h->O, T, ss, h->tl, h->fu, h->fx2, h->fy2, tin, tout,
                        h->any_hdiff ? 1 : 0, h->fused_bytes);
        if (prof) {
          cudaEventRecord(ev[1], st);
          h->ev.push_back({0, ev[0], ev[1]});
          h->ev.push_back({1, ev[0], ev[1]});
          cudaEventDestroy(ev[2]);
        }
        h->launches += h->fu.ntile > 0 ? 1 : 0;
      } else {
        const Tile tl = vd_classes(h, tw);
        tile32_substep(last, h->O.trasc == SHOC_TR_QUICKEST, h->O.ultimate != 0, st, h->G, h->F,
                       h->F3, h->W, h->O, T, ss, tl, h->fx2, h->fy2, tin, tout, h->rnd,
                       h->fu.carry, h->fzs64, h->comp ? h->lo[cur] : nullptr,
                       h->comp ? h->lo[cur ^ 1] : nullptr, tw, h->vd_pf ? 1 : 0,
                       h->any_hdiff ? 1 : 0, h->adv_flags, prof ? ev : nullptr);
        if (prof) {  // pairs share events; sync destroys each event once
          h->ev.push_back({0, ev[0], ev[2]});
          h->ev.push_back({1, ev[0], ev[1]});
          h->ev.push_back({2, ev[1], ev[2]});
        }
        h->launches += (T.ntb > 0 && tl.nwet > 0 ? 1 : 0);
        for (int k = 0; k < tl.nclass; k++) h->launches += tl.ctile[k + 1] > tl.ctile[k] ? 1 : 0;
      }
      int16_t *lo_out = h->comp ? h->lo[cur ^ 1] : nullptr;
      if (last)
        k_serial<true, float><<<kSerialBlocks, 64, 0, st>>>(h->G, h->F, h->W, h->O, T, ss,
                                                            tin, tout, c3row, c3_load, lo_out);
      else
        k_serial<false, float><<<kSerialBlocks, 64, 0, st>>>(h->G, h->F, h->W, h->O, T, ss,
                                                             tin, tout, c3row, c3_load, lo_out);
      h->launches++;
      cur ^= 1;
      continue;
    }
    const double *tin = (const double *)h->tr[cur];
    double *tout = (double *)h->tr[cur ^ 1];
    if (T.nslot > 0) {
      bool prof = h->profile && last;
      cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
      if (prof)
        for (auto &e : ev) cudaEventCreate(&e);
      const Tile tl = vd_classes(h, tw);
      const int nl = tile64_substep(h, last, ss, tl, T, tin, tout, tw, prof ? ev : nullptr);
      if (prof) {
        h->ev.push_back({0, ev[0], ev[2]});
        h->ev.push_back({1, ev[0], ev[1]});
        h->ev.push_back({2, ev[1], ev[2]});
      }
      h->launches += nl;
      if (last)
        k_serial<true, double><<<kSerialBlocks, 64, 0, st>>>(h->G, h->F, h->W, h->O, T, ss,
                                                             tin, tout, c3row, c3_load);
      else
        k_serial<false, double><<<kSerialBlocks, 64, 0, st>>>(h->G, h->F, h->W, h->O, T, ss,
                                                              tin, tout, c3row, c3_load);
      h->launches++;
    }
    cur ^= 1;
  }
  CK(cudaGetLastError());
  return 0;
}

int read_status(shoc_tr_gpu *h) {
  CK(cudaMemcpyAsync(h->h_dtm, h->W.dtm_bits, 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(h->h_status, h->W.status, 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(h->h_counts, h->d_counts, 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

// Part A of a step whose sub-step schedule is not known yet, then the
// sub-step minimum read back and the schedule built from it (tracers.c:
// 591-720).  lateral: whether part A fills every tracer's lateral boundary.
int probe_schedule(shoc_tr_gpu *h, bool lateral, Sched &s) {
  int rc = launch_part_a(h, h->cur, lateral);
  if (rc) return rc;
  rc = read_status(h);
  if (rc) return rc;
  int st = *h->h_status;
  if (st & (ST_LASTDRY | ST_GEOM)) {
    h->last_status = map_status(st);
    return h->last_status;
  }
  double dmin;
  unsigned long long b = *h->h_dtm;
  memcpy(&dmin, &b, 8);
  if (h->dmin_set > 0.0) dmin = h->dmin_set;  // the basin-wide minimum, given
  rc = make_schedule(h, dmin, s);
  if (rc) h->last_status = rc;
  return rc;
}

// Keep a probed schedule for the graph-replayed steps; graphs made for
// another schedule are dropped.
void adopt_schedule(shoc_tr_gpu *h, const Sched &s) {
  bool same = h->have_sched && s.sub.size() == h->sched.sub.size();
  if (same)
    for (size_t i = 0; i < s.sub.size(); i++)
      if (memcmp(&s.sub[i], &h->sched.sub[i], sizeof(SubStep)) != 0) same = false;
  if (!same) {
    for (int i = 0; i < 2; i++)
      if (h->graph[i]) {
        cudaGraphExecDestroy(h->graph[i]);
        h->graph[i] = nullptr;
      }
  }
  h->sched = s;
  h->have_sched = true;
  if (h->probe_left > 0) h->probe_left--;
}

// One step.  When the schedule is not yet known the step synchronises after
// k_set_dz to read the sub-step minimum; afterwards steps replay a graph.
int step_async(shoc_tr_gpu *h) {
  if (h->probe_left > 0 || !h->have_sched) {
    Sched s;
    int rc = probe_schedule(h, true, s);
    if (rc) return rc;
    rc = launch_part_b(h, s, h->cur, h->T);
    if (rc) return rc;
    if (s.sub.size() & 1) h->cur ^= 1;
    adopt_schedule(h, s);
    return 0;
  }
  if (h->profile) {
    // profiling launches directly so each transport launch is timed
    int rc = launch_part_a(h, h->cur);
    if (rc) return rc;
    rc = launch_part_b(h, h->sched, h->cur, h->T);
    if (rc) return rc;
    if (h->sched.sub.size() & 1) h->cur ^= 1;
    return 0;
  }
  int gi = h->cur;
  if (!h->graph[gi]) {
    // An odd number of sub-steps alternates the buffers from step to step:
    // both graphs are captured and uploaded together, so no later step pays
    // for a capture or a first upload.
    const int ng = (h->sched.sub.size() & 1) ? 2 : 1;
    for (int k = 0; k < ng; ++k) {
      const int g = gi ^ k;
      if (h->graph[g]) continue;
      cudaGraph_t graph;
      long long l0 = h->launches;
      CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      int rc = launch_part_a(h, g);
      if (!rc) rc = launch_part_b(h, h->sched, g, h->T);
      cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
      if (rc) return rc;
      CK(e);
      CK(cudaGraphInstantiate(&h->graph[g], graph, 0));
      cudaGraphDestroy(graph);
      CK(cudaGraphUpload(h->graph[g], h->stream));
      h->graph_launches[g] = h->launches - l0;  // kernels in the graph
      h->launches = l0;
    }
  }
  CK(cudaGraphLaunch(h->graph[gi], h->stream));
  h->launches += h->graph_launches[gi];
  if (h->sched.sub.size() & 1) h->cur ^= 1;
  return 0;
}

// ---------------------------------------------------------------------------
// The drop-in step on host arrays, pipelined.  The tracers cross the host
// link in chunks of slots: chunk j goes up on one copy stream, is stepped on
// the main stream and comes back on a second copy stream, so the way back of
// chunk j overlaps the way up of the chunks after it (the link is full
// duplex) and every chunk's transport overlaps both.  Per tracer the kernels
// and their order are those of a whole step: the tracers of a step are
// independent apart from the general path's thin-surface cursor, which
// k_serial carries from chunk to chunk (c3s); set_dz reads no tracer, so the
// lateral boundaries of a chunk may follow it.

// slots per chunk: about a twelfth of the tracers, so the first chunk is
// back on its way while most are still going up and the last chunk's step
// and copy back (the part nothing overlaps) are short
int pipe_chunk_slots(const shoc_tr_gpu *h) { return std::max(1, (h->nslot + 11) / 12); }

int pipe_init(shoc_tr_gpu *h) {
  if (h->s_up) return 0;
  CK(cudaStreamCreateWithFlags(&h->s_up, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&h->s_dn, cudaStreamNonBlocking));
  if (h->esize == sizeof(float)) {
    int rc = dalloc(h, &h->xout, (size_t)h->S);
    if (rc) return rc;
  }
  int rc = dalloc(h, &h->c3s, (size_t)(kItermax + 2) * h->ncol);
  if (rc) return rc;
  h->pev.assign(1 + 2 * (size_t)h->nslot, nullptr);
  for (auto &e : h->pev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return 0;
}

// wait for every copy that may still touch the caller's host arrays
void pipe_drain(shoc_tr_gpu *h) {
  cudaStreamSynchronize(h->s_up);
  cudaStreamSynchronize(h->s_dn);
  cudaStreamSynchronize(h->stream);
}

int up_tracer(shoc_tr_gpu *h, int cur, int n, const double *src) {
  cudaStream_t s = h->s_up;
  const size_t S = (size_t)h->S;
  if (h->esize == sizeof(double)) {
    double *a = (double *)h->tr[cur] + n * S, *b = (double *)h->tr[cur ^ 1] + n * S;
    CK(cudaMemcpyAsync(a, src, S * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(b, a, S * sizeof(double), cudaMemcpyDeviceToDevice, s));
  } else {
    float *a = (float *)h->tr[cur] + n * S, *b = (float *)h->tr[cur ^ 1] + n * S;
    CK(cudaMemcpyAsync(h->xfer, src, S * sizeof(double), cudaMemcpyHostToDevice, s));
    k_to_f32x2<<<592, 256, 0, s>>>(h->xfer, a, b, S, h->comp ? h->lo[cur] + n * S : nullptr,
                                   h->comp ? h->lo[cur ^ 1] + n * S : nullptr);
    h->launches++;
  }
  return 0;
}

int down_tracer(shoc_tr_gpu *h, int buf, int n, double *dst) {
  cudaStream_t s = h->s_dn;
  const size_t S = (size_t)h->S;
  if (h->esize == sizeof(double)) {
    CK(cudaMemcpyAsync(dst, (double *)h->tr[buf] + n * S, S * sizeof(double),
                       cudaMemcpyDeviceToHost, s));
  } else {
    k_to_f64<<<592, 256, 0, s>>>((float *)h->tr[buf] + n * S, h->xout, S,
                                 h->comp ? h->lo[buf] + n * S : nullptr);
    h->launches++;
    CK(cudaMemcpyAsync(dst, h->xout, S * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  return 0;
}

int step_pipelined(shoc_tr_gpu *h, shoc_tr_state *st) {
  int rc = pipe_init(h);
  if (rc) return rc;
  rc = shoc_tr_gpu_set_flow(h, st);
  if (rc) return rc;
  const int cur = h->cur, csl = pipe_chunk_slots(h);
  const int nch = (h->nslot + csl - 1) / csl;
  cudaEvent_t *ev = h->pev.data();  // [0] flow sent, [1 + 2j] chunk j sent, [2 + 2j] stepped
  // the tracers follow the flow fields up the link
  CK(cudaEventRecord(ev[0], h->stream));
  CK(cudaStreamWaitEvent(h->s_up, ev[0], 0));
  for (int j = 0; j < nch; j++) {
    for (int sl = j * csl; sl < std::min(h->nslot, (j + 1) * csl); sl++) {
      const int n = h->slot_host[sl];
      rc = up_tracer(h, cur, n, st->tr_wc[n]);
      if (rc) {
        pipe_drain(h);
        return rc;
      }
    }
    CK(cudaEventRecord(ev[1 + 2 * j], h->s_up));
  }
  // the schedule from this step's flow, while the tracers travel
  Sched s;
  rc = probe_schedule(h, false, s);
  if (!rc && s.sub.size() > (size_t)kItermax + 2) rc = SHOC_TR_ESUBSTEP;
  if (rc) {
    pipe_drain(h);
    return rc;
  }
  const int fin = cur ^ (int)(s.sub.size() & 1);  // the buffer the step ends in
  for (int j = 0; j < nch; j++) {
    const int s0 = j * csl, ns = std::min(h->nslot - s0, csl);
    TrSet Tc = h->T;
    Tc.slot_tr = h->T.slot_tr + s0;
    Tc.nslot = ns;
    Tc.ntb = std::max(0, std::min(h->T.ntb - s0, ns));
    CK(cudaStreamWaitEvent(h->stream, ev[1 + 2 * j], 0));
    launch_lateral(h, cur, Tc);
    rc = launch_part_b(h, s, cur, Tc, h->c3s, j > 0);
    if (rc) {
      pipe_drain(h);
      return rc;
    }
    CK(cudaEventRecord(ev[2 + 2 * j], h->stream));
    CK(cudaStreamWaitEvent(h->s_dn, ev[2 + 2 * j], 0));
    for (int sl = s0; sl < s0 + ns; sl++) {
      const int n = h->slot_host[sl];
      rc = down_tracer(h, fin, n, st->tr_wc[n]);
      if (rc) {
        pipe_drain(h);
        return rc;
      }
    }
  }
  // the main stream (and so the status read after it) waits for the way back
  CK(cudaEventRecord(ev[0], h->s_dn));
  CK(cudaStreamWaitEvent(h->stream, ev[0], 0));
  h->cur = fin;
  adopt_schedule(h, s);
  return 0;
}

}  // namespace

extern "C" {

int shoc_tr_gpu_upload_tracers(shoc_tr_gpu *h, double *const *tr_wc) {
  if (!h || !tr_wc) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  const size_t S = (size_t)h->S;
  // new values: nothing is owed to any column
  if (h->fu.carry)
    CK(cudaMemsetAsync(h->fu.carry, 0, (size_t)h->ntr * h->ncol * sizeof(double), h->stream));
  for (int n = 0; n < h->ntr; n++) {
    if (h->esize == sizeof(double)) {
      double *a = (double *)h->tr[h->cur] + n * S, *b = (double *)h->tr[h->cur ^ 1] + n * S;
      CK(cudaMemcpyAsync(a, tr_wc[n], S * sizeof(double), cudaMemcpyHostToDevice, h->stream));
      CK(cudaMemcpyAsync(b, a, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    } else {
      float *a = (float *)h->tr[h->cur] + n * S, *b = (float *)h->tr[h->cur ^ 1] + n * S;
      CK(cudaMemcpyAsync(h->xfer, tr_wc[n], S * sizeof(double), cudaMemcpyHostToDevice,
                         h->stream));
      k_to_f32x2<<<592, 256, 0, h->stream>>>(h->xfer, a, b, S,
                                             h->comp ? h->lo[h->cur] + n * S : nullptr,
                                             h->comp ? h->lo[h->cur ^ 1] + n * S : nullptr);
      h->launches++;
    }
  }
  return 0;
}

int shoc_tr_gpu_download_tracers(shoc_tr_gpu *h, double **tr_wc) {
  if (!h || !tr_wc) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  const size_t S = (size_t)h->S;
  for (int n = 0; n < h->ntr; n++) {
    if (h->esize == sizeof(double)) {
      CK(cudaMemcpyAsync(tr_wc[n], (double *)h->tr[h->cur] + n * S, S * sizeof(double),
                         cudaMemcpyDeviceToHost, h->stream));
    } else {
      k_to_f64<<<592, 256, 0, h->stream>>>((float *)h->tr[h->cur] + n * S, h->xfer, S,
                                           h->comp ? h->lo[h->cur] + n * S : nullptr);
      h->launches++;
      CK(cudaMemcpyAsync(tr_wc[n], h->xfer, S * sizeof(double), cudaMemcpyDeviceToHost,
                         h->stream));
    }
  }
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int shoc_tr_gpu_set_flow(shoc_tr_gpu *h, const shoc_tr_state *st) {
  if (!h || !st) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  const size_t S = (size_t)h->S * sizeof(double), S2 = (size_t)h->S2 * sizeof(double);
  cudaStream_t s = h->stream;
  // with the flow preamble on, w, u1flux3d, u2flux3d, dzu1 and dzu2 are
  // computed by every step and not read from the state (they may be null)
  const bool pre = h->pre.on;
  const struct {
    const double *dst;
    const double *src;
    size_t n;
    bool need;
  } cp[] = {{h->F.u1, st->u1, S, true},
            {h->F.u2, st->u2, S, true},
            {h->F.w, st->w, S, !pre},
            {h->F.u1flux3d, st->u1flux3d, S, !pre},
            {h->F.u2flux3d, st->u2flux3d, S, !pre},
            {h->F.Kz, st->Kz, S, true},
            {h->F.eta, st->eta, S2, true},
            {h->F.oldeta, st->oldeta, S2, true}};
  for (auto &x : cp) {
    if (!x.need) continue;
    if (!x.src) return SHOC_TR_EARG;
    CK(cudaMemcpyAsync((void *)x.dst, x.src, x.n, cudaMemcpyHostToDevice, s));
  }
  if (h->any_hdiff) {
    if ((!pre && (!st->dzu1 || !st->dzu2)) || !st->u1kh || !st->u2kh) return SHOC_TR_EARG;
    if (!pre) {
      CK(cudaMemcpyAsync((void *)h->F.dzu1, st->dzu1, S, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync((void *)h->F.dzu2, st->dzu2, S, cudaMemcpyHostToDevice, s));
    }
    CK(cudaMemcpyAsync((void *)h->F.u1kh, st->u1kh, S, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync((void *)h->F.u2kh, st->u2kh, S, cudaMemcpyHostToDevice, s));
  }
  if (h->esize == sizeof(float)) {
    const size_t n = (size_t)h->S;
    k_to_f32<<<592, 256, 0, s>>>(h->F.u1, (float *)h->F3.u1, n);
    k_to_f32<<<592, 256, 0, s>>>(h->F.u2, (float *)h->F3.u2, n);
    h->launches += 2;
    if (!pre) {
      k_to_f32<<<592, 256, 0, s>>>(h->F.w, (float *)h->F3.w, n);
      h->launches++;
    }
    if (h->any_hdiff && !pre) {
      k_khfac<<<592, 256, 0, s>>>(h->G, h->F, (float *)h->F3.khx, (float *)h->F3.khy);
      h->launches++;
    }
    CK(cudaGetLastError());
  }
  if (st->sur_t && st->nsur_t) {
    CK(cudaMemcpyAsync(h->W.sur_t, st->sur_t + 1, (size_t)h->ncol * sizeof(int),
                       cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->W.nsur_t, st->nsur_t + 1, (size_t)h->ncol * sizeof(int),
                       cudaMemcpyHostToDevice, s));
  }
  if (st->dt != h->dt) {
    h->dt = st->dt;
    h->F.dt = st->dt;
    for (int i = 0; i < 2; i++)
      if (h->graph[i]) {
        cudaGraphExecDestroy(h->graph[i]);
        h->graph[i] = nullptr;
      }
    h->have_sched = false;
  }
  h->probe_left = 2;
  return 0;
}

int shoc_tr_gpu_get_surface(shoc_tr_gpu *h, int *sur_t, int *nsur_t) {
  if (!h) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  if (sur_t)
    CK(cudaMemcpyAsync(sur_t + 1, h->W.sur_t, (size_t)h->ncol * sizeof(int),
                       cudaMemcpyDeviceToHost, h->stream));
  if (nsur_t)
    CK(cudaMemcpyAsync(nsur_t + 1, h->W.nsur_t, (size_t)h->ncol * sizeof(int),
                       cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int shoc_tr_gpu_set_preamble(shoc_tr_gpu *h, int on) {
  if (!h) return SHOC_TR_EARG;
  if (on && !h->pre.ok) return SHOC_TR_EUNSUPPORTED;
  DeviceScope dev_(h->device);
  if (on) {
    int rc = 0;
    if (!rc && !h->F.dzu1) rc = dupload<double>(h, (double **)&h->F.dzu1, nullptr, (size_t)h->S);
    if (!rc && !h->F.dzu2) rc = dupload<double>(h, (double **)&h->F.dzu2, nullptr, (size_t)h->S);
    if (!rc && !h->pre.detadt) rc = dupload<double>(h, &h->pre.detadt, nullptr, (size_t)h->S2);
    if (rc) return rc;
  }
  if (h->pre.on != (on != 0)) {
    h->pre.on = on != 0;
    for (int i = 0; i < 2; i++)  // the captured steps hold the old part A
      if (h->graph[i]) {
        cudaGraphExecDestroy(h->graph[i]);
        h->graph[i] = nullptr;
      }
    h->probe_left = std::max(h->probe_left, 1);  // w, and so the sub-steps, change
  }
  return SHOC_TR_OK;
}

int shoc_tr_gpu_set_detadt(shoc_tr_gpu *h, const double *detadt) {
  if (!h || !detadt) return SHOC_TR_EARG;
  if (!h->pre.detadt) return SHOC_TR_EARG;  // the preamble was never enabled
  DeviceScope dev_(h->device);
  CK(cudaMemcpyAsync(h->pre.detadt, detadt, (size_t)h->S2 * sizeof(double),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SHOC_TR_OK;
}

int shoc_tr_gpu_get_flow(shoc_tr_gpu *h, double *u1flux3d, double *u2flux3d, double *w,
                         double *dzu1, double *dzu2) {
  if (!h) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  const size_t S = (size_t)h->S * sizeof(double);
  const struct {
    double *dst;
    const double *src;
  } cp[] = {{u1flux3d, h->F.u1flux3d}, {u2flux3d, h->F.u2flux3d}, {w, h->F.w},
            {dzu1, h->F.dzu1}, {dzu2, h->F.dzu2}};
  for (auto &x : cp) {
    if (!x.dst) continue;
    if (!x.src) return SHOC_TR_EARG;  // dzu1 / dzu2: neither uploaded nor computed
    CK(cudaMemcpyAsync(x.dst, x.src, S, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return SHOC_TR_OK;
}

// ---- checkpoint / resume: a versioned raw image of the resident state ----
// [header 8 x int64][tracers: ntr x S values of the handle's precision]
// [compensations: ntr x S int16, FP32_COMP only]
// [carry: ntr x ncol doubles, FP32-mixed path only][sur_t, nsur_t: ncol ints each]
namespace {
constexpr long long kStateMagic = 0x53484f4354524731ll;  // "SHOCTRG1"
void state_layout(const shoc_tr_gpu *h, long long hd[8]) {
  hd[0] = kStateMagic;
  hd[1] = 1;  // version
  hd[2] = h->precision;
  hd[3] = h->ntr;
  hd[4] = h->S;
  hd[5] = h->ncol;
  hd[6] = h->fu.carry ? 1 : 0;
  hd[7] = 0;
}
size_t state_bytes(const shoc_tr_gpu *h) {
  return 8 * sizeof(long long) + (size_t)h->ntr * h->S * h->esize +
         (h->comp ? (size_t)h->ntr * h->S * sizeof(int16_t) : 0) +
         (h->fu.carry ? (size_t)h->ntr * h->ncol * sizeof(double) : 0) +
         2 * (size_t)h->ncol * sizeof(int);
}
}  // namespace

int shoc_tr_gpu_state_size(shoc_tr_gpu *h, size_t *bytes) {
  if (!h || !bytes) return SHOC_TR_EARG;
  *bytes = state_bytes(h);
  return SHOC_TR_OK;
}

int shoc_tr_gpu_save_state(shoc_tr_gpu *h, void *buf, size_t bytes) {
  if (!h || !buf || bytes < state_bytes(h)) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  char *p = (char *)buf;
  long long hd[8];
  state_layout(h, hd);
  memcpy(p, hd, sizeof(hd));
  p += sizeof(hd);
  const size_t tb = (size_t)h->ntr * h->S * h->esize;
  CK(cudaMemcpyAsync(p, h->tr[h->cur], tb, cudaMemcpyDeviceToHost, h->stream));
  p += tb;
  if (h->comp) {
    const size_t lb = (size_t)h->ntr * h->S * sizeof(int16_t);
    CK(cudaMemcpyAsync(p, h->lo[h->cur], lb, cudaMemcpyDeviceToHost, h->stream));
    p += lb;
  }
  if (h->fu.carry) {
    const size_t cb = (size_t)h->ntr * h->ncol * sizeof(double);
    CK(cudaMemcpyAsync(p, h->fu.carry, cb, cudaMemcpyDeviceToHost, h->stream));
    p += cb;
  }
  CK(cudaMemcpyAsync(p, h->W.sur_t, (size_t)h->ncol * sizeof(int), cudaMemcpyDeviceToHost,
                     h->stream));
  p += (size_t)h->ncol * sizeof(int);
  CK(cudaMemcpyAsync(p, h->W.nsur_t, (size_t)h->ncol * sizeof(int), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SHOC_TR_OK;
}

int shoc_tr_gpu_load_state(shoc_tr_gpu *h, const void *buf, size_t bytes) {
  if (!h || !buf || bytes < state_bytes(h)) return SHOC_TR_EARG;
  long long hd[8], want[8];
  memcpy(hd, buf, sizeof(hd));
  state_layout(h, want);
  if (memcmp(hd, want, sizeof(hd)) != 0) return SHOC_TR_EARG;  // another window or precision
  DeviceScope dev_(h->device);
  const char *p = (const char *)buf + sizeof(hd);
  const size_t tb = (size_t)h->ntr * h->S * h->esize;
  // both ping-pong buffers hold the state (the values a step does not write
  // are read back from either)
  CK(cudaMemcpyAsync(h->tr[h->cur], p, tb, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->tr[h->cur ^ 1], h->tr[h->cur], tb, cudaMemcpyDeviceToDevice, h->stream));
  p += tb;
  if (h->comp) {
    const size_t lb = (size_t)h->ntr * h->S * sizeof(int16_t);
    CK(cudaMemcpyAsync(h->lo[h->cur], p, lb, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->lo[h->cur ^ 1], h->lo[h->cur], lb, cudaMemcpyDeviceToDevice,
                       h->stream));
    p += lb;
  }
  if (h->fu.carry) {
    const size_t cb = (size_t)h->ntr * h->ncol * sizeof(double);
    CK(cudaMemcpyAsync(h->fu.carry, p, cb, cudaMemcpyHostToDevice, h->stream));
    p += cb;
  }
  CK(cudaMemcpyAsync(h->W.sur_t, p, (size_t)h->ncol * sizeof(int), cudaMemcpyHostToDevice,
                     h->stream));
  p += (size_t)h->ncol * sizeof(int);
  CK(cudaMemcpyAsync(h->W.nsur_t, p, (size_t)h->ncol * sizeof(int), cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SHOC_TR_OK;
}

int shoc_tr_gpu_run(shoc_tr_gpu *h, int nsteps) {
  if (!h || nsteps < 0) return SHOC_TR_EARG;
  if (h->dt <= 0.0) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  for (int i = 0; i < nsteps; i++) {
    int rc = step_async(h);
    if (rc) return rc;
  }
  return 0;
}

int shoc_tr_gpu_sync(shoc_tr_gpu *h, shoc_tr_diag *diag) {
  if (!h) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  CK(cudaMemcpyAsync(h->h_status, h->W.status, 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(h->h_nwarn, h->W.nwarn, 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(h->h_counts, h->d_counts, 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemsetAsync(h->W.status, 0, 4, h->stream));
  CK(cudaMemsetAsync(h->W.nwarn, 0, 8, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  int rc = map_status(*h->h_status);
  if (!rc) rc = h->last_status;
  h->last_status = 0;
  if (diag) {
    diag->nsub = (int)h->sched.sub.size();
    diag->dtm = h->sched.dtm;
    diag->nwarn = (long long)*h->h_nwarn;
    diag->vcs = h->h_counts[0];
    diag->vc = h->h_counts[1];
  }
  if (h->profile) {
    std::vector<cudaEvent_t> done;
    for (auto &e : h->ev) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e.a, e.b);
      h->prof_ms[e.part] += ms;
      h->prof_n[e.part]++;
      for (cudaEvent_t x : {e.a, e.b})
        if (std::find(done.begin(), done.end(), x) == done.end()) done.push_back(x);
    }
    for (cudaEvent_t x : done) cudaEventDestroy(x);
    h->ev.clear();
  }
  return rc;
}

int shoc_tr_gpu_step(shoc_tr_gpu *h, shoc_tr_state *st, shoc_tr_diag *diag) {
  if (!h || !st || !st->tr_wc || st->ntr != h->ntr) return SHOC_TR_EARG;
  for (int n = 0; n < h->ntr; n++)
    if (!st->tr_wc[n]) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  int rc = step_pipelined(h, st);
  if (rc) {
    shoc_tr_gpu_sync(h, nullptr);
    return rc;
  }
  rc = shoc_tr_gpu_sync(h, diag);
  int rc2 = shoc_tr_gpu_get_surface(h, st->sur_t, st->nsur_t);
  if (!rc) rc = rc2;
  return rc;
}

int shoc_tr_gpu_host_register(void *ptr, size_t bytes) {
  if (!ptr || !bytes) return SHOC_TR_EARG;
  CK(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
  return 0;
}

int shoc_tr_gpu_host_unregister(void *ptr) {
  if (!ptr) return SHOC_TR_EARG;
  CK(cudaHostUnregister(ptr));
  return 0;
}

int shoc_tr_gpu_mass(shoc_tr_gpu *h, double *mass) {
  if (!h || !mass) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  const int nb = 148 * 2;
  double *part = nullptr;
  CK(cudaMallocAsync(&part, (size_t)nb * std::max(h->ntr, 1) * sizeof(double), h->stream));
  if (h->ntr > 0) {
    if (h->esize == sizeof(float))
      k_mass<float><<<dim3(nb, h->ntr), 256, 0, h->stream>>>(
          h->G, h->F, h->W, (const float *)h->tr[h->cur], h->fu.carry, part, nullptr, 0,
          h->lo[h->cur]);
    else
      k_mass<double><<<dim3(nb, h->ntr), 256, 0, h->stream>>>(
          h->G, h->F, h->W, (const double *)h->tr[h->cur], nullptr, part);
    h->launches++;
  }
  std::vector<double> hp((size_t)nb * h->ntr);
  CK(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaFreeAsync(part, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int n = 0; n < h->ntr; n++) {
    double s = 0.0, comp = 0.0;
    for (int b = 0; b < nb; b++) {
      double v = hp[(size_t)n * nb + b], u = s + v;
      comp += (fabs(s) >= fabs(v)) ? (s - u) + v : (v - u) + s;
      s = u;
    }
    mass[n] = s + comp;
  }
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Mass reduction that allocates nothing.
//
// For host frameworks that hand all device memory out of a pool reserved at
// start-up and forbid any other allocation once the run is going (a coupled
// model sharing the GPU with other components): shoc_tr_gpu_mass allocates a
// stream-ordered buffer per call, this one does not.  The block partials live
// in the fixed device array below; the caller passes the (already allocated)
// handle and a host array for the result.
namespace {

constexpr int kNoAllocBlocks = 148 * 2;     // partial sums per tracer
constexpr int kNoAllocMaxTracers = 64;      // largest tracer count it serves
// [kNoAllocMaxTracers][kNoAllocBlocks] partials, then kNoAllocMaxTracers sums;
// about 152 KB that every device loading the library holds until exit
__device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxTracers * kNoAllocBlocks +
                                                   kNoAllocMaxTracers];

// Per-tracer compensated sum of the block partials, in the order the
// allocating entry point sums them on the host (same result bit for bit).
__global__ void k_mass_finish(const double *part, int nb, int ntr, double *sums) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= ntr) return;
  double s = 0.0, comp = 0.0;
  for (int b = 0; b < nb; b++) {
    double v = part[(size_t)n * nb + b], u = s + v;
    comp += (fabs(s) >= fabs(v)) ? (s - u) + v : (v - u) + s;
    s = u;
  }
  sums[n] = s + comp;
}

std::mutex g_noalloc_mu;
double *g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array for the current device, looked up once
// per device and kept (the symbol's host-side name is not a device address).
// A reset of the device (cudaDeviceReset) invalidates the kept address, as it
// invalidates every handle's device memory.
int noalloc_scratch(int device, double **out) {
  if (device < 0 || device >= 64) return SHOC_TR_EARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      fprintf(stderr, "shoc_tr_gpu: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
      return SHOC_TR_ECUDA;
    }
    g_noalloc_ptr[device] = (double *)p;
  }
  *out = g_noalloc_ptr[device];
  return SHOC_TR_OK;
}

}  // namespace

extern "C" {

int shoc_tr_gpu_mass_noalloc(shoc_tr_gpu *h, double *mass) {
  if (!h || !mass) return SHOC_TR_EARG;
  if (h->ntr > kNoAllocMaxTracers) return SHOC_TR_ESCRATCH;
  DeviceScope dev_(h->device);
  if (!dev_.ok) return SHOC_TR_ECUDA;
  double *scr = nullptr;
  int rc = noalloc_scratch(h->device, &scr);
  if (rc) return rc;
  if (h->ntr == 0) return SHOC_TR_OK;
  // every partial and sum slot used below is written before it is read, so
  // nothing left over from an earlier call needs clearing
  double *part = scr, *sums = scr + (size_t)kNoAllocMaxTracers * kNoAllocBlocks;
  if (h->esize == sizeof(float))
    k_mass<float><<<dim3(kNoAllocBlocks, h->ntr), 256, 0, h->stream>>>(
        h->G, h->F, h->W, (const float *)h->tr[h->cur], h->fu.carry, part, nullptr, 0,
        h->lo[h->cur]);
  else
    k_mass<double><<<dim3(kNoAllocBlocks, h->ntr), 256, 0, h->stream>>>(
        h->G, h->F, h->W, (const double *)h->tr[h->cur], nullptr, part);
  k_mass_finish<<<(h->ntr + 63) / 64, 64, 0, h->stream>>>(part, kNoAllocBlocks, h->ntr, sums);
  h->launches += 2;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(mass, sums, (size_t)h->ntr * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SHOC_TR_OK;
}

int shoc_tr_gpu_compare(shoc_tr_gpu *a, shoc_tr_gpu *b, const int *region, int nregion,
                        double *maxabs, double *maxref, double *sumsq_diff, double *sumsq_ref) {
  if (!a || !b || !maxabs || !maxref || !sumsq_diff || !sumsq_ref) return SHOC_TR_EARG;
  if (nregion < 1 || (!region && nregion != 1)) return SHOC_TR_EARG;
  if (a->device != b->device || a->S != b->S || a->S2 != b->S2 || a->ncol != b->ncol ||
      a->ntr != b->ntr || a->nz != b->nz)
    return SHOC_TR_EARG;
  DeviceScope dev_(a->device);
  const int ntr = a->ntr;
  const size_t nout = (size_t)nregion * ntr;
  if (nout == 0) return SHOC_TR_OK;
  // both handles' work so far, then the comparison on a's stream
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ev, b->stream));
  CK(cudaStreamWaitEvent(a->stream, ev, 0));
  cudaEventDestroy(ev);
  cudaStream_t st = a->stream;
  // per column region ids (region is indexed by 2D cell, as SHOC's 2D arrays)
  char *buf = nullptr;
  const size_t bytes = nout * 4 * sizeof(double) + (region ? (size_t)a->ncol * sizeof(int) : 0);
  CK(cudaMallocAsync((void **)&buf, bytes, st));
  unsigned long long *dmax = (unsigned long long *)buf, *dref = dmax + nout;
  double *dsd = (double *)(dref + nout), *dsr = dsd + nout;
  int *dreg = nullptr;
  CK(cudaMemsetAsync(buf, 0, nout * 4 * sizeof(double), st));
  std::vector<int> hcol;
  if (region) {
    std::vector<int> top(a->ncol);
    CK(cudaMemcpyAsync(top.data(), a->G.col_top, (size_t)a->ncol * sizeof(int),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    hcol.resize(a->ncol);
    for (int c = 0; c < a->ncol; c++) hcol[c] = region[top[c]];
    dreg = (int *)(dsr + nout);
    CK(cudaMemcpyAsync(dreg, hcol.data(), (size_t)a->ncol * sizeof(int),
                       cudaMemcpyHostToDevice, st));
  }
  const dim3 grid(148 * 2, ntr);
  const bool fa = a->esize == sizeof(float), fb = b->esize == sizeof(float);
  const void *ta = a->tr[a->cur], *tb = b->tr[b->cur];
  if (fa && fb)
    k_compare<float, float><<<grid, 256, 0, st>>>(a->G, a->tl, b->G.colntr, (const float *)ta,
                                                 (const float *)tb, dreg, nregion, dmax, dref,
                                                 dsd, dsr, a->lo[a->cur], b->lo[b->cur]);
  else if (fa)
    k_compare<float, double><<<grid, 256, 0, st>>>(a->G, a->tl, b->G.colntr, (const float *)ta,
                                                  (const double *)tb, dreg, nregion, dmax,
                                                  dref, dsd, dsr, a->lo[a->cur], b->lo[b->cur]);
  else if (fb)
    k_compare<double, float><<<grid, 256, 0, st>>>(a->G, a->tl, b->G.colntr, (const double *)ta,
                                                  (const float *)tb, dreg, nregion, dmax, dref,
                                                  dsd, dsr, a->lo[a->cur], b->lo[b->cur]);
  else
    k_compare<double, double><<<grid, 256, 0, st>>>(a->G, a->tl, b->G.colntr,
                                                   (const double *)ta, (const double *)tb, dreg,
                                                   nregion, dmax, dref, dsd, dsr, a->lo[a->cur], b->lo[b->cur]);
  a->launches++;
  CK(cudaGetLastError());
  std::vector<double> out(nout * 4);
  CK(cudaMemcpyAsync(out.data(), buf, nout * 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaFreeAsync(buf, st));
  CK(cudaStreamSynchronize(st));
  memcpy(maxabs, out.data(), nout * sizeof(double));
  memcpy(maxref, out.data() + nout, nout * sizeof(double));
  memcpy(sumsq_diff, out.data() + 2 * nout, nout * sizeof(double));
  memcpy(sumsq_ref, out.data() + 3 * nout, nout * sizeof(double));
  return SHOC_TR_OK;
}

// device arrays of the column-solve entry points: nine [S] fields and three
// [S2] fields, allocated on the first call
static int cols_buffer(shoc_tr_gpu *h) {
  if (h->cols) return 0;
  return dalloc(h, &h->cols, (size_t)9 * h->S + (size_t)3 * h->S2);
}

static int cols_status(shoc_tr_gpu *h) {
  CK(cudaMemcpyAsync(h->h_status, h->W.status, 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemsetAsync(h->W.status, 0, 4, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return map_status(*h->h_status);
}

int shoc_tr_gpu_tridiag(shoc_tr_gpu *h, const double *C, const double *Cm1, const double *Cp1,
                        const double *rhs, double *var, double minvar) {
  if (!h || !C || !Cm1 || !Cp1 || !rhs || !var) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  int rc = cols_buffer(h);
  if (rc) return rc;
  const size_t S = (size_t)h->S, b = S * sizeof(double);
  double *dC = h->cols, *dCm1 = dC + S, *dCp1 = dCm1 + S, *dr = dCp1 + S, *dv = dr + S;
  double *dsol = dv + S, *dud = dsol + S;
  cudaStream_t st = h->stream;
  CK(cudaMemcpyAsync(dC, C, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dCm1, Cm1, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dCp1, Cp1, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dr, rhs, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dv, var, b, cudaMemcpyHostToDevice, st));
  k_tridiag<<<(h->ncol + 127) / 128, 128, 0, st>>>(h->G, h->W, dC, dCm1, dCp1, dr, dv, dsol, dud,
                                                   minvar);
  h->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(var, dv, b, cudaMemcpyDeviceToHost, st));
  return cols_status(h);
}

int shoc_tr_gpu_vdiff_cols(shoc_tr_gpu *h, double *var, const double *dzcell, const double *C,
                           const double *Cm1, const double *Cp1, const double *fb,
                           const double *ft, const double *Splus, const double *Sminus,
                           const double *scale, double dt) {
  if (!h || !var || !dzcell || !C || !Cm1 || !Cp1 || !fb || !ft || !scale || !(dt > 0.0))
    return SHOC_TR_EARG;
  if (h->dt <= 0.0) return SHOC_TR_EARG;  // the window's dt (set_flow) is read too
  DeviceScope dev_(h->device);
  int rc = cols_buffer(h);
  if (rc) return rc;
  const size_t S = (size_t)h->S, b = S * sizeof(double), b2 = (size_t)h->S2 * sizeof(double);
  double *dC = h->cols, *dCm1 = dC + S, *dCp1 = dCm1 + S, *ddz = dCp1 + S, *dv = ddz + S;
  double *dsol = dv + S, *dud = dsol + S, *dsp = dud + S, *dsm = dsp + S;
  double *dfb = dsm + S, *dft = dfb + h->S2, *dsc = dft + h->S2;
  cudaStream_t st = h->stream;
  CK(cudaMemcpyAsync(dC, C, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dCm1, Cm1, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dCp1, Cp1, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ddz, dzcell, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dv, var, b, cudaMemcpyHostToDevice, st));
  if (Splus) CK(cudaMemcpyAsync(dsp, Splus, b, cudaMemcpyHostToDevice, st));
  if (Sminus) CK(cudaMemcpyAsync(dsm, Sminus, b, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dfb, fb, b2, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dft, ft, b2, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dsc, scale, b2, cudaMemcpyHostToDevice, st));
  k_vdiff_cols<<<(h->ncol + 127) / 128, 128, 0, st>>>(
      h->G, h->W, dv, ddz, dC, dCm1, dCp1, dfb, dft, Splus ? dsp : nullptr,
      Sminus ? dsm : nullptr, dsc, dsol, dud, dt, h->dt, h->O.hmin);
  h->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(var, dv, b, cudaMemcpyDeviceToHost, st));
  return cols_status(h);
}

int shoc_tr_gpu_halo_plan(shoc_tr_gpu *h, int nsend, const int *send_cells, int nrecv,
                          const int *recv_cells) {
  if (!h || nsend < 0 || nrecv < 0 || (nsend && !send_cells) || (nrecv && !recv_cells))
    return SHOC_TR_EARG;
  for (int i = 0; i < nsend; i++)
    if (send_cells[i] < 1 || send_cells[i] >= h->S) return SHOC_TR_EARG;
  for (int i = 0; i < nrecv; i++)
    if (recv_cells[i] < 1 || recv_cells[i] >= h->S) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  int rc;
  if (nsend > h->nhalo_send && (rc = dalloc(h, &h->halo_send, (size_t)nsend))) return rc;
  if (nrecv > h->nhalo_recv && (rc = dalloc(h, &h->halo_recv, (size_t)nrecv))) return rc;
  if (nsend)
    CK(cudaMemcpy(h->halo_send, send_cells, (size_t)nsend * sizeof(int), cudaMemcpyHostToDevice));
  if (nrecv)
    CK(cudaMemcpy(h->halo_recv, recv_cells, (size_t)nrecv * sizeof(int), cudaMemcpyHostToDevice));
  h->nhalo_send = nsend;
  h->nhalo_recv = nrecv;
  return SHOC_TR_OK;
}

int shoc_tr_gpu_halo_pack(shoc_tr_gpu *h, void *buf) {
  if (!h || (h->nhalo_send && !buf)) return SHOC_TR_EARG;
  if (h->comp) return SHOC_TR_EUNSUPPORTED;  // the halo carries no compensation
  DeviceScope dev_(h->device);
  const int n = h->nhalo_send;
  if (n && h->ntr) {
    const long long tot = (long long)n * h->ntr;
    const int blocks = (int)std::min<long long>((tot + 255) / 256, 148 * 8);
    if (h->esize == sizeof(float))
      k_halo_pack<float><<<blocks, 256, 0, h->stream>>>((const float *)h->tr[h->cur], h->S,
                                                        h->ntr, h->halo_send, n, (float *)buf);
    else
      k_halo_pack<double><<<blocks, 256, 0, h->stream>>>((const double *)h->tr[h->cur], h->S,
                                                         h->ntr, h->halo_send, n, (double *)buf);
    h->launches++;
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(h->stream));
  return SHOC_TR_OK;
}

int shoc_tr_gpu_halo_unpack(shoc_tr_gpu *h, const void *buf) {
  if (!h || (h->nhalo_recv && !buf)) return SHOC_TR_EARG;
  if (h->comp) return SHOC_TR_EUNSUPPORTED;
  DeviceScope dev_(h->device);
  const int n = h->nhalo_recv;
  if (n && h->ntr) {
    const long long tot = (long long)n * h->ntr;
    const int blocks = (int)std::min<long long>((tot + 255) / 256, 148 * 8);
    if (h->esize == sizeof(float))
      k_halo_unpack<float><<<blocks, 256, 0, h->stream>>>(
          (float *)h->tr[h->cur], (float *)h->tr[h->cur ^ 1], h->S, h->ntr, h->halo_recv, n,
          (const float *)buf);
    else
      k_halo_unpack<double><<<blocks, 256, 0, h->stream>>>(
          (double *)h->tr[h->cur], (double *)h->tr[h->cur ^ 1], h->S, h->ntr, h->halo_recv, n,
          (const double *)buf);
    h->launches++;
    CK(cudaGetLastError());
  }
  return SHOC_TR_OK;
}

int shoc_tr_gpu_mass_region(shoc_tr_gpu *h, const int *region, int reg, double *mass) {
  if (!h || !region || !mass) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  const int nb = 148 * 2;
  std::vector<int> top(h->ncol), cr(h->ncol);
  CK(cudaMemcpyAsync(top.data(), h->G.col_top, (size_t)h->ncol * sizeof(int),
                     cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int c = 0; c < h->ncol; c++) cr[c] = region[top[c]];
  char *buf = nullptr;
  const size_t pb = (size_t)nb * std::max(h->ntr, 1) * sizeof(double);
  CK(cudaMallocAsync((void **)&buf, pb + (size_t)h->ncol * sizeof(int), h->stream));
  double *part = (double *)buf;
  int *dreg = (int *)(buf + pb);
  CK(cudaMemcpyAsync(dreg, cr.data(), (size_t)h->ncol * sizeof(int), cudaMemcpyHostToDevice,
                     h->stream));
  if (h->ntr > 0) {
    if (h->esize == sizeof(float))
      k_mass<float><<<dim3(nb, h->ntr), 256, 0, h->stream>>>(
          h->G, h->F, h->W, (const float *)h->tr[h->cur], h->fu.carry, part, dreg, reg,
          h->lo[h->cur]);
    else
      k_mass<double><<<dim3(nb, h->ntr), 256, 0, h->stream>>>(
          h->G, h->F, h->W, (const double *)h->tr[h->cur], nullptr, part, dreg, reg);
    h->launches++;
  }
  std::vector<double> hp((size_t)nb * h->ntr);
  CK(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaFreeAsync(buf, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int n = 0; n < h->ntr; n++) {
    double s = 0.0, comp = 0.0;
    for (int b = 0; b < nb; b++) {
      double v = hp[(size_t)n * nb + b], u = s + v;
      comp += (fabs(s) >= fabs(v)) ? (s - u) + v : (v - u) + s;
      s = u;
    }
    mass[n] = s + comp;
  }
  return SHOC_TR_OK;
}

int shoc_tr_gpu_set_owned(shoc_tr_gpu *h, const int *owned2d) {
  if (!h) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  if (!owned2d) {
    h->colown = nullptr;  // every column counts again (the array stays allocated)
    return SHOC_TR_OK;
  }
  std::vector<int> top(h->ncol), own(h->ncol);
  CK(cudaMemcpy(top.data(), h->G.col_top, (size_t)h->ncol * sizeof(int), cudaMemcpyDeviceToHost));
  for (int c = 0; c < h->ncol; c++) own[c] = owned2d[top[c]] ? 1 : 0;
  int *d = nullptr;
  int rc = dupload(h, &d, own.data(), (size_t)h->ncol);
  if (rc) return rc;
  h->colown = d;
  return SHOC_TR_OK;
}

int shoc_tr_gpu_substep_min(shoc_tr_gpu *h, double *dmin) {
  if (!h || !dmin || h->dt <= 0.0) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  cudaStream_t st = h->stream;
  k_reset<<<1, 32, 0, st>>>(h->W, h->d_counts);
  const int nb = (h->ncol + 127) / 128;
  k_set_dz<<<nb, 128, 0, st>>>(h->G, h->F, h->W, h->O, h->tl, h->any_vdiff ? 1 : 0, h->d_counts,
                               h->staged ? 1 : 0, h->esize == sizeof(float) ? 1 : 0, h->colown,
                               1);
  h->launches += 2;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->h_dtm, h->W.dtm_bits, 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  unsigned long long b = *h->h_dtm;
  memcpy(dmin, &b, 8);
  return SHOC_TR_OK;
}

int shoc_tr_gpu_set_substep_min(shoc_tr_gpu *h, double dmin) {
  if (!h || dmin < 0.0) return SHOC_TR_EARG;
  if (dmin != h->dmin_set) {
    DeviceScope dev_(h->device);
    h->dmin_set = dmin;
    for (int i = 0; i < 2; i++)
      if (h->graph[i]) {
        cudaGraphExecDestroy(h->graph[i]);
        h->graph[i] = nullptr;
      }
    h->have_sched = false;
    h->probe_left = 2;
  }
  return SHOC_TR_OK;
}

void *shoc_tr_gpu_stream(shoc_tr_gpu *h) { return h ? (void *)h->stream : nullptr; }

int shoc_tr_gpu_set_tiling(shoc_tr_gpu *h, int cols_per_block, int tracers_per_block) {
  if (!h) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  if (cols_per_block != 0 && cols_per_block != 32) return SHOC_TR_EUNSUPPORTED;
  if (tracers_per_block <= 0) return SHOC_TR_OK;
  shoc_tr_tuning t = current_tuning(h);
  t.tracers_per_block = tracers_per_block;
  return apply_tuning(h, t);
}

int shoc_tr_gpu_get_tuning(shoc_tr_gpu *h, shoc_tr_tuning *t) {
  if (!h || !t) return SHOC_TR_EARG;
  *t = current_tuning(h);
  return SHOC_TR_OK;
}

int shoc_tr_gpu_set_tuning(shoc_tr_gpu *h, const shoc_tr_tuning *t) {
  if (!h || !t) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  return apply_tuning(h, *t);
}

}  // extern "C"

// ---- autotuner ----
namespace {

// The autotuner's cache: one line per GPU model and window configuration,
//   <key> <fused> <tracers_per_block> <tile_x> <phase_b_warps> <prefetch> <ms>
// in the file SHOC_TR_TUNE_CACHE names (default
// $HOME/.cache/shoc_tr_gpu/tuning.txt; "off": none).
std::string tune_cache_path() {
  const char *e = getenv("SHOC_TR_TUNE_CACHE");
  if (e) return strcmp(e, "off") == 0 ? std::string() : std::string(e);
  const char *home = getenv("HOME");
  if (!home || !*home) return std::string();
  return std::string(home) + "/.cache/shoc_tr_gpu/tuning.txt";
}

std::string tune_key(const shoc_tr_gpu *h) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, h->device) != cudaSuccess) return std::string();
  std::string name = p.name;
  for (char &c : name)
    if (c == ' ' || c == '\t') c = '_';
  char buf[512];
  snprintf(buf, sizeof buf, "v2|%s|sm%d%d|S%d|C%d|Z%d|N%d|B%d|P%d|A%d|U%d|F%d|H%d|V%d",
           name.c_str(), p.major, p.minor, h->S, h->ncol, h->nz, h->ntr, h->T.ntb, h->precision,
           h->O.trasc, h->O.ultimate, h->adv_flags, h->any_hdiff ? 1 : 0, h->any_vdiff ? 1 : 0);
  return std::string(buf);
}

bool tune_cache_get(const std::string &path, const std::string &key, shoc_tr_tuning *t) {
  if (path.empty() || key.empty()) return false;
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (fgets(line, sizeof line, f)) {
    char k[600];
    shoc_tr_tuning v;
    double ms;
    if (sscanf(line, "%599s %d %d %d %d %d %lf", k, &v.fused, &v.tracers_per_block, &v.tile_x,
               &v.phase_b_warps, &v.prefetch, &ms) == 7 &&
        key == k) {
      *t = v;
      found = true;  // the last line for a key wins
    }
  }
  fclose(f);
  return found;
}

void tune_cache_put(const std::string &path, const std::string &key, const shoc_tr_tuning &t,
                    double ms) {
  if (path.empty() || key.empty()) return;
  // the directory, one level at a time
  for (size_t i = 1; i < path.size(); i++)
    if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
  std::vector<std::string> keep;
  if (FILE *f = fopen(path.c_str(), "r")) {
    char line[1024];
    while (fgets(line, sizeof line, f)) {
      char k[600];
      if (sscanf(line, "%599s", k) == 1 && key != k) keep.push_back(line);
    }
    fclose(f);
  }
  const std::string tmp = path + ".tmp" + std::to_string((long long)getpid());
  FILE *f = fopen(tmp.c_str(), "w");
  if (!f) return;
  for (auto &l : keep) fputs(l.c_str(), f);
  fprintf(f, "%s %d %d %d %d %d %.6f\n", key.c_str(), t.fused, t.tracers_per_block, t.tile_x,
          t.phase_b_warps, t.prefetch, ms);
  fclose(f);
  rename(tmp.c_str(), path.c_str());
}

// Device copy of the resident state (both tracer buffers, mass carry,
// surface vectors) the trial steps start from.
// The resident state the autotuner's trial steps start from: the current
// tracer buffer (and compensation), put back into both ping-pong buffers as
// shoc_tr_gpu_load_state does.
struct Snapshot {
  void *tr = nullptr;
  int16_t *lo = nullptr;  // FP32_COMP: the current buffer's compensations
  double *carry = nullptr;
  int *sur = nullptr, *nsur = nullptr;
  int cur = 0;
};

int snap_take(shoc_tr_gpu *h, Snapshot &s) {
  const size_t tb = (size_t)h->ntr * h->S * h->esize;
  const size_t cb = (size_t)h->ntr * h->ncol * sizeof(double);
  const size_t ib = (size_t)h->ncol * sizeof(int);
  CK(cudaMallocAsync(&s.tr, tb ? tb : 1, h->stream));
  if (h->fu.carry) CK(cudaMallocAsync((void **)&s.carry, cb ? cb : 1, h->stream));
  CK(cudaMallocAsync((void **)&s.sur, 2 * ib, h->stream));
  s.nsur = s.sur + h->ncol;
  s.cur = h->cur;
  CK(cudaMemcpyAsync(s.tr, h->tr[h->cur], tb, cudaMemcpyDeviceToDevice, h->stream));
  if (h->comp) {
    const size_t lb = (size_t)h->ntr * h->S * sizeof(int16_t);
    CK(cudaMallocAsync((void **)&s.lo, lb ? lb : 1, h->stream));
    CK(cudaMemcpyAsync(s.lo, h->lo[h->cur], lb, cudaMemcpyDeviceToDevice, h->stream));
  }
  if (s.carry) CK(cudaMemcpyAsync(s.carry, h->fu.carry, cb, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(s.sur, h->W.sur_t, ib, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(s.nsur, h->W.nsur_t, ib, cudaMemcpyDeviceToDevice, h->stream));
  return 0;
}

int snap_restore(shoc_tr_gpu *h, const Snapshot &s) {
  const size_t tb = (size_t)h->ntr * h->S * h->esize;
  const size_t cb = (size_t)h->ntr * h->ncol * sizeof(double);
  const size_t ib = (size_t)h->ncol * sizeof(int);
  h->cur = s.cur;
  for (int b = 0; b < 2; b++)
    CK(cudaMemcpyAsync(h->tr[b], s.tr, tb, cudaMemcpyDeviceToDevice, h->stream));
  if (s.lo) {
    const size_t lb = (size_t)h->ntr * h->S * sizeof(int16_t);
    for (int b = 0; b < 2; b++)
      CK(cudaMemcpyAsync(h->lo[b], s.lo, lb, cudaMemcpyDeviceToDevice, h->stream));
  }
  if (s.carry) CK(cudaMemcpyAsync(h->fu.carry, s.carry, cb, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->W.sur_t, s.sur, ib, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->W.nsur_t, s.nsur, ib, cudaMemcpyDeviceToDevice, h->stream));
  return 0;
}

void snap_free(shoc_tr_gpu *h, Snapshot &s) {
  if (s.tr) cudaFreeAsync(s.tr, h->stream);
  if (s.lo) cudaFreeAsync(s.lo, h->stream);
  if (s.carry) cudaFreeAsync(s.carry, h->stream);
  if (s.sur) cudaFreeAsync(s.sur, h->stream);
  cudaStreamSynchronize(h->stream);
  s = Snapshot();
}

}  // namespace

extern "C" {

int shoc_tr_gpu_autotune_ex(shoc_tr_gpu *h, int steps, int use_cache, shoc_tr_tuning *best,
                            int *from_cache) {
  if (!h || steps < 1) return SHOC_TR_EARG;
  DeviceScope dev_(h->device);
  if (from_cache) *from_cache = 0;
  const std::string path = use_cache ? tune_cache_path() : std::string();
  const std::string key = use_cache ? tune_key(h) : std::string();
  shoc_tr_tuning t;
  if (use_cache && tune_cache_get(path, key, &t) && apply_tuning(h, t) == SHOC_TR_OK) {
    if (best) *best = t;
    if (from_cache) *from_cache = 1;
    return SHOC_TR_OK;
  }
  // candidates: tracers per column-kernel block for the two-kernel sub-step;
  // tile widths and phase-B warps for the fused one (FP32-mixed, where it fits)
  std::vector<shoc_tr_tuning> cand;
  shoc_tr_tuning base = current_tuning(h);
  const std::vector<int> tws = h->esize == sizeof(float)
                                   ? std::vector<int>{2, 3, 4, 5, 6, 8, 12, 16}
                                   : std::vector<int>{2, 3, 4, 5, 6, 8};
  for (int pf : {0, 1}) {
    if (pf && h->esize != sizeof(float)) continue;
    for (int tw : tws) {
      shoc_tr_tuning c = base;
      c.fused = 0;
      c.tracers_per_block = tw;
      c.prefetch = pf;
      cand.push_back(c);
    }
  }
  if (h->esize == sizeof(float) && h->fnwb_max) {
    std::vector<int> nwbs = {h->fnwb_max};
    if (h->fnwb_max / 2 >= 1 && h->fnwb_max / 2 != h->fnwb_max) nwbs.push_back(h->fnwb_max / 2);
    for (int tx : {8, 16, 32})
      for (int nwb : nwbs) {
        shoc_tr_tuning c = base;
        c.fused = 1;
        c.prefetch = 0;
        c.tile_x = tx;
        c.phase_b_warps = nwb;
        cand.push_back(c);
      }
  }
  Snapshot snap;
  int rc = snap_take(h, snap);
  if (rc) {  // no room for the copy: nothing has run, the handle is unchanged
    cudaGetLastError();
    snap_free(h, snap);
    return SHOC_TR_ENOMEM;
  }
  const bool prof0 = h->profile;
  shoc_tr_tuning win = base;
  double best_ms = 1e300;
  for (const auto &c : cand) {
    if (apply_tuning(h, c) != SHOC_TR_OK) continue;
    shoc_tr_gpu_profile(h, 1);
    rc = shoc_tr_gpu_run(h, steps);
    if (!rc) rc = shoc_tr_gpu_sync(h, nullptr);
    double ms = 0.0;
    int n = 0;
    shoc_tr_gpu_kernel_time(h, &ms, &n);
    if (!rc) rc = snap_restore(h, snap);
    if (rc) break;
    if (n > 0 && ms < best_ms) {
      best_ms = ms;
      win = c;
    }
  }
  if (!rc) rc = snap_restore(h, snap);
  snap_free(h, snap);
  h->profile = prof0;
  shoc_tr_gpu_profile(h, prof0 ? 1 : 0);
  const int rc2 = apply_tuning(h, win);
  if (rc) return rc;
  if (rc2) return rc2;
  if (use_cache && best_ms < 1e300) tune_cache_put(path, key, win, best_ms);
  if (best) *best = win;
  return SHOC_TR_OK;
}

int shoc_tr_gpu_autotune(shoc_tr_gpu *h, int steps, int *tracers_per_block) {
  shoc_tr_tuning t;
  const int rc = shoc_tr_gpu_autotune_ex(h, steps, 0, &t, nullptr);
  if (!rc && tracers_per_block) *tracers_per_block = t.tracers_per_block;
  return rc;
}

int shoc_tr_gpu_profile(shoc_tr_gpu *h, int enable) {
  if (!h) return SHOC_TR_EARG;
  h->profile = enable != 0;
  for (int i = 0; i < 3; i++) {
    h->prof_ms[i] = 0.0;
    h->prof_n[i] = 0;
  }
  return 0;
}

int shoc_tr_gpu_kernel_time_part(shoc_tr_gpu *h, int part, double *ms, int *n) {
  if (!h || part < 0 || part > 2) return SHOC_TR_EARG;
  if (ms) *ms = h->prof_n[part] ? h->prof_ms[part] / h->prof_n[part] : 0.0;
  if (n) *n = h->prof_n[part];
  h->prof_ms[part] = 0.0;
  h->prof_n[part] = 0;
  return 0;
}

int shoc_tr_gpu_kernel_time(shoc_tr_gpu *h, double *ms, int *n) {
  return shoc_tr_gpu_kernel_time_part(h, 0, ms, n);
}

long long shoc_tr_gpu_launch_count(shoc_tr_gpu *h) { return h ? h->launches : 0; }

}  // extern "C"
