// shoc_tr_f32.cu -- the FP32-mixed transport kernels' instances and their
// launcher.  Compiled with FMA contraction on (the FP64 reference path in
// shoc_tr_gpu.cu is compiled without it); the FP64 sums of the kernels use
// explicitly rounded operations where contraction would change them.
#include "shoc_tr_launch.h"

namespace shoc {

namespace {
template <class K>
cudaError_t attr(K k, int bytes = 227 * 1024) {
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <bool Q, bool U, int M>
void adv(int grid, cudaStream_t st, const Geo &G, const Flow32 &F3, const Work &W, const TrSet &T,
         const SubStep &ss, const Tile &Tl, const f32::Face2 *fx2, const f32::Face2 *fy2,
         const float *tin, float *tout, float *rnd, double *fzs, int hd,
         const int16_t *loi) {
  const size_t sm = M != 0 ? kAdvSmem : 0;
  if (loi)
    k_adv32<Q, U, M, true><<<grid, kAdv32Block, sm, st>>>(G, F3, W, T, ss, Tl, fx2, fy2, tin,
                                                          tout, rnd, fzs, hd, loi);
  else
    k_adv32<Q, U, M, false><<<grid, kAdv32Block, sm, st>>>(G, F3, W, T, ss, Tl, fx2, fy2, tin,
                                                           tout, rnd, fzs, hd, nullptr);
}
template <bool Q, bool U>
void adv_mode(int mode, int grid, cudaStream_t st, const Geo &G, const Flow32 &F3,
              const Work &W, const TrSet &T, const SubStep &ss, const Tile &Tl,
              const f32::Face2 *fx2, const f32::Face2 *fy2, const float *tin, float *tout,
              float *rnd, double *fzs, int hd, const int16_t *loi) {
  if (mode == 1)
    adv<Q, U, 1>(grid, st, G, F3, W, T, ss, Tl, fx2, fy2, tin, tout, rnd, fzs, hd, loi);
  else if (mode == 2)
    adv<Q, U, 2>(grid, st, G, F3, W, T, ss, Tl, fx2, fy2, tin, tout, rnd, fzs, hd, loi);
  else
    adv<Q, U, 0>(grid, st, G, F3, W, T, ss, Tl, fx2, fy2, tin, tout, rnd, fzs, hd, loi);
}
}  // namespace

cudaError_t tile32_set_smem_attr() {
  cudaError_t e = cudaSuccess;
  const int a = (int)kAdvSmem;
  const cudaError_t r[24] = {
      attr(k_vd32<true, false, false>),  attr(k_vd32<false, false, false>),
      attr(k_vd32<true, true, false>),   attr(k_vd32<false, true, false>),
      attr(k_vd32<true, false, true>),   attr(k_vd32<false, false, true>),
      attr(k_vd32<true, true, true>),    attr(k_vd32<false, true, true>),
      attr(k_adv32<true, true, 1, false>, a), attr(k_adv32<true, true, 2, false>, a),
      attr(k_adv32<true, false, 1, false>, a), attr(k_adv32<true, false, 2, false>, a),
      attr(k_adv32<false, true, 1, false>, a), attr(k_adv32<false, true, 2, false>, a),
      attr(k_adv32<false, false, 1, false>, a), attr(k_adv32<false, false, 2, false>, a),
      attr(k_adv32<true, true, 1, true>, a), attr(k_adv32<true, true, 2, true>, a),
      attr(k_adv32<true, false, 1, true>, a), attr(k_adv32<true, false, 2, true>, a),
      attr(k_adv32<false, true, 1, true>, a), attr(k_adv32<false, true, 2, true>, a),
      attr(k_adv32<false, false, 1, true>, a), attr(k_adv32<false, false, 2, true>, a)};
  for (auto x : r)
    if (x != cudaSuccess) e = x;
  return e;
}

void tile32_substep(bool last, bool quick, bool ult, cudaStream_t st, const Geo &G,
                    const Flow &F, const Flow32 &F3, const Work &W, const Opt &O,
                    const TrSet &T, const SubStep &ss, const Tile &Tl, const f32::Face2 *fx2,
                    const f32::Face2 *fy2, const float *tin, float *tout, float *rnd,
                    double *carry, double *fzs, const int16_t *lo_in, int16_t *lo_out,
                    int vd_nw, int vd_pf, int any_hd, int adv_flags, cudaEvent_t *ev) {
  if (ev) cudaEventRecord(ev[0], st);
  if (T.ntb > 0 && Tl.nwet > 0) {
    const int grid = (Tl.nwet + kAdv32Block - 1) / kAdv32Block;
    if (quick && ult)
      adv_mode<true, true>(adv_flags, grid, st, G, F3, W, T, ss, Tl, fx2, fy2, tin, tout, rnd,
                           fzs, any_hd, lo_in);
    else if (quick)
      adv_mode<true, false>(adv_flags, grid, st, G, F3, W, T, ss, Tl, fx2, fy2, tin, tout, rnd,
                            fzs, any_hd, lo_in);
    else if (ult)
      adv_mode<false, true>(adv_flags, grid, st, G, F3, W, T, ss, Tl, fx2, fy2, tin, tout, rnd,
                            fzs, any_hd, lo_in);
    else
      adv_mode<false, false>(adv_flags, grid, st, G, F3, W, T, ss, Tl, fx2, fy2, tin, tout, rnd,
                             fzs, any_hd, lo_in);
  }
  if (ev) cudaEventRecord(ev[1], st);
  const dim3 blk(32, vd_nw);
  for (int i = 0; i < Tl.nclass; i++) {
    const int t0 = Tl.ctile[i], nt = Tl.ctile[i + 1] - t0, kbase = Tl.cbase[i];
    if (nt <= 0) continue;
    const bool comp = lo_out != nullptr;
    const size_t smem = vd32_smem(G.nz - kbase, vd_nw, vd_pf != 0, comp);
    auto kern = comp ? (last ? (vd_pf ? k_vd32<true, true, true> : k_vd32<true, false, true>)
                             : (vd_pf ? k_vd32<false, true, true> : k_vd32<false, false, true>))
                     : (last ? (vd_pf ? k_vd32<true, true, false> : k_vd32<true, false, false>)
                             : (vd_pf ? k_vd32<false, true, false> : k_vd32<false, false, false>));
    kern<<<nt, blk, smem, st>>>(G, F, W, O, T, ss, Tl, W.lu32, tin, tout, rnd, carry, fzs, lo_in,
                                lo_out, vd_nw, t0, kbase);
  }
  if (ev) cudaEventRecord(ev[2], st);
}

namespace {
template <bool Q, bool U, bool L>
void step32(int grid, cudaStream_t st, size_t smem, const Geo &G, const Flow &F, const Flow32 &F3,
            const Work &W, const Opt &O, const TrSet &T, const SubStep &ss, const Tile &Tl,
            const Fused &Fu, const f32::Face2 *fx2, const f32::Face2 *fy2, const float *tin,
            float *tout, int hd) {
  k_step32<Q, U, L><<<grid, kFusedThreads, smem, st>>>(G, F, F3, W, O, T, ss, Tl, Fu, fx2, fy2,
                                                        tin, tout, hd, 0);
}
template <bool Q, bool U>
void step32_last(bool last, int grid, cudaStream_t st, size_t smem, const Geo &G, const Flow &F,
                 const Flow32 &F3, const Work &W, const Opt &O, const TrSet &T,
                 const SubStep &ss, const Tile &Tl, const Fused &Fu, const f32::Face2 *fx2,
                 const f32::Face2 *fy2, const float *tin, float *tout, int hd) {
  if (last)
    step32<Q, U, true>(grid, st, smem, G, F, F3, W, O, T, ss, Tl, Fu, fx2, fy2, tin, tout, hd);
  else
    step32<Q, U, false>(grid, st, smem, G, F, F3, W, O, T, ss, Tl, Fu, fx2, fy2, tin, tout, hd);
}
}  // namespace

cudaError_t fused32_set_smem_attr(int bytes) {
  cudaError_t e = cudaSuccess;
  const cudaError_t r[8] = {
      attr(k_step32<true, true, true>, bytes),   attr(k_step32<true, true, false>, bytes),
      attr(k_step32<true, false, true>, bytes),  attr(k_step32<true, false, false>, bytes),
      attr(k_step32<false, true, true>, bytes),  attr(k_step32<false, true, false>, bytes),
      attr(k_step32<false, false, true>, bytes), attr(k_step32<false, false, false>, bytes)};
  for (auto x : r)
    if (x != cudaSuccess) e = x;
  return e;
}

void fused32_substep(bool last, bool quick, bool ult, cudaStream_t st, const Geo &G,
                     const Flow &F, const Flow32 &F3, const Work &W, const Opt &O,
                     const TrSet &T, const SubStep &ss, const Tile &Tl, const Fused &Fu,
                     const f32::Face2 *fx2, const f32::Face2 *fy2, const float *tin, float *tout,
                     int any_hd, size_t smem) {
  const int grid = Fu.ntile;
  if (grid <= 0) return;
  if (quick && ult)
    step32_last<true, true>(last, grid, st, smem, G, F, F3, W, O, T, ss, Tl, Fu, fx2, fy2, tin,
                            tout, any_hd);
  else if (quick)
    step32_last<true, false>(last, grid, st, smem, G, F, F3, W, O, T, ss, Tl, Fu, fx2, fy2, tin,
                             tout, any_hd);
  else if (ult)
    step32_last<false, true>(last, grid, st, smem, G, F, F3, W, O, T, ss, Tl, Fu, fx2, fy2, tin,
                             tout, any_hd);
  else
    step32_last<false, false>(last, grid, st, smem, G, F, F3, W, O, T, ss, Tl, Fu, fx2, fy2, tin,
                              tout, any_hd);
}

}  // namespace shoc
