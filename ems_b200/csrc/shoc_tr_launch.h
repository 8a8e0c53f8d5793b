// shoc_tr_launch.h -- host entry points of the kernels compiled in their own
// translation units (the FP32-mixed kernels are built with FMA contraction,
// the FP64 path without).
#pragma once
#include <cuda_runtime.h>

#include "shoc_tr_fused.cuh"

namespace shoc {

// allow every k_vd32 instance the opt-in shared memory size
cudaError_t tile32_set_smem_attr();

// one FP32-mixed transport sub-step over the staged columns: k_adv32 then
// k_vd32 (vd_nw warps per k_vd32 block, vd_pf: staging the next tracer's
// column while the current one is solved); rnd [ntr][S] holds k_adv32's
// rounding residuals, carry [ntr][ncol] the columns' FP64 mass carry.
// adv_flags: 1 every advected
// tracer has advection and no horizontal diffusion, 2 both, 0 mixed.  With
// ev != nullptr, events are recorded before, between and after the two
// launches.
void tile32_substep(bool last, bool quick, bool ult, cudaStream_t st, const Geo &G,
                    const Flow &F, const Flow32 &F3, const Work &W, const Opt &O,
                    const TrSet &T, const SubStep &ss, const Tile &Tl, const f32::Face2 *fx2,
                    const f32::Face2 *fy2, const float *tin, float *tout, float *rnd,
                    double *carry, double *fzs, const int16_t *lo_in, int16_t *lo_out,
                    int vd_nw, int vd_pf, int any_hd, int adv_flags, cudaEvent_t *ev);

// allow every k_step32 instance `bytes` of dynamic shared memory
cudaError_t fused32_set_smem_attr(int bytes);

// one FP32-mixed transport sub-step over the staged columns as one fused
// launch (k_step32: one block per tile of 8 x 4 columns, `smem` bytes)
void fused32_substep(bool last, bool quick, bool ult, cudaStream_t st, const Geo &G,
                     const Flow &F, const Flow32 &F3, const Work &W, const Opt &O,
                     const TrSet &T, const SubStep &ss, const Tile &Tl, const Fused &Fu,
                     const f32::Face2 *fx2, const f32::Face2 *fy2, const float *tin, float *tout,
                     int any_hd, size_t smem);

}  // namespace shoc
