// shoc_tr_launch.h -- host entry points of the kernels compiled in their own
// translation units (the FP32-mixed kernels are built with FMA contraction,
// the FP64 path without).
#pragma once
#include <cuda_runtime.h>

#include "shoc_tr_tile.cuh"

namespace shoc {

// allow every k_vd32 instance the opt-in shared memory size
cudaError_t tile32_set_smem_attr();

// one FP32-mixed transport sub-step over the staged columns: k_adv32 then
// k_vd32 (vd_nw tracers per k_vd32 block).  adv_flags: 1 every advected
// tracer has advection and no horizontal diffusion, 2 both, 0 mixed.  With
// ev != nullptr, events are recorded before, between and after the two
// launches.
void tile32_substep(bool last, bool quick, bool ult, cudaStream_t st, const Geo &G,
                    const Flow &F, const Flow32 &F3, const Work &W, const Opt &O,
                    const TrSet &T, const SubStep &ss, const Tile &Tl, const f32::Face2 *fx2,
                    const f32::Face2 *fy2, const float *tin, float *tout, float *fzs, int vd_nw,
                    int any_hd, int adv_flags, cudaEvent_t *ev);

}  // namespace shoc
