// Internal declarations shared between the translation units of the library.
#pragma once

#include <cuda_runtime.h>

#include "../../include/tfg_pt.h"

namespace tfg {

// Returns 0 when `dev` is a compute-capability 10.x device (the only target
// this library is built for), else TFG_E_UNSUPPORTED with a message.
int require_sm100(int dev);

int render_pass(const TfgRenderParams& prm, const TfgCamara* d_cam, const TfgPrimitiva* prims, int nprims,
                const TfgLuzPuntual* lights, int nlights, int W, int H, int frame, const TfgTinyBVHD_GPU* bvh,
                const float* tris_wt, const TfgPrimitiva* mesh, int nmesh, TfgColor* img, float* accum,
                TfgRegistroEntrenamiento* regs, uint32_t* reg_counter, int reg_cap, TfgDatosMLP* infer,
                TfgColor* thr_out, int use_inf, int train, cudaStream_t stream);

int trace_rays(const TfgTinyBVHD_GPU* bvh, const float* tris_wt, int fmt, const float* rays, int n, float* hits,
               cudaStream_t stream);

int camera_rays(const TfgCamara* d_cam, int W, int H, int frame, float* rays, cudaStream_t stream);

}  // namespace tfg
