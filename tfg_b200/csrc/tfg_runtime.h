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

// Workspace slots per device: passes in flight at the same time (branches of
// a batched frame) must use different slots.
constexpr int kWorkspaceSlots = 4;

// render_pass with a device-side frame number / cache-query gate (both
// optional), a prepare-only mode that validates and allocates without
// launching (so a later call can be captured in a CUDA graph), and the
// workspace slot to run on.
int render_pass_ex(const TfgRenderParams& prm, const TfgCamara* d_cam, const TfgPrimitiva* prims, int nprims,
                   const TfgLuzPuntual* lights, int nlights, int W, int H, int frame, const int32_t* frame_dev,
                   const uint32_t* use_inf_dev, const TfgTinyBVHD_GPU* bvh, const float* tris_wt,
                   const TfgPrimitiva* mesh, int nmesh, TfgColor* img, float* accum, TfgRegistroEntrenamiento* regs,
                   uint32_t* reg_counter, int reg_cap, TfgDatosMLP* infer, TfgColor* thr_out, int use_inf, int train,
                   bool prepare_only, int ws_slot, cudaStream_t stream);

// Changes whenever the workspace of (dev, slot) is reallocated: a CUDA graph
// captured before holds stale queue pointers then.
uint32_t workspace_generation(int dev, int slot);

// One scene of a batched pass.
struct PassScene {
    const TfgCamara* cam; const TfgPrimitiva* prims; int nprims;
    const TfgLuzPuntual* lights; int nlights; int W, H;
    const TfgTinyBVHD_GPU* bvh; const float* tris_wt; const TfgPrimitiva* mesh; int nmesh;
    TfgColor* img; float* accum;
    TfgRegistroEntrenamiento* regs; uint32_t* reg_counter; int reg_cap;
    TfgDatosMLP* infer; TfgColor* thr_out;
    const uint32_t* use_inf_dev; int use_inf;
};

// 1 to 16 scenes with the same settings rendered as one wavefront series
// (one launch per stage for all of them), on workspace slot `ws_slot`.
int render_pass_multi(const TfgRenderParams& prm, const PassScene* scenes, int n, int frame, const int32_t* frame_dev,
                      int train, bool prepare_only, int ws_slot, cudaStream_t stream);

// Launch tuning of device `dev` (render.cu).  The generation number changes
// with every successful set.
int render_tuning_check(const TfgRenderTuning& t);
int render_tuning_set(int dev, const TfgRenderTuning& t);
int render_tuning_get(int dev, TfgRenderTuning* out, uint32_t* generation);

int trace_rays(const TfgTinyBVHD_GPU* bvh, const float* tris_wt, int fmt, const float* rays, int n, float* hits,
               cudaStream_t stream);

int camera_rays(const TfgCamara* d_cam, int W, int H, int frame, int samples, int order, float* rays,
                cudaStream_t stream);

// Small frame kernels with a device-side count: 0 tail queries (a = records,
// b = DatosMLP out), 1 targets (a = records, c = tail predictions, b = out),
// 2 record count (a = ring counter, b = count out, cap), 3 accumulate
// (a = image, b = FP32 accumulation, cap = pixels).
int launch_nrc_frame_small(int which, const void* a, void* b, const void* c, const uint32_t* n_dev, uint32_t cap,
                           uint32_t min_n, cudaStream_t s);

// Cache model internals used by the frame driver (nrc_mlp.cu).
struct ColorMlp;
int mlp_prepare(ColorMlp* n);
uint32_t* mlp_state(ColorMlp* n);
uint32_t* mlp_gate(ColorMlp* n);
uint32_t* mlp_navail(ColorMlp* n);
int mlp_enqueue_infer(ColorMlp* n, const TfgDatosMLP* in, TfgColor* out, TfgColor* img, const TfgColor* thr,
                      uint32_t max_count, const uint32_t* n_dev, cudaStream_t s);
int mlp_enqueue_train(ColorMlp* n, const TfgDatosMLP* buf, uint32_t min_n, cudaStream_t s);
void mlp_set_gate_threshold(ColorMlp* n, float g);
int mlp_precision(const ColorMlp* n);   // inference precision (part of a frame graph's identity)
uint32_t mlp_tuning_generation(const ColorMlp* n);   // changes with every tuning set

}  // namespace tfg
