// Internal declarations shared between the translation units of the library.
#pragma once

#include <cuda_runtime.h>

#include "../../include/tfg_pt.h"

namespace tfg {

// Per-device state (workspaces, tunings, launch shapes, graphs, the static
// scratch address) is kept in tables indexed by the device ordinal.
constexpr int kMaxDevices = 16;

// Returns 0 when `dev` is a compute-capability 10.x device (the only target
// this library is built for) with an ordinal below kMaxDevices; else
// TFG_E_INVALID (ordinal out of range) or TFG_E_UNSUPPORTED, with a message.
// Every entry point that touches per-device state calls it first.
int require_sm100(int dev);

int render_pass(const TfgRenderParams& prm, const TfgCamara* d_cam, const TfgPrimitiva* prims, int nprims,
                const TfgLuzPuntual* lights, int nlights, int W, int H, int frame, const TfgTinyBVHD_GPU* bvh,
                const float* tris_wt, const TfgPrimitiva* mesh, int nmesh, TfgColor* img, float* accum,
                TfgRegistroEntrenamiento* regs, uint32_t* reg_counter, int reg_cap, TfgDatosMLP* infer,
                TfgColor* thr_out, int use_inf, int train, cudaStream_t stream);

// Workspace slots per device: passes in flight at the same time (branches of
// a batched frame) must use different slots.
constexpr int kWorkspaceSlots = 4;

// Resolution per axis of a cache model's gate grid over its scene bounds.
constexpr int kGateRes = 32;
constexpr int kGateCells = kGateRes * kGateRes * kGateRes;

// How a render pass uses the radiance cache.  The defaults are the
// reference's policy (render.h:86-202, :443): a path queries the cache (or a
// training path records its head) at its first diffuse, non-specular vertex
// whose footprint a_suffix has reached `footprint` x a_0, and a share
// `train_fraction` of the paths is traced for training while queries are on.
// With `gate_bits`, a path queries, records a bootstrapped head or cuts its
// suffix into the cache only at a vertex whose cell of the gate grid is open
// (bit set); elsewhere it goes on as a plain path.  The training and unbiased
// draws then come from a per-pixel stream of their own, so that a path's own
// random numbers are those of a plain pass.
struct CachePolicy {
    float footprint = 0.01f;        // render.h:102
    float train_fraction = 0.05f;   // render.h:443
    const uint32_t* gate_bits = nullptr;   // kGateCells bits, null: every cell open
    float gate_lo[3] = {0.0f, 0.0f, 0.0f};
    float gate_inv[3] = {0.0f, 0.0f, 0.0f};   // kGateRes / (hi - lo) per axis
};

// render_pass with a device-side frame number (optional), the cache policy
// (null: the reference's), a prepare-only mode that validates and allocates
// without launching (so a later call can be captured in a CUDA graph), and
// the workspace slot to run on.
int render_pass_ex(const TfgRenderParams& prm, const TfgCamara* d_cam, const TfgPrimitiva* prims, int nprims,
                   const TfgLuzPuntual* lights, int nlights, int W, int H, int frame, const int32_t* frame_dev,
                   const CachePolicy* policy, const TfgTinyBVHD_GPU* bvh, const float* tris_wt,
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
    CachePolicy policy; int use_inf;
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
// (a = image, b = FP32 accumulation, cap = pixels), 4 tail queries of a gated
// frame (as 0, but a complete record -- no bootstrapped tail -- queries its
// head, for the gate update).
int launch_nrc_frame_small(int which, const void* a, void* b, const void* c, const uint32_t* n_dev, uint32_t cap,
                           uint32_t min_n, cudaStream_t s);

// Cache model internals used by the frame driver (nrc_mlp.cu).
struct ColorMlp;
int mlp_prepare(ColorMlp* n);
uint32_t* mlp_state(ColorMlp* n);
// The model's gate grid as a render pass reads it (allocated by
// mlp_set_gate_threshold with a threshold > 0).
void mlp_gate_view(ColorMlp* n, CachePolicy& p);
// Gate update after a frame's tail inference: every complete record (no
// bootstrapped tail) compares the cache's prediction at its head, which the
// gated tail queries put in `tail_pred`, with its own unbiased target, in the
// head's cell; then every cell's running relative error is set against the
// threshold.
int mlp_enqueue_gate_update(ColorMlp* n, const TfgRegistroEntrenamiento* regs, const TfgColor* tail_pred,
                            const uint32_t* n_dev, uint32_t cap, uint32_t min_n, cudaStream_t s);
uint32_t* mlp_navail(ColorMlp* n);
int mlp_enqueue_infer(ColorMlp* n, const TfgDatosMLP* in, TfgColor* out, TfgColor* img, const TfgColor* thr,
                      uint32_t max_count, const uint32_t* n_dev, cudaStream_t s);
int mlp_enqueue_train(ColorMlp* n, const TfgDatosMLP* buf, uint32_t min_n, cudaStream_t s);
int mlp_set_gate_threshold(ColorMlp* n, float g);
int mlp_precision(const ColorMlp* n);   // inference precision (part of a frame graph's identity)
uint32_t mlp_tuning_generation(const ColorMlp* n);   // changes with every tuning set

}  // namespace tfg
