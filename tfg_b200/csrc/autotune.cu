// The render autotuner: picks the wavefront launch settings of one device by
// timing plain passes of the caller's scene.
//
// The settings (TfgRenderTuning) change only how the same paths are
// scheduled -- the wavefront (queue) size, the traversal CTA size and
// residency, the refill threshold of the persistent traversal lanes, how
// many lanes share a shading point's shadow rays, the first bounce's refill
// threshold, and whether the shadow stage overlaps the next trace -- never
// what a path
// computes, so every candidate renders the same image.  The search is one
// pass of coordinate descent in that order, starting from the device's
// current setting; a candidate replaces the best only when it is at least 1%
// faster, so run-to-run noise does not move the setting.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/tfg_pt.h"
#include "tfg_errors.h"
#include "tfg_runtime.h"

namespace tfg {
namespace {

struct TuneScene {
    TfgRenderParams prm;
    const TfgCamara* cam; const TfgPrimitiva* prims; int nprims;
    const TfgLuzPuntual* lights; int nlights;
    int W, H;
    const TfgTinyBVHD_GPU* bvh; const float* tris_wt; const TfgPrimitiva* mesh; int nmesh;
};

int one_pass(const TuneScene& sc, int frame, cudaStream_t s) {
    return render_pass_ex(sc.prm, sc.cam, sc.prims, sc.nprims, sc.lights, sc.nlights, sc.W, sc.H, frame, nullptr,
                          nullptr, sc.bvh, sc.tris_wt, sc.mesh, sc.nmesh, nullptr, nullptr, nullptr, nullptr, 0, nullptr,
                          nullptr, 0, 0, false, 0, s);
}

// Mean pass time of `t`: one warm-up pass (which also sizes the workspace
// outside the timed region), then `repeats` passes between two events.
int time_tuning(int dev, const TuneScene& sc, const TfgRenderTuning& t, int repeats, cudaStream_t s, cudaEvent_t e0,
                cudaEvent_t e1, float* ms) {
    if (int rc = render_tuning_set(dev, t)) return rc;
    if (int rc = one_pass(sc, 0, s)) return rc;
    cudaError_t e = cudaEventRecord(e0, s);
    if (e != cudaSuccess) return fail((int)e, std::string("tfgRenderAutotune: ") + cudaGetErrorString(e));
    for (int r = 0; r < repeats; ++r)
        if (int rc = one_pass(sc, 1 + r * sc.prm.spp, s)) return rc;
    e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    if (e != cudaSuccess) return fail((int)e, std::string("tfgRenderAutotune: ") + cudaGetErrorString(e));
    *ms /= (float)repeats;
    return ok();
}

// Candidate values of setting `k` for a call of `paths` paths over `npix`
// pixels.
std::vector<int32_t> candidates(int k, uint32_t npix, uint64_t paths) {
    std::vector<int32_t> v;
    switch (k) {
        case 0: {   // wavefront: 1/8 .. 16 samples of the image, 0 = exactly one
            v.push_back(0);
            const uint64_t sizes[] = {npix / 8u, npix / 4u, npix / 2u, 2ull * npix, 4ull * npix, 8ull * npix,
                                      16ull * npix};
            for (uint64_t w : sizes)
                if (w >= 1024 && w <= (1u << 26) && w <= paths) v.push_back((int32_t)w);
            break;
        }
        case 1: v = {64, 128, 256}; break;
        case 2: v = {0, 8, 16, 24}; break;
        case 3: v = {4, 8, 12, 16, 24, 32}; break;
        case 4: v = {0, 1}; break;
        case 5: v = {0, 16, 24, 32}; break;
        case 6: v = {0, 1}; break;
    }
    return v;
}

int32_t& field(TfgRenderTuning& t, int k) {
    switch (k) {
        case 0: return t.wavefront_paths;
        case 1: return t.trace_threads;
        case 2: return t.trace_warps_per_sm;
        case 3: return t.refill_min;
        case 4: return t.shadow_one_lane;
        case 5: return t.refill_min_primary;
        default: return t.overlap_shadow;
    }
}

}  // namespace
}  // namespace tfg

extern "C" int tfgRenderAutotune(const TfgRenderParams* params, const TfgCamara* camara,
                                 const TfgPrimitiva* primitivas, int32_t num_primitivas, const TfgLuzPuntual* luces,
                                 int32_t num_luces, int32_t ancho_img, int32_t alto_img,
                                 const TfgTinyBVHD_GPU* nodos_bvh, const float* tris_wt,
                                 const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh, int32_t repeats,
                                 TfgRenderTuning* out, TfgTuneRecord* records, int32_t max_records,
                                 int32_t* num_records, void* stream) {
    using namespace tfg;
    if (!params) return fail(TFG_E_INVALID, "tfgRenderAutotune: params is null");
    if (records && max_records < 0) return fail(TFG_E_INVALID, "tfgRenderAutotune: negative max_records");
    if (ancho_img <= 0 || alto_img <= 0) return fail(TFG_E_INVALID, "tfgRenderAutotune: bad image size");
    if (params->spp < 1) return fail(TFG_E_INVALID, "tfgRenderAutotune: spp < 1");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    TuneScene sc{*params, camara, primitivas, num_primitivas, luces, num_luces, ancho_img, alto_img,
                 nodos_bvh, tris_wt, primitivas_bvh, num_prims_bvh};
    sc.prm.spp = std::min(params->spp, 16);
    sc.prm.accumulate = 0;
    sc.prm.profile = 0;
    repeats = repeats > 0 ? std::min(repeats, 100) : 3;
    const uint32_t npix = (uint32_t)ancho_img * (uint32_t)alto_img;
    const uint64_t paths = (uint64_t)sc.prm.spp * npix;

    TfgRenderTuning start;
    render_tuning_get(dev, &start, nullptr);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    int rc = e == cudaSuccess ? 0 : fail((int)e, std::string("tfgRenderAutotune: ") + cudaGetErrorString(e));
    int32_t nrec = 0;
    auto record = [&](const TfgRenderTuning& t, float ms) {
        if (records && nrec < max_records) {
            records[nrec].tuning = t;
            records[nrec].ms = ms;
            records[nrec].reserved = 0;
        }
        ++nrec;
    };
    TfgRenderTuning best = start;
    float best_ms = 0.0f;
    if (!rc) rc = time_tuning(dev, sc, best, repeats, s, e0, e1, &best_ms);
    if (!rc) record(best, best_ms);
    for (int k = 0; k < 7 && !rc; ++k) {
        for (int32_t v : candidates(k, npix, paths)) {
            TfgRenderTuning cand = best;
            if (field(cand, k) == v) continue;
            field(cand, k) = v;
            if (render_tuning_check(cand) != 0) { ok(); continue; }
            float ms = 0.0f;
            rc = time_tuning(dev, sc, cand, repeats, s, e0, e1, &ms);
            if (rc) break;
            record(cand, ms);
            if (ms < 0.99f * best_ms) { best = cand; best_ms = ms; }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc) {
        render_tuning_set(dev, start);
        return rc;
    }
    if (num_records) *num_records = nrec;
    if (out) *out = best;
    return render_tuning_set(dev, best);
}
