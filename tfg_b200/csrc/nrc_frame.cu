// One radiance-cache frame on the GPU: the reference's per-frame host loop
// (main.cpp:995-1061) with every host synchronisation removed.
//
//   render (1 spp, cache queries + training records)      main.cpp:1016
//   cache inference fused with the composite              main.cpp:1028-1029
//   record count, capped and rounded to 4, in device memory main.cpp:1033-1039
//   tail queries -> tail inference -> targets             main.cpp:1046-1052
//   `train_steps` Adam steps on the targets               main.cpp:1056
//
// Counts and the step / Adam counters never leave the device, so the whole
// frame can be captured once as a CUDA graph and replayed; only the frame
// number (RNG seed) is written before each launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tfg_pt.h"
#include "tfg_errors.h"
#include "tfg_runtime.h"

namespace tfg {
namespace {

__global__ void k_set_frame(int32_t* frame_dev, int32_t frame) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *frame_dev = frame;
}

struct FrameKey {
    const void* ptrs[20];
    int32_t ints[20];
    float gate, footprint, train_fraction;
    bool operator==(const FrameKey& o) const { return std::memcmp(this, &o, sizeof(FrameKey)) == 0; }
};

struct FrameGraph {
    FrameKey key;
    bool valid = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

std::mutex g_frame_mutex;
int32_t* g_frame_dev[kMaxDevices] = {nullptr};
FrameGraph g_graph[kMaxDevices];

struct FrameCall {
    ColorMlp* mlp;
    TfgNrcFrameConfig cfg;
    TfgRenderParams prm;
    const TfgCamara* cam; const TfgPrimitiva* prims; int nprims;
    const TfgLuzPuntual* lights; int nlights;
    int W, H;
    const TfgTinyBVHD_GPU* bvh; const float* tris_wt; const TfgPrimitiva* mesh; int nmesh;
    TfgNrcBuffers b;
    int32_t* frame_dev;
    int ws_slot = 0;   // render workspace slot
    int branch = 0;    // branch of a batched frame that runs this scene's cache steps
};

int enqueue_cache_steps(const FrameCall& c, cudaStream_t s);

// The frame's cache policy: footprint and training share from the frame
// settings, the model's gate grid when the gate is on.
CachePolicy policy_of(const FrameCall& c) {
    CachePolicy p;
    p.footprint = c.cfg.footprint;
    p.train_fraction = c.cfg.train_fraction;
    mlp_gate_view(c.mlp, p);
    return p;
}

int enqueue_frame(const FrameCall& c, bool prepare_only, cudaStream_t s) {
    const CachePolicy pol = policy_of(c);
    if (prepare_only) {
        if (int rc = mlp_prepare(c.mlp)) return rc;
    } else {
        cudaError_t e = cudaMemsetAsync(c.b.counter, 0, sizeof(uint32_t), s);
        if (e != cudaSuccess) return fail((int)e, std::string("nrc frame: ") + cudaGetErrorString(e));
    }
    if (int rc = render_pass_ex(c.prm, c.cam, c.prims, c.nprims, c.lights, c.nlights, c.W, c.H, 0, c.frame_dev, &pol,
                                c.bvh, c.tris_wt, c.mesh, c.nmesh, c.b.img, nullptr, c.b.regs, c.b.counter,
                                (int)c.b.ring_cap, c.b.infer, c.b.thr, c.cfg.warmup ? 0 : 1, 1, prepare_only,
                                c.ws_slot, s))
        return rc;
    if (prepare_only) return ok();
    return enqueue_cache_steps(c, s);
}

// The scene as one member of a batched render pass.
PassScene pass_scene(const FrameCall& c) {
    PassScene p{};
    p.cam = c.cam; p.prims = c.prims; p.nprims = c.nprims; p.lights = c.lights; p.nlights = c.nlights;
    p.W = c.W; p.H = c.H;
    p.bvh = c.bvh; p.tris_wt = c.tris_wt; p.mesh = c.mesh; p.nmesh = c.nmesh;
    p.img = c.b.img; p.accum = nullptr;
    p.regs = c.b.regs; p.reg_counter = c.b.counter; p.reg_cap = (int)c.b.ring_cap;
    p.infer = c.b.infer; p.thr_out = c.b.thr;
    p.policy = policy_of(c);
    p.use_inf = c.cfg.warmup ? 0 : 1;
    return p;
}

// After the render: answer and composite the cache queries, accumulate,
// bootstrap targets from the tail queries and train (main.cpp:1016-1061).
int enqueue_cache_steps(const FrameCall& c, cudaStream_t s) {
    const uint32_t npx = (uint32_t)c.W * (uint32_t)c.H;
    const uint32_t min_n = std::max(c.cfg.min_records + 1u, 100u);
    uint32_t* navail = mlp_navail(c.mlp);
    if (int rc = mlp_enqueue_infer(c.mlp, c.b.infer, nullptr, c.b.img, c.b.thr, npx, nullptr, s)) return rc;
    if (c.b.accum)
        if (int rc = launch_nrc_frame_small(3, c.b.img, c.b.accum, nullptr, nullptr, npx, 0, s)) return rc;
    if (int rc = launch_nrc_frame_small(2, c.b.counter, navail, nullptr, nullptr, c.cfg.max_records, 0, s)) return rc;
    const bool gated = c.cfg.gate_threshold > 0.0f;
    if (int rc = launch_nrc_frame_small(gated ? 4 : 0, c.b.regs, c.b.tail_in, nullptr, navail, c.cfg.max_records,
                                        min_n, s))
        return rc;
    if (int rc = mlp_enqueue_infer(c.mlp, c.b.tail_in, c.b.tail_pred, nullptr, nullptr, c.cfg.max_records, navail, s))
        return rc;
    if (int rc = launch_nrc_frame_small(1, c.b.regs, c.b.train_buf, c.b.tail_pred, navail, c.cfg.max_records, min_n, s))
        return rc;
    if (gated)
        if (int rc = mlp_enqueue_gate_update(c.mlp, c.b.regs, c.b.tail_pred, navail, c.cfg.max_records, min_n, s))
            return rc;
    for (int k = 0; k < c.cfg.train_steps; ++k)
        if (int rc = mlp_enqueue_train(c.mlp, c.b.train_buf, min_n, s)) return rc;
    return ok();
}

int current_device() {
    int dev = 0;
    cudaGetDevice(&dev);
    return dev;
}

// Launch tuning of the current device: a change re-captures the frame graph.
uint32_t render_generation() {
    uint32_t g = 0;
    render_tuning_get(current_device(), nullptr, &g);
    return g;
}

FrameKey key_of(const FrameCall& c) {
    FrameKey k;
    std::memset(&k, 0, sizeof(k));
    const void* p[] = {c.mlp, c.cam, c.prims, c.lights, c.bvh ? c.bvh->d_nodos : nullptr,
                       c.bvh ? c.bvh->d_tris : nullptr, c.tris_wt, c.mesh, c.b.img, c.b.accum, c.b.infer, c.b.thr,
                       c.b.regs, c.b.counter, c.b.tail_in, c.b.tail_pred, c.b.train_buf, c.frame_dev};
    std::memcpy(k.ptrs, p, sizeof(p));
    const int32_t v[] = {c.nprims, c.nlights, c.W, c.H, c.nmesh, (int32_t)c.b.ring_cap, c.cfg.train_steps,
                         (int32_t)c.cfg.max_records, (int32_t)c.cfg.min_records, c.cfg.warmup, c.prm.max_depth,
                         c.prm.rr_min_depth, c.prm.shadow_mesh, c.prm.tri_format, c.ws_slot,
                         mlp_precision(c.mlp), (int32_t)render_generation(), (int32_t)mlp_tuning_generation(c.mlp),
                         (int32_t)workspace_generation(current_device(), c.ws_slot), c.branch};
    static_assert(sizeof(v) <= sizeof(k.ints), "frame key: too many ints");
    std::memcpy(k.ints, v, sizeof(v));
    k.gate = c.cfg.gate_threshold;
    k.footprint = c.cfg.footprint;
    k.train_fraction = c.cfg.train_fraction;
    return k;
}

// Validated FrameCall from the public arguments (spp 1, no accumulation or
// profiling inside a frame).
int make_call(TfgColorMLP* mlp, const TfgNrcFrameConfig* cfg, const TfgRenderParams* params,
              const TfgCamara* camara, const TfgPrimitiva* primitivas, int32_t num_primitivas,
              const TfgLuzPuntual* luces, int32_t num_luces, int32_t W, int32_t H, const TfgTinyBVHD_GPU* bvh,
              const float* tris_wt, const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh,
              const TfgNrcBuffers* buffers, int32_t* frame_dev, FrameCall& c) {
    if (!mlp || !cfg || !params || !buffers) return fail(TFG_E_INVALID, "nrc frame: null argument");
    const TfgNrcBuffers& b = *buffers;
    if (!b.img || !b.infer || !b.thr || !b.regs || !b.counter || !b.tail_in || !b.tail_pred || !b.train_buf)
        return fail(TFG_E_INVALID, "nrc frame: a required buffer is null");
    if (cfg->train_steps < 0 || cfg->max_records == 0 || b.ring_cap < cfg->max_records)
        return fail(TFG_E_INVALID, "nrc frame: ring capacity below max_records");
    if (!(cfg->footprint >= 0.0f) || !(cfg->train_fraction >= 0.0f && cfg->train_fraction <= 1.0f) ||
        !(cfg->gate_threshold >= 0.0f))
        return fail(TFG_E_INVALID, "nrc frame: footprint, gate_threshold >= 0 and train_fraction in [0, 1]");
    c.mlp = reinterpret_cast<ColorMlp*>(mlp);
    c.cfg = *cfg;
    c.prm = *params;
    c.prm.spp = 1;
    c.prm.accumulate = 0;
    c.prm.profile = 0;
    c.cam = camara; c.prims = primitivas; c.nprims = num_primitivas; c.lights = luces; c.nlights = num_luces;
    c.W = W; c.H = H; c.bvh = bvh; c.tris_wt = tris_wt; c.mesh = primitivas_bvh; c.nmesh = num_prims_bvh;
    c.b = b;
    c.frame_dev = frame_dev;
    c.ws_slot = 0;
    return ok();
}

int frame_word(int dev, int32_t** out) {
    if (!g_frame_dev[dev]) {
        cudaError_t e = cudaMalloc((void**)&g_frame_dev[dev], sizeof(int32_t));
        if (e != cudaSuccess) return fail((int)e, std::string("nrc frame: ") + cudaGetErrorString(e));
    }
    *out = g_frame_dev[dev];
    return ok();
}

// ------------------------------------------------------------------ batched frames
struct BatchGraph {
    std::vector<FrameKey> keys;
    bool valid = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};
BatchGraph g_batch[kMaxDevices];
cudaStream_t g_branch[kMaxDevices][kWorkspaceSlots] = {};
cudaEvent_t g_fork[kMaxDevices] = {};
cudaEvent_t g_join[kMaxDevices][kWorkspaceSlots] = {};

int branch_resources(int dev, int nb) {
    cudaError_t e = cudaSuccess;
    if (!g_fork[dev]) e = cudaEventCreateWithFlags(&g_fork[dev], cudaEventDisableTiming);
    for (int b = 1; b < nb && e == cudaSuccess; ++b) {
        if (!g_branch[dev][b]) e = cudaStreamCreateWithFlags(&g_branch[dev][b], cudaStreamNonBlocking);
        if (e == cudaSuccess && !g_join[dev][b])
            e = cudaEventCreateWithFlags(&g_join[dev][b], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrameBatch: ") + cudaGetErrorString(e));
    return ok();
}

// Scenes that share their render settings (at most 16) render as one
// wavefront series; otherwise each scene renders on its own branch.
bool merged_render(const std::vector<FrameCall>& calls) {
    if (calls.size() > 16) return false;
    for (const FrameCall& c : calls) {
        const TfgRenderParams& p = c.prm, & q = calls[0].prm;
        if (p.max_depth != q.max_depth || p.rr_min_depth != q.rr_min_depth || p.shadow_mesh != q.shadow_mesh ||
            p.tri_format != q.tri_format || p.spp != q.spp || p.profile != q.profile)
            return false;
    }
    return true;
}

int render_merged(const std::vector<FrameCall>& calls, bool prepare_only, cudaStream_t s) {
    PassScene ps[16];
    for (size_t i = 0; i < calls.size(); ++i) ps[i] = pass_scene(calls[i]);
    return render_pass_multi(calls[0].prm, ps, (int)calls.size(), 0, calls[0].frame_dev, 1, prepare_only, 0, s);
}

// Fork `nb` branches off `s`, enqueue every scene on its branch, join back.
// With `merged`, the scenes render first as one wavefront series on `s` and
// only their cache steps run on the branches.
int enqueue_batch(const std::vector<FrameCall>& calls, int nb, int dev, bool merged, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    int rc = 0;
    if (merged) {
        for (const FrameCall& c : calls)
            if (e == cudaSuccess) e = cudaMemsetAsync(c.b.counter, 0, sizeof(uint32_t), s);
        if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrameBatch: ") + cudaGetErrorString(e));
        if (int r = render_merged(calls, false, s)) return r;
    }
    e = cudaEventRecord(g_fork[dev], s);
    for (int b = 1; b < nb && e == cudaSuccess; ++b) e = cudaStreamWaitEvent(g_branch[dev][b], g_fork[dev], 0);
    if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrameBatch fork: ") + cudaGetErrorString(e));
    for (const FrameCall& c : calls) {
        cudaStream_t bs = c.branch == 0 ? s : g_branch[dev][c.branch];
        rc = merged ? enqueue_cache_steps(c, bs) : enqueue_frame(c, false, bs);
        if (rc) break;
    }
    // join every branch even after a failure, so a capture can end cleanly
    for (int b = 1; b < nb; ++b) {
        cudaError_t e2 = cudaEventRecord(g_join[dev][b], g_branch[dev][b]);
        if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(s, g_join[dev][b], 0);
        if (e2 != cudaSuccess && !rc) rc = fail((int)e2, std::string("tfgNrcFrameBatch join: ") + cudaGetErrorString(e2));
    }
    return rc;
}

}  // namespace
}  // namespace tfg

extern "C" void tfgNrcFrameConfigReference(TfgNrcFrameConfig* c) {
    if (!c) return;
    c->train_steps = 1;
    c->max_records = 65536;
    c->min_records = 1024;
    c->warmup = 0;
    c->gate_threshold = 0.0f;
    c->use_graph = 0;
    c->footprint = 0.01f;
    c->train_fraction = 0.05f;
}

extern "C" int tfgNrcFrame(TfgColorMLP* mlp, const TfgNrcFrameConfig* cfg, const TfgRenderParams* params,
                           const TfgCamara* camara, const TfgPrimitiva* primitivas, int32_t num_primitivas,
                           const TfgLuzPuntual* luces, int32_t num_luces, int32_t W, int32_t H,
                           const TfgTinyBVHD_GPU* bvh, const float* tris_wt, const TfgPrimitiva* primitivas_bvh,
                           int32_t num_prims_bvh, const TfgNrcBuffers* buffers, int32_t frame, void* stream) {
    using namespace tfg;
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    std::lock_guard<std::mutex> lk(g_frame_mutex);
    int32_t* frame_dev = nullptr;
    if (int rc = frame_word(dev, &frame_dev)) return rc;
    FrameCall c;
    if (int rc = make_call(mlp, cfg, params, camara, primitivas, num_primitivas, luces, num_luces, W, H, bvh, tris_wt,
                           primitivas_bvh, num_prims_bvh, buffers, frame_dev, c))
        return rc;
    if (int rc = mlp_set_gate_threshold(c.mlp, cfg->gate_threshold)) return rc;
    k_set_frame<<<1, 32, 0, s>>>(c.frame_dev, frame);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrame: ") + cudaGetErrorString(e));
    const bool graph = cfg->use_graph && s != nullptr;
    if (!graph) {
        if (int rc = enqueue_frame(c, true, s)) return rc;
        return enqueue_frame(c, false, s);
    }
    FrameGraph& g = g_graph[dev];
    // Prepare first: a workspace that had to grow since the capture changes
    // the key, and the frame is captured again.
    if (int rc = enqueue_frame(c, true, s)) return rc;
    const FrameKey key = key_of(c);
    if (!g.valid || !(g.key == key)) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
        g.exec = nullptr; g.graph = nullptr; g.valid = false;
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrame capture: ") + cudaGetErrorString(e));
        const int rc = enqueue_frame(c, false, s);
        cudaGraph_t gr = nullptr;
        e = cudaStreamEndCapture(s, &gr);
        if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
        if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrame capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&g.exec, gr, 0);
        if (e != cudaSuccess) { cudaGraphDestroy(gr); return fail((int)e, std::string("tfgNrcFrame instantiate: ") + cudaGetErrorString(e)); }
        g.graph = gr;
        g.key = key;
        g.valid = true;
    }
    e = cudaGraphLaunch(g.exec, s);
    if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrame launch: ") + cudaGetErrorString(e));
    return ok();
}

extern "C" int tfgNrcFrameBatch(int32_t n, const TfgNrcSceneFrame* scenes, int32_t frame, int32_t use_graph,
                                void* stream) {
    using namespace tfg;
    if (n < 0 || (n > 0 && !scenes)) return fail(TFG_E_INVALID, "tfgNrcFrameBatch: bad scene array");
    if (n == 0) return ok();
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    std::lock_guard<std::mutex> lk(g_frame_mutex);
    int32_t* frame_dev = nullptr;
    if (int rc = frame_word(dev, &frame_dev)) return rc;
    std::vector<FrameCall> calls((size_t)n);
    for (int i = 0; i < n; ++i) {
        const TfgNrcSceneFrame& f = scenes[i];
        if (int rc = make_call(f.mlp, f.cfg, f.params, f.camara, f.primitivas, f.num_primitivas, f.luces, f.num_luces,
                               f.ancho_img, f.alto_img, f.bvh, f.tris_wt, f.primitivas_bvh, f.num_prims_bvh, f.buffers,
                               frame_dev, calls[(size_t)i]))
            return rc;
        for (int j = 0; j < i; ++j)
            if (calls[(size_t)j].mlp == calls[(size_t)i].mlp || calls[(size_t)j].b.img == calls[(size_t)i].b.img ||
                calls[(size_t)j].b.regs == calls[(size_t)i].b.regs)
                return fail(TFG_E_INVALID, "tfgNrcFrameBatch: scenes share a cache model or buffers");
    }
    // Largest scenes first, each to the branch with the fewest pixels so far.
    const int nb = std::min(n, kWorkspaceSlots);
    std::vector<int> order((size_t)n);
    for (int i = 0; i < n; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return (int64_t)calls[(size_t)x].W * calls[(size_t)x].H > (int64_t)calls[(size_t)y].W * calls[(size_t)y].H;
    });
    const bool merged = merged_render(calls);
    std::vector<int64_t> load((size_t)nb, 0);
    for (int i : order) {
        const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        calls[(size_t)i].branch = b;
        calls[(size_t)i].ws_slot = merged ? 0 : b;
        load[(size_t)b] += (int64_t)calls[(size_t)i].W * calls[(size_t)i].H;
    }
    if (int rc = branch_resources(dev, nb)) return rc;
    for (const FrameCall& c : calls) {
        if (int rc = mlp_set_gate_threshold(c.mlp, c.cfg.gate_threshold)) return rc;
        if (merged) {
            if (int rc = mlp_prepare(c.mlp)) return rc;
        } else if (int rc = enqueue_frame(c, true, s)) {
            return rc;
        }
    }
    if (merged)
        if (int rc = render_merged(calls, true, s)) return rc;
    k_set_frame<<<1, 32, 0, s>>>(frame_dev, frame);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrameBatch: ") + cudaGetErrorString(e));
    if (!(use_graph && s != nullptr)) return enqueue_batch(calls, nb, dev, merged, s);
    BatchGraph& g = g_batch[dev];
    std::vector<FrameKey> keys;
    for (const FrameCall& c : calls) keys.push_back(key_of(c));
    if (!g.valid || g.keys.size() != keys.size() ||
        !std::equal(keys.begin(), keys.end(), g.keys.begin())) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
        g.exec = nullptr; g.graph = nullptr; g.valid = false;
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrameBatch capture: ") + cudaGetErrorString(e));
        const int rc = enqueue_batch(calls, nb, dev, merged, s);
        cudaGraph_t gr = nullptr;
        e = cudaStreamEndCapture(s, &gr);
        if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
        if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrameBatch capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&g.exec, gr, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(gr);
            return fail((int)e, std::string("tfgNrcFrameBatch instantiate: ") + cudaGetErrorString(e));
        }
        g.graph = gr;
        g.keys = keys;
        g.valid = true;
    }
    e = cudaGraphLaunch(g.exec, s);
    if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcFrameBatch launch: ") + cudaGetErrorString(e));
    return ok();
}

// The reference's reconstruction mode (main.cpp:454-668) without its host
// round trips: `spp` samples, each rendered with cache queries and no
// training (main.cpp:566-575), answered by the cache and composited
// (main.cpp:594-595), and summed into `accum` on the device (main.cpp:600-603).
extern "C" int tfgNrcReconstruct(TfgColorMLP* mlp, const TfgRenderParams* params, const TfgCamara* camara,
                                 const TfgPrimitiva* primitivas, int32_t num_primitivas, const TfgLuzPuntual* luces,
                                 int32_t num_luces, int32_t W, int32_t H, const TfgTinyBVHD_GPU* bvh,
                                 const float* tris_wt, const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh,
                                 int32_t spp, int32_t first_frame, TfgColor* img, TfgDatosMLP* infer, TfgColor* thr,
                                 float* accum, void* stream) {
    using namespace tfg;
    if (!mlp || !params || !img || !infer || !thr || !accum) return fail(TFG_E_INVALID, "tfgNrcReconstruct: null argument");
    if (spp < 1) return fail(TFG_E_INVALID, "tfgNrcReconstruct: spp < 1");
    if (W <= 0 || H <= 0) return fail(TFG_E_INVALID, "tfgNrcReconstruct: bad image size");
    cudaStream_t s = (cudaStream_t)stream;
    ColorMlp* m = reinterpret_cast<ColorMlp*>(mlp);
    TfgRenderParams prm = *params;
    prm.spp = 1;
    prm.accumulate = 0;
    prm.profile = 0;
    const uint32_t npx = (uint32_t)W * (uint32_t)H;
    cudaError_t e = cudaMemsetAsync(accum, 0, (size_t)npx * 3 * sizeof(float), s);
    if (e != cudaSuccess) return fail((int)e, std::string("tfgNrcReconstruct: ") + cudaGetErrorString(e));
    for (int k = 0; k < spp; ++k) {
        if (int rc = render_pass_ex(prm, camara, primitivas, num_primitivas, luces, num_luces, W, H, first_frame + k,
                                    nullptr, nullptr, bvh, tris_wt, primitivas_bvh, num_prims_bvh, img, nullptr,
                                    nullptr, nullptr, 0, infer, thr, 1, 0, false, 0, s))
            return rc;
        if (int rc = mlp_enqueue_infer(m, infer, nullptr, img, thr, npx, nullptr, s)) return rc;
        if (int rc = launch_nrc_frame_small(3, img, accum, nullptr, nullptr, npx, 0, s)) return rc;
    }
    return ok();
}

extern "C" int tfgMlpGetState(TfgColorMLP* mlp, uint32_t* out8) {
    using namespace tfg;
    if (!mlp || !out8) return fail(TFG_E_INVALID, "tfgMlpGetState: null argument");
    cudaError_t e = cudaMemcpy(out8, mlp_state(reinterpret_cast<ColorMlp*>(mlp)), 8 * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail((int)e, std::string("tfgMlpGetState: ") + cudaGetErrorString(e));
    return ok();
}
