// Wavefront path tracer: the reference's per-pixel megakernel
// (RenderKernel.cu:28-47 -> render.h:416-466 -> render.h:33-262) split into
// queue stages.
//
//   generate   one thread per pixel: RNG seed + jitter + NRC draws, camera ray
//   trace      persistent warps pull rays from the queue (one atomic per warp),
//              closest hit over analytic primitives then the CWBVH
//   shade      emission, NRC footprint / capture logic, BSDF sampling, Russian
//              roulette; survivors are compacted into the next ray queue and
//              diffuse hits into the shadow queue (warp ballot + one atomic)
//   shadow     next-event estimation to every point light, in light order,
//              added to the path's radiance
//   resolve    per pixel: image, accumulation, inference/throughput buffers,
//              training records
//
// A path's bounce count equals the queue it sits in, so no depth is stored.
// Random numbers are drawn in the reference's order, so a path consumes the
// same stream as in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/tfg_pt.h"
#include "cwbvh_traverse.cuh"
#include "pt_common.cuh"
#include "tfg_errors.h"
#include "tfg_runtime.h"

namespace tfg {

// ------------------------------------------------------------------ state
enum : uint32_t {
    F_TRAIN = 1u,       // es_ruta_entrenamiento (render.h:443)
    F_UNBIASED = 2u,    // es_ruta_insesgada (render.h:65)
    F_CAPTURED = 4u,    // punto_entrenamiento_encontrado
    F_INF = 8u,         // inference query written by shade
    F_TAIL = 16u,       // tail vertex recorded
    F_FULL = 32u,       // training path whose head lies in a closed gate cell: its suffix runs to the end
                        // and its radiance counts in the pixel as well (a plain path with a record)
};

constexpr uint32_t kMissId = 0xFFFFFFFFu;

// Traversal work totals for TFG_PROFILE_COUNTS: rays, nodes, triangle tests
// for closest-hit rays, then the same for shadow rays.
__device__ unsigned long long g_work[6];

__device__ __forceinline__ void flush_work(int base, uint32_t rays, const TravCounts& c) {
    unsigned long long v[3] = {rays, c.nodes, c.tris};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        unsigned long long x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, o);
        if ((threadIdx.x & 31u) == 0 && x) atomicAdd(&g_work[base + k], x);
    }
}
constexpr uint32_t kAnalyticBit = 0x80000000u;
constexpr int kMaxBounces = 64;
constexpr int kSmemPrims = 128;

struct Workspace {
    size_t cap = 0;          // paths
    size_t train_cap = 0;    // paths with training scratch
    float4* ray[2] = {nullptr, nullptr};   // 2 float4 per ray: (O, tmax), (D, pixel)
    float4* hit = nullptr;                  // (t, u, v, id)
    float4* shadow = nullptr;               // 4 float4 per item
    float4* thr = nullptr;                  // camino.rgb, ior
    uint4* st = nullptr;                    // rng, flags, pdf bits, -
    float4* lpre = nullptr;                 // L_pre.rgb, a_0
    float4* lsuf = nullptr;                 // L_suf.rgb, a_current
    float4* nrc = nullptr;                  // a_suffix, a_prefix
    float4* ts = nullptr;                   // training scratch, 10 float4 per path
    uint32_t* counters = nullptr;           // per bounce: rays, fetch, shadows, spare
    uint32_t generation = 0;                // changes whenever a buffer is reallocated
    // A second stream for the shadow stage, which then runs beside the next
    // bounce's closest-hit trace: fork / join events per bounce.
    cudaStream_t side = nullptr;
    cudaEvent_t fork[kMaxBounces] = {};
    cudaEvent_t join[kMaxBounces] = {};
};

struct PassArgs {
    const TfgPrimitiva* prims; int nprims;
    const TfgLuzPuntual* lights; int nlights;
    const float4* nodes; const float4* tris; int has_bvh;
    const TfgPrimitiva* mesh; int nmesh;
    const TfgCamara* cam;        // device pointer, read by k_generate
    const int32_t* frame_dev;    // optional device-side base frame number
    CachePolicy pol;             // footprint, training share, gate grid
    int W, H, frame;
    TfgColor* img; float* accum;
    TfgRegistroEntrenamiento* regs; uint32_t* reg_counter; int reg_cap;
    TfgDatosMLP* infer; TfgColor* thr_out;
    int use_inf, train;
    int max_depth, rr_min_depth, shadow_mesh;
    // The call's paths are `spp` samples of every pixel, numbered sample-major
    // (path q = sample * npix + pixel).  A wavefront runs `nq` consecutive
    // paths starting at pixel p0 of sample s0; its per-path state is indexed
    // by the path's slot in the wavefront (0 .. nq-1).
    uint32_t npix, nq, p0;
    int s0, last_sample;      // samples relative to `frame`; the last one writes `img`
    int refill_min;           // idle lanes that trigger a traversal warp's refill
    int refill_primary;       // the same for the first bounce
    int shadow_one_lane;      // 1: one lane traces all lights of a shading point
    Workspace ws;
};

// Several scenes in one wavefront (a batch): the scenes' pixels are
// concatenated (scene i owns global pixels pix0 .. pix0 + W*H - 1) and every
// path carries its scene index, in the ray queue entry's first w (closest-hit
// rays always start with t_max = 1e9) and in the shadow item.  The table
// travels by value in the kernel parameters, so a captured graph keeps the
// table it was captured with.
constexpr int kMaxBatchScenes = 16;
struct SceneDesc {
    const TfgPrimitiva* prims; const TfgLuzPuntual* lights;
    const float4* nodes; const float4* tris; const TfgPrimitiva* mesh;
    const TfgCamara* cam; CachePolicy pol;
    TfgColor* img; float* accum;
    TfgRegistroEntrenamiento* regs; uint32_t* reg_counter;
    TfgDatosMLP* infer; TfgColor* thr_out;
    int nprims, nlights, has_bvh, nmesh, W, H, reg_cap, use_inf;
    uint32_t pix0;
};
struct SceneTable {
    SceneDesc s[kMaxBatchScenes];
    int n;
};
struct NoTable {};
template <bool MS> using TableOf = typename std::conditional<MS, SceneTable, NoTable>::type;

// The geometry a path sees.
struct Geo {
    const TfgPrimitiva* prims; const float4* nodes; const float4* tris; const TfgPrimitiva* mesh;
    int nprims, has_bvh;
};

// Per-pixel outputs of a path's scene.
struct Outs {
    TfgColor* img; float* accum;
    TfgRegistroEntrenamiento* regs; uint32_t* reg_counter; int reg_cap;
    TfgDatosMLP* infer; TfgColor* thr_out;
};

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

template <bool MS>
__device__ __forceinline__ Geo geo_of(const PassArgs& a, const TableOf<MS>& tab, uint32_t sc) {
    if constexpr (MS) {
        const SceneDesc& d = tab.s[sc];
        return Geo{d.prims, d.nodes, d.tris, d.mesh, d.nprims, d.has_bvh};
    } else {
        (void)tab; (void)sc;
        return Geo{a.prims, a.nodes, a.tris, a.mesh, a.nprims, a.has_bvh};
    }
}

template <bool MS>
__device__ __forceinline__ Outs outs_of(const PassArgs& a, const TableOf<MS>& tab, uint32_t sc) {
    if constexpr (MS) {
        const SceneDesc& d = tab.s[sc];
        return Outs{d.img, d.accum, d.regs, d.reg_counter, d.reg_cap, d.infer, d.thr_out};
    } else {
        (void)tab; (void)sc;
        return Outs{a.img, a.accum, a.regs, a.reg_counter, a.reg_cap, a.infer, a.thr_out};
    }
}

// Scene owning global pixel g (scenes in pixel order).
__device__ __forceinline__ uint32_t scene_of_pixel(const SceneTable& tab, uint32_t g) {
    uint32_t sc = 0;
    while ((int)sc + 1 < tab.n && g >= tab.s[sc + 1].pix0) ++sc;
    return sc;
}

// Pixel (y * W + x) of the l-th path of a sample of a W x H image: bands of
// 4 rows cut into 8 x 4 tiles left to right (the band's last tile narrower
// when W is not a multiple of 8, the last band lower when H is not a
// multiple of 4), so the 32 paths of a warp start from one 8 x 4 block of
// pixels and their primary and first shadow rays stay coherent.  A
// bijection on [0, W*H).
__host__ __device__ __forceinline__ uint32_t tiled_pixel(uint32_t l, uint32_t W, uint32_t H) {
    const uint32_t band = l / (4u * W), y0 = 4u * band;
    const uint32_t h = H - y0 < 4u ? H - y0 : 4u;
    const uint32_t o = l - band * 4u * W;
    const uint32_t full = W / 8u;
    uint32_t x, y;
    if (o < full * 8u * h) {
        const uint32_t tc = o / (8u * h), i = o - tc * 8u * h;
        x = 8u * tc + (i & 7u);
        y = y0 + (i >> 3);
    } else {
        const uint32_t wr = W - 8u * full, i = o - full * 8u * h;
        x = 8u * full + i % wr;
        y = y0 + i / wr;
    }
    return y * W + x;
}

// Warp-aggregated queue append: every lane with `want` gets a unique slot.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
    const uint32_t mask = __activemask();
    const uint32_t vote = __ballot_sync(mask, want);
    if (!vote) return 0xFFFFFFFFu;
    const uint32_t leader = __ffs(vote) - 1u;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(counter, (uint32_t)__popc(vote));
    base = __shfl_sync(mask, base, leader);
    return want ? base + __popc(vote & ((1u << lane_id()) - 1u)) : 0xFFFFFFFFu;
}

__device__ __forceinline__ V3 xyz(float4 a) { return v3(a.x, a.y, a.z); }

__device__ __forceinline__ const TfgPrimitiva* prim_of(const Geo& g, uint32_t id) {
    return (id & kAnalyticBit) ? &g.prims[id & ~kAnalyticBit] : &g.mesh[id];
}

// Closest analytic hit (escenario.h:323-334): strict t < best, t > 1e-6.
__device__ __forceinline__ int analytic_closest(const APrim* sp, int nsm, const TfgPrimitiva* gp, int n, V3 O, V3 D,
                                                float& best, float& bu, float& bv) {
    int hit = -1;
    for (int i = 0; i < n; ++i) {
        APrim q;
        if (i < nsm) q = sp[i];
        else aprim_load(gp[i], q);
        float t, u, v;
        if (aprim_hit(q, O, D, t, u, v) && t < best && t > 1e-6f) { best = t; bu = u; bv = v; hit = i; }
    }
    return hit;
}

__device__ __forceinline__ bool analytic_any(const APrim* sp, int nsm, const TfgPrimitiva* gp, int n, V3 O, V3 D,
                                             float dist) {
    for (int i = 0; i < n; ++i) {
        APrim q;
        if (i < nsm) q = sp[i];
        else aprim_load(gp[i], q);
        float t, u, v;
        if (aprim_hit(q, O, D, t, u, v) && t > 1e-6f && t < dist) return true;
    }
    return false;
}

__device__ __forceinline__ int load_aprims_smem(APrim* sp, const TfgPrimitiva* gp, int n) {
    const int nsm = min(n, kSmemPrims);
    for (int i = threadIdx.x; i < nsm; i += blockDim.x) aprim_load(gp[i], sp[i]);
    __syncthreads();
    return nsm;
}

// ------------------------------------------------------------------ generate
// render.h:424-447: seed, jitter draws, training / unbiased draws, camera ray.
__device__ __forceinline__ int use_inf_of(const PassArgs& a) { return a.use_inf; }
__device__ __forceinline__ int use_inf_of(const SceneDesc& d) { return d.use_inf; }

template <bool MS>
__device__ __forceinline__ const CachePolicy& policy_of(const PassArgs& a, const TableOf<MS>& tab, uint32_t sc) {
    if constexpr (MS) return tab.s[sc].pol;
    else { (void)tab; (void)sc; return a.pol; }
}

// Whether the gate lets a path use the cache at P (always without a gate).
__device__ __forceinline__ bool gate_open(const CachePolicy& c, V3 P) {
    if (!c.gate_bits) return true;
    const uint32_t cell = gate_cell(c.gate_lo, c.gate_inv, P.x, P.y, P.z);
    return (__ldg(&c.gate_bits[cell >> 5]) >> (cell & 31u)) & 1u;
}

template <bool MS>
__global__ void k_generate(PassArgs a, TableOf<MS> tab) {
    const uint32_t N = a.npix;
    TfgCamara cam;
    int use_inf = 0;
    if constexpr (!MS) { cam = *a.cam; use_inf = use_inf_of(a); }
    const int frame0 = a.frame + a.s0 + (a.frame_dev ? *a.frame_dev : 0);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.nq; p += gridDim.x * blockDim.x) {
        const uint32_t q = a.p0 + p, s = q / N;
        uint32_t pix = q - s * N, sc = 0;
        int W = a.W, H = a.H;
        if constexpr (MS) {
            sc = scene_of_pixel(tab, pix);
            const SceneDesc& d = tab.s[sc];
            pix -= d.pix0;
            W = d.W; H = d.H;
            cam = *d.cam;
            use_inf = use_inf_of(d);
        }
        pix = tiled_pixel(pix, (uint32_t)W, (uint32_t)H);
        const int x = (int)(pix % (uint32_t)W), y = (int)(pix / (uint32_t)W);
        uint32_t rng = seed_pixel(x, y, frame0 + (int)s);
        const float ox = pcg_uniform(rng);
        const float oy = pcg_uniform(rng);
        V3 O, D;
        camera_ray(cam, x, y, W, H, ox, oy, O, D);
        uint32_t flags = 0;
        if (a.train) {
            const CachePolicy& pol = policy_of<MS>(a, tab, sc);
            // Gated passes draw the training decisions from a stream of their
            // own, so the path's stream stays that of a plain pass.
            uint32_t side = seed_pixel(x, y, frame0 + (int)s) ^ 0x9E3779B9u;
            uint32_t& r = pol.gate_bits ? side : rng;
            const bool training = use_inf ? (pcg_uniform(r) < pol.train_fraction) : true;
            if (training) {
                flags |= F_TRAIN;
                if (pcg_uniform(r) < 0.0625f) flags |= F_UNBIASED;
            }
        }
        a.ws.ray[0][2 * p + 0] = make_float4(O.x, O.y, O.z, MS ? __uint_as_float(sc) : 1e9f);
        a.ws.ray[0][2 * p + 1] = make_float4(D.x, D.y, D.z, __uint_as_float(p));
        a.ws.thr[p] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        a.ws.st[p] = make_uint4(rng, flags, __float_as_uint(1.0f), pix);   // w: the path's pixel in its image
        a.ws.lpre[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (a.use_inf || a.train) {
            a.ws.lsuf[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            a.ws.nrc[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ws.counters[0] = a.nq;
}

// ------------------------------------------------------------------ trace
template <int TRI_FMT, bool STATS, bool MS>
__global__ void __launch_bounds__(256) k_trace(PassArgs a, int bounce, TableOf<MS> tab) {
    extern __shared__ unsigned char smem_raw[];
    uint2* sstack = reinterpret_cast<uint2*>(smem_raw);
    APrim* sprims = reinterpret_cast<APrim*>(smem_raw + sizeof(uint2) * kSmemStack * blockDim.x);
    // one scene: its analytic primitives are cached in shared memory
    const int nsm = MS ? 0 : load_aprims_smem(sprims, a.prims, a.nprims);
    Geo g = geo_of<MS>(a, tab, 0);
    TravStack st;
    st.smem = sstack; st.stride = blockDim.x; st.tid = threadIdx.x;
    const float4* rays = a.ws.ray[bounce & 1];
    const uint32_t n = a.ws.counters[4 * bounce + 0];
    uint32_t* fetch = &a.ws.counters[4 * bounce + 1];
    TravCounts cnt;
    uint32_t nrays = 0;
    // Persistent lanes: a lane whose ray is done takes a new one as soon as
    // a.refill_min lanes of its warp are idle, instead of waiting for the
    // slowest ray of a 32-ray batch.
    const uint32_t lane = lane_id(), lt = (1u << lane) - 1u;
    const int refill = bounce == 0 ? a.refill_primary : a.refill_min;
    CwbvhRay<TRI_FMT, false> r;
    uint32_t csc = 0;   // a batch: the current ray's scene, whose tree is looked up again at every step
    uint32_t cur = kMissId, bid = kMissId;
    float best = 0.0f, bu = 0.0f, bv = 0.0f;
    bool exhausted = false;
    while (true) {
        const bool idle = cur == kMissId;
        const uint32_t im = __ballot_sync(0xFFFFFFFFu, idle);
        if (exhausted) {
            if (im == 0xFFFFFFFFu) break;
        } else if (__popc(im) >= refill) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(fetch, (uint32_t)__popc(im));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            exhausted = base + (uint32_t)__popc(im) >= n;
            const uint32_t k = base + (uint32_t)__popc(im & lt);
            if (idle && k < n) {
                cur = k;
                const float4 o4 = rays[2 * k], d4 = rays[2 * k + 1];
                const V3 O = xyz(o4), D = xyz(d4);
                if constexpr (MS) { csc = __float_as_uint(o4.w); g = geo_of<MS>(a, tab, csc); best = 1e9f; }
                else best = o4.w;
                bu = 0.0f; bv = 0.0f; bid = kMissId;
                const int ai = analytic_closest(sprims, nsm, g.prims, g.nprims, O, D, best, bu, bv);
                if (ai >= 0) bid = kAnalyticBit | (uint32_t)ai;
                r.init(O, D, 0.0f, best);
            }
        }
        if constexpr (MS) {
            if (cur != kMissId) g = geo_of<MS>(a, tab, csc);
        }
        if (cur != kMissId && !(g.has_bvh && r.step(g.nodes, g.tris, st))) {
            if (g.has_bvh) {
                if (r.found && r.tmax < best && r.tmax > kEps) { best = r.tmax; bu = r.hu; bv = r.hv; bid = r.id; }
                if (STATS) { cnt.nodes += r.nsteps; cnt.tris += r.ntris; }
            }
            a.ws.hit[cur] = make_float4(best, bu, bv, __uint_as_float(bid));
            ++nrays;
            cur = kMissId;
        }
    }
    if (STATS) flush_work(0, nrays, cnt);
}

// ------------------------------------------------------------------ shade
__device__ __forceinline__ void put_geo(float4* dst, V3 P, V3 dir, V3 n, V3 kd, V3 ks) {
    dst[0] = make_float4(P.x, P.y, P.z, dir.x);
    dst[1] = make_float4(dir.y, dir.z, n.x, n.y);
    dst[2] = make_float4(n.z, kd.x, kd.y, kd.z);
    dst[3] = make_float4(ks.x, ks.y, ks.z, 0.0f);
}

__device__ __forceinline__ V3 map01(V3 d) { return v3(d.x * 0.5f + 0.5f, d.y * 0.5f + 0.5f, d.z * 0.5f + 0.5f); }

__device__ __forceinline__ void write_datos(TfgDatosMLP* d, V3 P, V3 dir, V3 n, V3 kd, V3 ks) {
    TfgDatosMLP r;
    r.posicion.x = P.x; r.posicion.y = P.y; r.posicion.z = P.z;
    r.direccion.x = dir.x; r.direccion.y = dir.y; r.direccion.z = dir.z;
    r.normal.x = n.x; r.normal.y = n.y; r.normal.z = n.z;
    r.difuso.r = kd.x; r.difuso.g = kd.y; r.difuso.b = kd.z;
    r.especular.r = ks.x; r.especular.g = ks.y; r.especular.b = ks.z;
    r.color.r = 0.0f; r.color.g = 0.0f; r.color.b = 0.0f;
    *d = r;
}

template <bool MS>
__global__ void __launch_bounds__(256) k_shade(PassArgs a, int bounce, TableOf<MS> tab) {
    const uint32_t n = a.ws.counters[4 * bounce + 0];
    const float4* rays = a.ws.ray[bounce & 1];
    float4* next = a.ws.ray[(bounce + 1) & 1];
    uint32_t* next_count = &a.ws.counters[4 * (bounce + 1) + 0];
    uint32_t* shadow_count = &a.ws.counters[4 * bounce + 2];
    const bool nrc = a.use_inf || a.train;
    const int use_inf_single = MS ? 0 : use_inf_of(a);
    const uint32_t stride = gridDim.x * blockDim.x;
    // Uniform trip count so that every lane of a warp reaches the warp-wide appends.
    const uint32_t n_round = (n + stride - 1) / stride * stride;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += stride) {
        bool live = i < n, want_shadow = false, survive = false;
        float4 sh0, sh1, sh2, sh3, nr0, nr1;
        uint32_t p = 0;
        if (live) {
            const float4 o4 = rays[2 * i], d4 = rays[2 * i + 1], h = a.ws.hit[i];
            p = __float_as_uint(d4.w);
            const uint32_t sc = MS ? __float_as_uint(o4.w) : 0u;
            const Geo g = geo_of<MS>(a, tab, sc);
            int use_inf = use_inf_single;
            if constexpr (MS) use_inf = use_inf_of(tab.s[sc]);
            const CachePolicy& pol = policy_of<MS>(a, tab, sc);
            V3 O = xyz(o4), D = xyz(d4);
            float4 thr4 = a.ws.thr[p];
            uint4 st = a.ws.st[p];
            V3 cam = xyz(thr4);
            float ior = thr4.w;
            uint32_t rng = st.x, flags = st.y;
            float pdf_last = __uint_as_float(st.z);
            const uint32_t id = __float_as_uint(h.w);
            float4 lpre = a.ws.lpre[p];
            float4 lsuf = make_float4(0, 0, 0, 0), nrc4 = make_float4(0, 0, 0, 0);
            if (nrc) { lsuf = a.ws.lsuf[p]; nrc4 = a.ws.nrc[p]; }
            bool end = false;
            if (id == kMissId) {
                end = true;   // background is black (render.h:227-239)
            } else {
                const TfgPrimitiva* pr = prim_of(g, id);
                const float t = h.x;
                const V3 P = O + D * t;
                const V3 nrm = surface_normal(pr, P, h.y, h.z);
                const V3 view = -D;
                const float cos_t = fabsf(dot(nrm, -D));
                const Material m = load_material(pr);
                const bool es_dif = cmax(m.difuso) > kEps;
                const bool es_esp = cmax(m.especular) > kEps;
                const bool captured = (flags & F_CAPTURED) != 0;
                bool foot_ok = false;
                if (nrc) {
                    // Footprint heuristic, render.h:86-102.
                    const float dist_sq = t * t;
                    if (bounce == 0) {
                        lpre.w = dist_sq / (4.0f * kPiF * fmaxf(cos_t, 1e-4f));
                        lsuf.w = 0.0f;
                    } else {
                        const float spread = dist_sq / (fmaxf(pdf_last, 1e-4f) * fmaxf(cos_t, 1e-4f));
                        if (!captured) lsuf.w += spread;
                        else nrc4.x += spread;
                    }
                    foot_ok = lsuf.w >= lpre.w * pol.footprint;
                }
                if (cmax(m.emision) > 0.0f) {
                    // Emission ends the path (render.h:104-123).
                    const V3 c = mul(cam, m.emision);
                    if (captured) {
                        lsuf.x += c.x; lsuf.y += c.y; lsuf.z += c.z;
                        if (flags & F_FULL) { lpre.x += c.x; lpre.y += c.y; lpre.z += c.z; }
                        put_geo(&a.ws.ts[10 * (size_t)p + 4], P, normalized(-D), nrm, v3(0, 0, 0), v3(0, 0, 0));
                        a.ws.ts[10 * (size_t)p + 9] = make_float4(0, 0, 0, 0);
                        flags |= F_TAIL;
                    } else {
                        lpre.x += c.x; lpre.y += c.y; lpre.z += c.z;
                    }
                    end = true;
                } else {
                    if (es_dif) {
                        // Next-event estimation is deferred to the shadow stage (render.h:126-131).
                        const V3 ps = P + nrm * kEps;
                        want_shadow = true;
                        sh0 = make_float4(ps.x, ps.y, ps.z, __uint_as_float(p));
                        // bit 0: the suffix's radiance; bit 1: the pixel's as well (F_FULL)
                        sh1 = make_float4(nrm.x, nrm.y, nrm.z,
                                          __uint_as_float(captured ? ((flags & F_FULL) ? 3u : 1u) : 0u));
                        sh2 = make_float4(m.difuso.x, m.difuso.y, m.difuso.z, MS ? __uint_as_float(sc) : 0.0f);
                        sh3 = make_float4(cam.x, cam.y, cam.z, 0.0f);
                    }
                    if (captured) {
                        // Suffix bootstrap termination (render.h:134-163).
                        const bool stop = !(flags & (F_UNBIASED | F_FULL)) && (nrc4.x >= nrc4.y) && gate_open(pol, P);
                        if (stop) {
                            put_geo(&a.ws.ts[10 * (size_t)p + 4], P, map01(view), map01(nrm), m.difuso, m.especular);
                            const V3 refl = m.difuso + m.especular + m.transmision;
                            const V3 ts = mul(cam, refl);
                            a.ws.ts[10 * (size_t)p + 9] = make_float4(ts.x, ts.y, ts.z, 0.0f);
                            flags |= F_TAIL;
                            end = true;
                        }
                    }
                    if (!end && es_dif && !es_esp && foot_ok) {
                        // Cache query / training head capture (render.h:166-202).
                        V3 refl = m.difuso + m.especular + m.transmision;
                        refl = v3(fmaxf(refl.x, 1e-3f), fmaxf(refl.y, 1e-3f), fmaxf(refl.z, 1e-3f));
                        const bool training = (flags & F_TRAIN) != 0;
                        if (!training && use_inf && gate_open(pol, P)) {
                            const Outs o = outs_of<MS>(a, tab, sc);
                            const uint32_t px = st.w;
                            write_datos(&o.infer[px], P, map01(view), map01(nrm), m.difuso, m.especular);
                            const V3 tt = mul(cam, refl);
                            o.thr_out[px] = TfgColor{tt.x, tt.y, tt.z};
                            flags |= F_INF;
                            end = true;
                        } else if (training && !captured) {
                            put_geo(&a.ws.ts[10 * (size_t)p + 0], P, map01(view), map01(nrm), m.difuso, m.especular);
                            const V3 tt = mul(cam, refl);
                            a.ws.ts[10 * (size_t)p + 8] = make_float4(tt.x, tt.y, tt.z, 0.0f);
                            nrc4.y = lsuf.w;   // a_prefix = a_current
                            flags |= F_CAPTURED;
                            if (!gate_open(pol, P)) flags |= F_FULL;
                            // This bounce's NEE still belongs to the prefix: sh1.w stays 0.
                        }
                    }
                    if (!end) {
                        // BSDF sampling, render.h:264-335.
                        const float mkd = cmax(m.difuso), mks = cmax(m.especular), mkt = cmax(m.transmision);
                        const float sum = mkd + mks + mkt;
                        if (sum <= 0.0f) {
                            cam = v3(0.0f, 0.0f, 0.0f);
                        } else {
                            const float pd = mkd / sum, ps = mks / sum, pt = 1.0f - pd - ps;
                            const float r = pcg_uniform(rng);
                            if (r < pd) {
                                cam = div_or_black(mul(cam, m.difuso), pd);
                                const float r1 = pcg_uniform(rng);
                                const float r2 = pcg_uniform(rng);
                                const float phi = 2.0f * kPiF * r1;
                                const float z = sqrtf(1.0f - r2);
                                if (z > kEps) {
                                    const float s = sqrtf(r2);
                                    float sp, cp;
                                    sincosf(phi, &sp, &cp);
                                    const V3 wi = to_world(v3(s * cp, s * sp, z), nrm);
                                    O = P + wi * kEps;
                                    D = normalized(wi);
                                    float c = fabsf(dot(wi, nrm));
                                    if (c < 1e-4f) c = 1e-4f;
                                    pdf_last = c / kPiF;
                                }
                            } else if (r < pd + ps) {
                                const V3 wr = reflect_dir(D, nrm);
                                cam = div_or_black(mul(cam, m.especular), ps);
                                O = P + wr * kEps;
                                D = normalized(wr);
                                pdf_last = 1e6f;
                            } else {
                                const V3 wt = refract_dir(D, nrm, m.ior, ior);
                                cam = div_or_black(mul(cam, m.transmision), pt);
                                O = P + wt * kEps;
                                D = normalized(wt);
                                pdf_last = 1e6f;
                            }
                        }
                        // Russian roulette, render.h:209-224.
                        if (bounce >= a.rr_min_depth) {
                            float prob = fmaxf(cam.x, fmaxf(cam.y, cam.z));
                            if (prob > 0.95f) prob = 0.95f;
                            if (pcg_uniform(rng) > prob) end = true;
                            else cam = div_or_black(cam, prob);
                        }
                        if (!end && bounce + 1 < a.max_depth) survive = true;
                    }
                }
            }
            a.ws.thr[p] = make_float4(cam.x, cam.y, cam.z, ior);
            a.ws.st[p] = make_uint4(rng, flags, __float_as_uint(pdf_last), st.w);
            a.ws.lpre[p] = lpre;
            if (nrc) { a.ws.lsuf[p] = lsuf; a.ws.nrc[p] = nrc4; }
            nr0 = make_float4(O.x, O.y, O.z, MS ? __uint_as_float(sc) : 1e9f);
            nr1 = make_float4(D.x, D.y, D.z, __uint_as_float(p));
        }
        const uint32_t slot = warp_append(next_count, survive);
        if (survive) { next[2 * slot] = nr0; next[2 * slot + 1] = nr1; }
        const uint32_t sslot = warp_append(shadow_count, want_shadow);
        if (want_shadow) {
            float4* s = &a.ws.shadow[4 * (size_t)sslot];
            s[0] = sh0; s[1] = sh1; s[2] = sh2; s[3] = sh3;
        }
    }
}

// ------------------------------------------------------------------ shadow
// escenario.h:144-184: every light in order, Lambert BRDF kd/pi, inverse-square
// falloff with the distance clamped to >= 1, summed then scaled by the path
// throughput (render.h:128-130).

__device__ __forceinline__ float dot_rn(V3 a, V3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}

// One light of a shading point: the shadow ray (origin nudged off the
// surface, unit direction, length) and the term the light adds when nothing
// occludes it, I / max(d, 1)^2 * kd / pi * cos.  False when the light is
// behind the surface.  Every operation is rounded on its own, so all shadow
// kernels compute the same rays and terms whatever the compiler fuses around
// them.
struct LightRay {
    V3 so, dl, term;
    float dist;
};
__device__ __forceinline__ bool light_ray(const TfgLuzPuntual& lz, V3 P, V3 N, V3 kd, LightRay& s) {
    const V3 lp = ld3(lz.posicion);
    V3 dl = v3(__fsub_rn(lp.x, P.x), __fsub_rn(lp.y, P.y), __fsub_rn(lp.z, P.z));
    const float dist = __fsqrt_rn(dot_rn(dl, dl));
    if (dist > 0.0f) {
        const float inv = __fdiv_rn(1.0f, dist);
        dl = v3(__fmul_rn(dl.x, inv), __fmul_rn(dl.y, inv), __fmul_rn(dl.z, inv));
    }
    const float c = dot_rn(N, dl);
    if (!(c > 0.0f)) return false;
    s.so = v3(__fadd_rn(P.x, __fmul_rn(dl.x, kEps)), __fadd_rn(P.y, __fmul_rn(dl.y, kEps)),
              __fadd_rn(P.z, __fmul_rn(dl.z, kEps)));
    s.dl = dl;
    s.dist = dist;
    const float dd = fmaxf(dist, 1.0f), d2 = __fmul_rn(dd, dd);
    s.term = v3(__fmul_rn(__fmul_rn(__fdiv_rn(lz.intensidad.r, d2), __fdiv_rn(kd.x, kPiF)), c),
                __fmul_rn(__fmul_rn(__fdiv_rn(lz.intensidad.g, d2), __fdiv_rn(kd.y, kPiF)), c),
                __fmul_rn(__fmul_rn(__fdiv_rn(lz.intensidad.b, d2), __fdiv_rn(kd.z, kPiF)), c));
    return true;
}

// The shading point's radiance (throughput x light sum) into the path's
// prefix and / or suffix radiance (dest bit 0: suffix; not 1: prefix too).
__device__ __forceinline__ void add_direct(const PassArgs& a, uint32_t p, uint32_t dest, V3 cam, V3 L) {
    const V3 add = mul(cam, L);
    if (dest & 1u) {
        float4 v = a.ws.lsuf[p];
        v.x += add.x; v.y += add.y; v.z += add.z;
        a.ws.lsuf[p] = v;
    }
    if (dest != 1u) {
        float4 v = a.ws.lpre[p];
        v.x += add.x; v.y += add.y; v.z += add.z;
        a.ws.lpre[p] = v;
    }
}

// A 16-byte load that the compiler keeps where it is written (not hoisted out
// of a loop and held in registers).
__device__ __forceinline__ float4 ld_item(const float4* p) {
    float4 v;
    asm volatile("ld.global.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
    return v;
}

template <int TRI_FMT, bool STATS, bool MS>
__global__ void __launch_bounds__(256) k_shadow(PassArgs a, int bounce, TableOf<MS> tab) {
    extern __shared__ unsigned char smem_raw[];
    uint2* sstack = reinterpret_cast<uint2*>(smem_raw);
    APrim* sprims = reinterpret_cast<APrim*>(smem_raw + sizeof(uint2) * kSmemStack * blockDim.x);
    const int nsm = MS ? 0 : load_aprims_smem(sprims, a.prims, a.nprims);
    TravStack stck;
    stck.smem = sstack; stck.stride = blockDim.x; stck.tid = threadIdx.x;
    const uint32_t n = a.ws.counters[4 * bounce + 2];
    uint32_t* fetch = &a.ws.counters[4 * bounce + 3];
    TravCounts cnt;
    uint32_t nrays = 0;
    // One shadow ray per lane: the lights of an item sit on G adjacent lanes
    // (G = light count rounded up to a power of two; more than 32 lights,
    // a.shadow_one_lane, or a batch of scenes with their own light counts give
    // one lane looping over them), and warps fetch items dynamically.
    const int nl = a.nlights;
    const uint32_t G = (MS || a.shadow_one_lane) ? 1u
                       : nl <= 1 ? 1u : nl <= 2 ? 2u : nl <= 4 ? 4u : nl <= 8 ? 8u : nl <= 16 ? 16u : nl <= 32 ? 32u : 1u;
    const uint32_t lane = lane_id(), lg = lane & (G - 1u), group0 = lane & ~(G - 1u);
    const int l_begin = G == 1u ? 0 : (int)lg;
    const int l_end = G == 1u ? nl : min(nl, (int)lg + 1);
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(fetch, 32u / G);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= n) break;
        const uint32_t i = base + lane / G;
        const bool have = i < n;
        V3 L = v3(0.0f, 0.0f, 0.0f);
        // The item (shading point, albedo, throughput, pixel, destination) is
        // read where it is used -- the point for every light, the rest after
        // the traversals -- so that none of it is held in registers through a
        // traversal (L1 serves the re-reads).
        const float4* s = &a.ws.shadow[4 * (size_t)(have ? i : 0u)];
        if (have) {
            for (int l = l_begin;; ++l) {
                // A batch's scene (its lights, primitives and tree) is looked
                // up again for every light from the item's scene index, for
                // the same reason.
                const uint32_t sc = MS ? __float_as_uint(ld_item(s + 2).w) : 0u;
                const Geo g = geo_of<MS>(a, tab, sc);
                const TfgLuzPuntual* lights = a.lights;
                int lend = l_end;
                if constexpr (MS) { lights = tab.s[sc].lights; lend = tab.s[sc].nlights; }
                if (l >= lend) break;
                LightRay lr;
                if (!light_ray(lights[l], xyz(ld_item(s)), xyz(ld_item(s + 1)), xyz(ld_item(s + 2)), lr)) continue;
                if (STATS) ++nrays;
                if (analytic_any(sprims, nsm, g.prims, g.nprims, lr.so, lr.dl, lr.dist)) continue;
                if (a.shadow_mesh && g.has_bvh) {
                    float tm = lr.dist, hu, hv;
                    uint32_t hid;
                    if (cwbvh_trace<TRI_FMT, true>(g.nodes, g.tris, lr.so, lr.dl, kEps, tm, hid, hu, hv, stck,
                                                   STATS ? &cnt : nullptr)) continue;
                }
                // Each light's term is rounded before it is added, so one lane
                // looping over the lights sums the same values in the same
                // order as the lanes of a group.
                L = v3(__fadd_rn(L.x, lr.term.x), __fadd_rn(L.y, lr.term.y), __fadd_rn(L.z, lr.term.z));
            }
        }
        // Sum the group's lights in light order on its first lane (an occluded
        // or back-facing light adds an exact zero), as the sequential loop does.
        for (uint32_t j = 1; j < G; ++j) {
            const float x = __shfl_sync(0xFFFFFFFFu, L.x, group0 + j);
            const float y = __shfl_sync(0xFFFFFFFFu, L.y, group0 + j);
            const float z = __shfl_sync(0xFFFFFFFFu, L.z, group0 + j);
            if (lg == 0u && (int)j < nl) L = L + v3(x, y, z);
        }
        if (have && lg == 0u) {
            const float4 s0 = ld_item(s), s1 = ld_item(s + 1), s3 = ld_item(s + 3);
            add_direct(a, __float_as_uint(s0.w), __float_as_uint(s1.w), xyz(s3), L);
        }
    }
    if (STATS) flush_work(3, nrays, cnt);
}

// ------------------------------------------------------------------ resolve
__device__ __forceinline__ void get_geo(const float4* src, TfgDatosGeometricos& g) {
    const float4 a0 = src[0], a1 = src[1], a2 = src[2], a3 = src[3];
    g.posicion.x = a0.x; g.posicion.y = a0.y; g.posicion.z = a0.z;
    g.direccion.x = a0.w; g.direccion.y = a1.x; g.direccion.z = a1.y;
    g.normal.x = a1.z; g.normal.y = a1.w; g.normal.z = a2.x;
    g.difuso = TfgColor{a2.y, a2.z, a2.w};
    g.especular = TfgColor{a3.x, a3.y, a3.z};
}

// One thread per pixel of the wavefront: slots j, j + npix, j + 2 npix ...
// hold that pixel's samples in order, so the accumulation adds them in sample
// order whatever the wavefront size.
template <bool MS>
__global__ void k_resolve(PassArgs a, TableOf<MS> tab) {
    const uint32_t N = a.npix;
    const bool nrc = a.use_inf || a.train;
    const uint32_t first = min(a.nq, N);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < first; j += gridDim.x * blockDim.x) {
        const uint32_t q = a.p0 + j, s_rel = q / N;
        uint32_t px = q - s_rel * N, sc = 0;
        uint32_t W = (uint32_t)a.W, H = (uint32_t)a.H;
        if constexpr (MS) { sc = scene_of_pixel(tab, px); px -= tab.s[sc].pix0; W = tab.s[sc].W; H = tab.s[sc].H; }
        px = tiled_pixel(px, W, H);
        const Outs o = outs_of<MS>(a, tab, sc);
        int sample = a.s0 + (int)s_rel;
        for (uint32_t p = j; p < a.nq; p += N, ++sample) {
            const float4 lp = a.ws.lpre[p];
            if (o.img && sample == a.last_sample) o.img[px] = TfgColor{lp.x, lp.y, lp.z};
            if (o.accum) {
                o.accum[3 * (size_t)px] += lp.x; o.accum[3 * (size_t)px + 1] += lp.y; o.accum[3 * (size_t)px + 2] += lp.z;
            }
            const uint32_t flags = a.ws.st[p].y;
            const bool rec = nrc && (flags & F_TRAIN) && (flags & F_CAPTURED);
            const bool head_query = rec && !(flags & F_FULL);
            if (o.thr_out && !(flags & F_INF) && !head_query) o.thr_out[px] = TfgColor{0.0f, 0.0f, 0.0f};
            if (!rec) continue;
            // Training path with a head vertex: its pixel keeps the prefix radiance and
            // asks the cache at the head (render.h:243-260); the record goes to the ring
            // (render.h:461-464).
            const float4* ts = &a.ws.ts[10 * (size_t)p];
            TfgDatosGeometricos head, tail;
            get_geo(ts, head);
            const float4 thr_train = ts[8];
            if (o.infer && head_query) {
                TfgDatosMLP d;
                d.posicion = head.posicion; d.direccion = head.direccion; d.normal = head.normal;
                d.difuso = head.difuso; d.especular = head.especular; d.color = TfgColor{0.0f, 0.0f, 0.0f};
                o.infer[px] = d;
            }
            if (o.thr_out && head_query) o.thr_out[px] = TfgColor{thr_train.x, thr_train.y, thr_train.z};
            if (o.reg_counter && o.regs && o.reg_cap > 0) {
                TfgRegistroEntrenamiento r;
                r.head = head;
                float4 thr_suf = make_float4(0, 0, 0, 0);
                if (flags & F_TAIL) { get_geo(ts + 4, tail); thr_suf = ts[9]; }
                else { memset(&tail, 0, sizeof(tail)); }
                r.tail = tail;
                const float4 ls = a.ws.lsuf[p];
                r.luz_acumulada_sufijo = TfgColor{ls.x, ls.y, ls.z};
                r.throughput_sufijo = TfgColor{thr_suf.x, thr_suf.y, thr_suf.z};
                r.factor_normalizacion = TfgColor{thr_train.x, thr_train.y, thr_train.z};
                r.valido = 1;
                const uint32_t idx = atomicAdd(o.reg_counter, 1u);
                o.regs[idx % (uint32_t)o.reg_cap] = r;
            }
        }
    }
}

// ------------------------------------------------------------------ host side
namespace {

// Queues and per-path state, one set per (device, slot): passes that may run
// concurrently (the branches of a batched multi-scene frame) use different
// slots; everything else uses slot 0.
std::mutex g_ws_mutex;
Workspace g_ws[kMaxDevices][kWorkspaceSlots];

int ensure_workspace(int dev, int slot, size_t paths, bool nrc, Workspace& out) {
    if (slot < 0 || slot >= kWorkspaceSlots) return fail(TFG_E_INVALID, "render: workspace slot out of range");
    std::lock_guard<std::mutex> lk(g_ws_mutex);
    Workspace& w = g_ws[dev][slot];
    auto grow = [](void** p, size_t bytes) -> cudaError_t {
        if (*p) cudaFree(*p);
        *p = nullptr;
        return cudaMalloc(p, bytes);
    };
    cudaError_t e = cudaSuccess;
    if (w.cap < paths) {
        size_t cap = paths;
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) e = grow((void**)&w.ray[k], cap * 2 * sizeof(float4));
        if (e == cudaSuccess) e = grow((void**)&w.hit, cap * sizeof(float4));
        if (e == cudaSuccess) e = grow((void**)&w.shadow, cap * 4 * sizeof(float4));
        if (e == cudaSuccess) e = grow((void**)&w.thr, cap * sizeof(float4));
        if (e == cudaSuccess) e = grow((void**)&w.st, cap * sizeof(uint4));
        if (e == cudaSuccess) e = grow((void**)&w.lpre, cap * sizeof(float4));
        if (e == cudaSuccess) e = grow((void**)&w.lsuf, cap * sizeof(float4));
        if (e == cudaSuccess) e = grow((void**)&w.nrc, cap * sizeof(float4));
        if (e == cudaSuccess && !w.counters) e = cudaMalloc((void**)&w.counters, 4 * (kMaxBounces + 1) * sizeof(uint32_t));
        ++w.generation;
        if (e != cudaSuccess) { w.cap = 0; return fail((int)e, std::string("render workspace: ") + cudaGetErrorString(e)); }
        w.cap = cap;
    }
    if (!w.side) {
        e = cudaStreamCreateWithFlags(&w.side, cudaStreamNonBlocking);
        for (int b = 0; b < kMaxBounces && e == cudaSuccess; ++b) {
            e = cudaEventCreateWithFlags(&w.fork[b], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.join[b], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) { w.side = nullptr; return fail((int)e, std::string("render streams: ") + cudaGetErrorString(e)); }
    }
    if (nrc && w.train_cap < paths) {
        e = grow((void**)&w.ts, paths * 10 * sizeof(float4));
        ++w.generation;
        if (e != cudaSuccess) { w.train_cap = 0; return fail((int)e, std::string("training scratch: ") + cudaGetErrorString(e)); }
        w.train_cap = paths;
    }
    out = w;
    return 0;
}

// Launch tuning of each device (tfgRenderTuningSet / tfgRenderAutotune).
// Every setting computes the same image; the generation number changes with
// every set, so captured frame graphs know when to re-capture.
std::mutex g_tune_mutex;
TfgRenderTuning g_tune[kMaxDevices];
bool g_tune_valid[kMaxDevices] = {false};
uint32_t g_tune_generation = 1;

constexpr int kThreadChoices[3] = {64, 128, 256};
int threads_index(int t) { return t == 64 ? 0 : t == 256 ? 2 : 1; }

}  // namespace

uint32_t workspace_generation(int dev, int slot) {
    std::lock_guard<std::mutex> lk(g_ws_mutex);
    return g_ws[dev][slot & (kWorkspaceSlots - 1)].generation;
}

namespace {

struct LaunchShapes {
    int sms = 0;
    // resident CTAs per SM: [one scene / batch][triangle format][64, 128, 256 threads]
    int trace_occ[2][2][3] = {};
    int shadow_occ[2][2][3] = {};
    int shade_blocks[2] = {0, 0};
};
LaunchShapes g_shapes[kMaxDevices];
std::mutex g_shapes_mutex;   // first calls on several host threads fill a device's entry once

size_t trace_smem(int nprims, int threads) {
    return sizeof(uint2) * kSmemStack * (size_t)threads + sizeof(APrim) * (size_t)std::min(nprims, kSmemPrims);
}

int shapes_for(int dev, LaunchShapes& s) {
    std::lock_guard<std::mutex> lk(g_shapes_mutex);
    LaunchShapes& g = g_shapes[dev];
    if (g.sms == 0) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        auto occ_of = [](auto kernel, int bt, size_t sm) {
            int occ = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, bt, sm);
            return std::max(occ, 1);
        };
        for (int k = 0; k < 3; ++k) {
            const int bt = kThreadChoices[k];
            const size_t sm = trace_smem(kSmemPrims, bt), sm_ms = trace_smem(0, bt);
            g.trace_occ[0][0][k] = occ_of(k_trace<0, false, false>, bt, sm);
            g.trace_occ[0][1][k] = occ_of(k_trace<1, false, false>, bt, sm);
            g.shadow_occ[0][0][k] = occ_of(k_shadow<0, false, false>, bt, sm);
            g.shadow_occ[0][1][k] = occ_of(k_shadow<1, false, false>, bt, sm);
            g.trace_occ[1][0][k] = occ_of(k_trace<0, false, true>, bt, sm_ms);
            g.trace_occ[1][1][k] = occ_of(k_trace<1, false, true>, bt, sm_ms);
            g.shadow_occ[1][0][k] = occ_of(k_shadow<0, false, true>, bt, sm_ms);
            g.shadow_occ[1][1][k] = occ_of(k_shadow<1, false, true>, bt, sm_ms);
        }
        g.shade_blocks[0] = sms * occ_of(k_shade<false>, 256, 0);
        g.shade_blocks[1] = sms * occ_of(k_shade<true>, 256, 0);
        g.sms = sms;
    }
    s = g;
    return 0;
}

// A device's tuning resolved for one call: the wavefront in paths, capped by
// the call's path count (and by one sample of the image for cache passes,
// whose per-pixel outputs take one sample per pixel at a time).
struct Tuning {
    uint32_t wavefront = 0;
    int threads = 128, warps_per_sm = 0, refill = 8, refill_primary = 8, shadow_one_lane = 0, overlap_shadow = 0;
};

Tuning resolve_tuning(int dev, uint32_t npix, int spp, bool nrc, uint32_t* generation) {
    TfgRenderTuning t;
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        if (g_tune_valid[dev]) t = g_tune[dev];
        else tfgRenderTuningDefault(&t);
        if (generation) *generation = g_tune_generation;
    }
    Tuning r;
    uint64_t wf = t.wavefront_paths > 0 ? (uint64_t)t.wavefront_paths : npix;
    if (nrc) wf = std::min<uint64_t>(wf, npix);
    wf = std::min<uint64_t>(wf, (uint64_t)spp * npix);
    r.wavefront = (uint32_t)std::max<uint64_t>(wf, 1);
    r.threads = t.trace_threads;
    r.warps_per_sm = t.trace_warps_per_sm;
    r.refill = t.refill_min;
    r.refill_primary = t.refill_min_primary > 0 ? t.refill_min_primary : t.refill_min;
    r.shadow_one_lane = t.shadow_one_lane;
    r.overlap_shadow = t.overlap_shadow;
    return r;
}

// Persistent traversal grid: every SM holds as many CTAs as fit, or the
// tuned number of warps.
int persistent_grid(const LaunchShapes& sh, int occ, const Tuning& t) {
    int per_sm = occ;
    if (t.warps_per_sm > 0) per_sm = std::max(1, std::min(occ, t.warps_per_sm * 32 / t.threads));
    return sh.sms * per_sm;
}

}  // namespace

int render_tuning_check(const TfgRenderTuning& t) {
    if (t.wavefront_paths != 0 && (t.wavefront_paths < 1024 || t.wavefront_paths > (1 << 26)))
        return fail(TFG_E_INVALID, "render tuning: wavefront_paths must be 0 or in [1024, 2^26]");
    if (t.trace_threads != 64 && t.trace_threads != 128 && t.trace_threads != 256)
        return fail(TFG_E_INVALID, "render tuning: trace_threads must be 64, 128 or 256");
    if (t.trace_warps_per_sm < 0 || t.trace_warps_per_sm > 64)
        return fail(TFG_E_INVALID, "render tuning: trace_warps_per_sm must be in [0, 64]");
    if (t.refill_min < 1 || t.refill_min > 32) return fail(TFG_E_INVALID, "render tuning: refill_min must be in [1, 32]");
    if (t.shadow_one_lane != 0 && t.shadow_one_lane != 1)
        return fail(TFG_E_INVALID, "render tuning: shadow_one_lane must be 0 or 1");
    if (t.refill_min_primary < 0 || t.refill_min_primary > 32)
        return fail(TFG_E_INVALID, "render tuning: refill_min_primary must be in [0, 32]");
    if (t.overlap_shadow != 0 && t.overlap_shadow != 1)
        return fail(TFG_E_INVALID, "render tuning: overlap_shadow must be 0 or 1");
    return ok();
}

int render_tuning_set(int dev, const TfgRenderTuning& t) {
    if (int rc = render_tuning_check(t)) return rc;
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tune[dev] = t;
    g_tune_valid[dev] = true;
    ++g_tune_generation;
    return ok();
}

int render_tuning_get(int dev, TfgRenderTuning* out, uint32_t* generation) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    if (out) {
        if (g_tune_valid[dev]) *out = g_tune[dev];
        else tfgRenderTuningDefault(out);
    }
    if (generation) *generation = g_tune_generation;
    return ok();
}

namespace {

// Stage timing with CUDA events (TFG_PROFILE_TIMES): one start/stop pair per
// launch, summed by tfgRenderProfileGet.
struct StageEvents {
    cudaEvent_t start, stop;
    int stage;
};
std::mutex g_prof_mutex;
std::vector<StageEvents> g_prof_events;
size_t g_prof_used = 0;
double g_prof_ms[5] = {0, 0, 0, 0, 0};
uint64_t g_prof_launches[5] = {0, 0, 0, 0, 0};

StageEvents profiler_pair(int stage) {
    std::lock_guard<std::mutex> lk(g_prof_mutex);
    if (g_prof_used == g_prof_events.size()) {
        StageEvents ev{};
        cudaEventCreate(&ev.start);
        cudaEventCreate(&ev.stop);
        g_prof_events.push_back(ev);
    }
    StageEvents& ev = g_prof_events[g_prof_used++];
    ev.stage = stage;
    return ev;
}

}  // namespace

int profile_reset() {
    std::lock_guard<std::mutex> lk(g_prof_mutex);
    g_prof_used = 0;
    for (int i = 0; i < 5; ++i) { g_prof_ms[i] = 0.0; g_prof_launches[i] = 0; }
    unsigned long long zero[6] = {0, 0, 0, 0, 0, 0};
    cudaError_t e = cudaMemcpyToSymbol(g_work, zero, sizeof(zero));
    if (e != cudaSuccess) return fail((int)e, std::string("profile reset: ") + cudaGetErrorString(e));
    return ok();
}

int profile_get(TfgRenderProfile* out) {
    if (!out) return fail(TFG_E_INVALID, "tfgRenderProfileGet: out is null");
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail((int)e, std::string("profile get: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lk(g_prof_mutex);
    for (size_t i = 0; i < g_prof_used; ++i) {
        float ms = 0.0f;
        e = cudaEventElapsedTime(&ms, g_prof_events[i].start, g_prof_events[i].stop);
        if (e != cudaSuccess) return fail((int)e, std::string("profile events: ") + cudaGetErrorString(e));
        g_prof_ms[g_prof_events[i].stage] += ms;
        g_prof_launches[g_prof_events[i].stage] += 1;
    }
    g_prof_used = 0;
    unsigned long long w[6];
    e = cudaMemcpyFromSymbol(w, g_work, sizeof(w));
    if (e != cudaSuccess) return fail((int)e, std::string("profile counters: ") + cudaGetErrorString(e));
    for (int i = 0; i < 5; ++i) { out->ms[i] = g_prof_ms[i]; out->launches[i] = g_prof_launches[i]; }
    out->rays = w[0]; out->nodes = w[1]; out->tri_tests = w[2];
    out->shadow_rays = w[3]; out->shadow_nodes = w[4]; out->shadow_tri_tests = w[5];
    return ok();
}

template <bool MS>
int enqueue_pass(PassArgs a, const TableOf<MS>& tab, const TfgRenderParams& prm, int frame, TfgColor* img,
                 const LaunchShapes& sh, const Tuning& tu, cudaStream_t stream);

int render_pass(const TfgRenderParams& prm, const TfgCamara* d_cam, const TfgPrimitiva* prims, int nprims,
                const TfgLuzPuntual* lights, int nlights, int W, int H, int frame, const TfgTinyBVHD_GPU* bvh,
                const float* tris_wt, const TfgPrimitiva* mesh, int nmesh, TfgColor* img, float* accum,
                TfgRegistroEntrenamiento* regs, uint32_t* reg_counter, int reg_cap, TfgDatosMLP* infer,
                TfgColor* thr_out, int use_inf, int train, cudaStream_t stream) {
    return render_pass_ex(prm, d_cam, prims, nprims, lights, nlights, W, H, frame, nullptr, nullptr, bvh, tris_wt,
                          mesh, nmesh, img, accum, regs, reg_counter, reg_cap, infer, thr_out, use_inf, train, false,
                          0, stream);
}

int render_pass_ex(const TfgRenderParams& prm, const TfgCamara* d_cam, const TfgPrimitiva* prims, int nprims,
                   const TfgLuzPuntual* lights, int nlights, int W, int H, int frame, const int32_t* frame_dev,
                   const CachePolicy* policy, const TfgTinyBVHD_GPU* bvh, const float* tris_wt,
                   const TfgPrimitiva* mesh, int nmesh, TfgColor* img, float* accum, TfgRegistroEntrenamiento* regs,
                   uint32_t* reg_counter, int reg_cap, TfgDatosMLP* infer, TfgColor* thr_out, int use_inf, int train,
                   bool prepare_only, int ws_slot, cudaStream_t stream) {
    if (W <= 0 || H <= 0 || (size_t)W * (size_t)H > (1u << 28)) return fail(TFG_E_INVALID, "render: bad image size");
    if (!d_cam) return fail(TFG_E_INVALID, "render: camara is null");
    if (nprims < 0 || nlights < 0 || nmesh < 0) return fail(TFG_E_INVALID, "render: negative count");
    if ((nprims > 0 && !prims) || (nlights > 0 && !lights)) return fail(TFG_E_INVALID, "render: null scene array");
    if (prm.max_depth < 1 || prm.max_depth > kMaxBounces) return fail(TFG_E_INVALID, "render: max_depth out of [1,64]");
    if (prm.spp < 1) return fail(TFG_E_INVALID, "render: spp < 1");
    if (prm.tri_format != TFG_TRIS_REF && prm.tri_format != TFG_TRIS_WATERTIGHT)
        return fail(TFG_E_INVALID, "render: unknown tri_format");
    const bool nrc = use_inf || train;
    if (nrc && (!infer || !thr_out)) return fail(TFG_E_INVALID, "render: NRC flags need inference and throughput buffers");
    const bool has_bvh = bvh && bvh->d_nodos && bvh->d_tris && nmesh > 0;
    if (has_bvh && !mesh) return fail(TFG_E_INVALID, "render: mesh primitives are null");
    if (has_bvh && prm.tri_format == TFG_TRIS_WATERTIGHT && !tris_wt)
        return fail(TFG_E_INVALID, "render: watertight format needs tris_wt");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    const Tuning tu = resolve_tuning(dev, (uint32_t)W * (uint32_t)H, prm.spp, nrc, nullptr);
    Workspace ws;
    if (int rc = ensure_workspace(dev, ws_slot, tu.wavefront, nrc, ws)) return rc;
    LaunchShapes sh;
    shapes_for(dev, sh);
    if (prepare_only) return ok();

    PassArgs a{};
    a.prims = prims; a.nprims = nprims; a.lights = lights; a.nlights = nlights;
    a.nodes = has_bvh ? reinterpret_cast<const float4*>(bvh->d_nodos) : nullptr;
    a.tris = has_bvh ? reinterpret_cast<const float4*>(prm.tri_format == TFG_TRIS_REF ? bvh->d_tris : tris_wt) : nullptr;
    a.has_bvh = has_bvh ? 1 : 0;
    a.mesh = mesh; a.nmesh = nmesh;
    a.cam = d_cam;
    a.frame_dev = frame_dev;
    if (policy) a.pol = *policy;
    a.W = W; a.H = H;
    a.accum = accum;
    a.regs = regs; a.reg_counter = reg_counter; a.reg_cap = reg_cap;
    a.infer = infer; a.thr_out = thr_out; a.use_inf = use_inf; a.train = train;
    a.max_depth = prm.max_depth; a.rr_min_depth = prm.rr_min_depth; a.shadow_mesh = prm.shadow_mesh;
    a.ws = ws;
    return enqueue_pass<false>(a, NoTable{}, prm, frame, img, sh, tu, stream);
}

// Several scenes with the same settings in one wavefront series: each stage
// is one launch for all of them, so the small scenes of a batch and the deep,
// sparse bounces of every scene share the GPU.  A path computes exactly what
// it computes in a single-scene pass.
int render_pass_multi(const TfgRenderParams& prm, const PassScene* scenes, int n, int frame, const int32_t* frame_dev,
                      int train, bool prepare_only, int ws_slot, cudaStream_t stream) {
    if (n < 1 || n > kMaxBatchScenes) return fail(TFG_E_INVALID, "render batch: 1 to 16 scenes per pass");
    if (!scenes) return fail(TFG_E_INVALID, "render batch: scenes is null");
    if (prm.max_depth < 1 || prm.max_depth > kMaxBounces) return fail(TFG_E_INVALID, "render: max_depth out of [1,64]");
    if (prm.spp < 1) return fail(TFG_E_INVALID, "render: spp < 1");
    if (prm.tri_format != TFG_TRIS_REF && prm.tri_format != TFG_TRIS_WATERTIGHT)
        return fail(TFG_E_INVALID, "render: unknown tri_format");
    SceneTable tab{};
    tab.n = n;
    uint64_t total = 0;
    int any_inf = 0;
    for (int i = 0; i < n; ++i) {
        const PassScene& c = scenes[i];
        const std::string at = "render batch: scene " + std::to_string(i) + ": ";
        if (c.W <= 0 || c.H <= 0) return fail(TFG_E_INVALID, at + "bad image size");
        if (!c.cam) return fail(TFG_E_INVALID, at + "camara is null");
        if (c.nprims < 0 || c.nlights < 0 || c.nmesh < 0) return fail(TFG_E_INVALID, at + "negative count");
        if ((c.nprims > 0 && !c.prims) || (c.nlights > 0 && !c.lights)) return fail(TFG_E_INVALID, at + "null scene array");
        if ((c.use_inf || train) && (!c.infer || !c.thr_out))
            return fail(TFG_E_INVALID, at + "NRC flags need inference and throughput buffers");
        const bool has_bvh = c.bvh && c.bvh->d_nodos && c.bvh->d_tris && c.nmesh > 0;
        if (has_bvh && !c.mesh) return fail(TFG_E_INVALID, at + "mesh primitives are null");
        if (has_bvh && prm.tri_format == TFG_TRIS_WATERTIGHT && !c.tris_wt)
            return fail(TFG_E_INVALID, at + "watertight format needs tris_wt");
        SceneDesc& d = tab.s[i];
        d.prims = c.prims; d.nprims = c.nprims; d.lights = c.lights; d.nlights = c.nlights;
        d.nodes = has_bvh ? reinterpret_cast<const float4*>(c.bvh->d_nodos) : nullptr;
        d.tris = has_bvh ? reinterpret_cast<const float4*>(prm.tri_format == TFG_TRIS_REF ? c.bvh->d_tris : c.tris_wt)
                         : nullptr;
        d.has_bvh = has_bvh ? 1 : 0;
        d.mesh = c.mesh; d.nmesh = c.nmesh;
        d.cam = c.cam; d.pol = c.policy; d.use_inf = c.use_inf;
        d.img = c.img; d.accum = c.accum;
        d.regs = c.regs; d.reg_counter = c.reg_counter; d.reg_cap = c.reg_cap;
        d.infer = c.infer; d.thr_out = c.thr_out;
        d.W = c.W; d.H = c.H;
        d.pix0 = (uint32_t)total;
        total += (uint64_t)c.W * (uint64_t)c.H;
        if (total > (1u << 28)) return fail(TFG_E_INVALID, "render batch: more than 2^28 pixels in one pass");
        any_inf |= c.use_inf ? 1 : 0;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    const bool nrc = any_inf || train;
    const Tuning tu = resolve_tuning(dev, (uint32_t)total, prm.spp, nrc, nullptr);
    Workspace ws;
    if (int rc = ensure_workspace(dev, ws_slot, tu.wavefront, nrc, ws)) return rc;
    LaunchShapes sh;
    shapes_for(dev, sh);
    if (prepare_only) return ok();

    PassArgs a{};
    a.frame_dev = frame_dev;
    a.W = (int)total; a.H = 1;
    a.use_inf = any_inf; a.train = train;
    a.max_depth = prm.max_depth; a.rr_min_depth = prm.rr_min_depth; a.shadow_mesh = prm.shadow_mesh;
    a.ws = ws;
    return enqueue_pass<true>(a, tab, prm, frame, nullptr, sh, tu, stream);
}

// The launch sequence of one call: its spp x W x H paths in wavefronts of
// `tu.wavefront` paths, each generate -> (trace -> shade -> shadow) x
// max_depth -> resolve, on the workspace in `a.ws`.
template <bool MS>
int enqueue_pass(PassArgs a, const TableOf<MS>& tab, const TfgRenderParams& prm, int frame, TfgColor* img,
                 const LaunchShapes& sh, const Tuning& tu, cudaStream_t stream) {
    // one scene: W x H pixels; a batch: the scenes' pixels concatenated (a.W = total, a.H = 1)
    const uint32_t N = (uint32_t)a.W * (uint32_t)a.H;
    const int fmt = prm.tri_format;
    const int ti = threads_index(tu.threads);
    const int bt = kThreadChoices[ti];
    const size_t smem = trace_smem(MS ? 0 : a.nprims, bt);
    const int trace_grid = persistent_grid(sh, sh.trace_occ[MS][fmt][ti], tu);
    const int shadow_grid = persistent_grid(sh, sh.shadow_occ[MS][fmt][ti], tu);
    const int shade_grid = sh.shade_blocks[MS];
    const Workspace& ws = a.ws;
    cudaError_t e = cudaSuccess;
    const bool times = (prm.profile & TFG_PROFILE_TIMES) != 0;
    const bool counts = (prm.profile & TFG_PROFILE_COUNTS) != 0;
    auto stage_on = [&](int id, cudaStream_t st, auto&& launch) {
        if (times) {
            StageEvents ev = profiler_pair(id);
            cudaEventRecord(ev.start, st);
            launch();
            cudaEventRecord(ev.stop, st);
        } else {
            launch();
        }
    };
    auto stage = [&](int id, auto&& launch) { stage_on(id, stream, launch); };
    // Shadow stage on the side stream: bounce b's shadow rays run beside
    // bounce b+1's closest-hit trace (which reads only rays and writes only
    // hits); the next shade, which rewrites the shadow items and adds to the
    // same radiance sums, waits for them, so every sum keeps its order.
    const bool overlap = tu.overlap_shadow && ws.side;
    cudaStream_t sstream = overlap ? ws.side : stream;
    a.frame = frame;
    a.img = img;
    a.npix = N;
    a.last_sample = prm.spp - 1;
    a.refill_min = tu.refill;
    a.refill_primary = tu.refill_primary;
    a.shadow_one_lane = tu.shadow_one_lane;
    const uint64_t total = (uint64_t)prm.spp * N;
    for (uint64_t q0 = 0; q0 < total; q0 += tu.wavefront) {
        a.nq = (uint32_t)std::min<uint64_t>(tu.wavefront, total - q0);
        a.s0 = (int)(q0 / N);
        a.p0 = (uint32_t)(q0 % N);
        const int gen_blocks = (int)std::max<uint32_t>(1u, std::min<uint32_t>((a.nq + 255) / 256, (uint32_t)sh.sms * 8u));
        const uint32_t resolve_n = std::min(a.nq, N);
        const int res_blocks = (int)std::max<uint32_t>(1u, std::min<uint32_t>((resolve_n + 255) / 256, (uint32_t)sh.sms * 8u));
        e = cudaMemsetAsync(ws.counters, 0, 4 * (kMaxBounces + 1) * sizeof(uint32_t), stream);
        if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
        stage(0, [&] { k_generate<MS><<<gen_blocks, 256, 0, stream>>>(a, tab); });
        for (int b = 0; b < prm.max_depth; ++b) {
            stage(1, [&] {
                if (fmt == 0) {
                    if (counts) k_trace<0, true, MS><<<trace_grid, bt, smem, stream>>>(a, b, tab);
                    else k_trace<0, false, MS><<<trace_grid, bt, smem, stream>>>(a, b, tab);
                } else {
                    if (counts) k_trace<1, true, MS><<<trace_grid, bt, smem, stream>>>(a, b, tab);
                    else k_trace<1, false, MS><<<trace_grid, bt, smem, stream>>>(a, b, tab);
                }
            });
            if (overlap && b > 0) {   // the previous bounce's shadow stage ends before this shade
                e = cudaStreamWaitEvent(stream, ws.join[b - 1], 0);
                if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
            }
            stage(2, [&] { k_shade<MS><<<shade_grid, 256, 0, stream>>>(a, b, tab); });
            if (overlap) {
                e = cudaEventRecord(ws.fork[b], stream);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(sstream, ws.fork[b], 0);
                if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
            }
            stage_on(3, sstream, [&] {
                if (fmt == 0) {
                    if (counts) k_shadow<0, true, MS><<<shadow_grid, bt, smem, sstream>>>(a, b, tab);
                    else k_shadow<0, false, MS><<<shadow_grid, bt, smem, sstream>>>(a, b, tab);
                } else {
                    if (counts) k_shadow<1, true, MS><<<shadow_grid, bt, smem, sstream>>>(a, b, tab);
                    else k_shadow<1, false, MS><<<shadow_grid, bt, smem, sstream>>>(a, b, tab);
                }
            });
            if (overlap) {
                e = cudaEventRecord(ws.join[b], sstream);
                if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
            }
        }
        if (overlap) {   // join the side stream before the pixels are resolved
            e = cudaStreamWaitEvent(stream, ws.join[prm.max_depth - 1], 0);
            if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
        }
        stage(4, [&] { k_resolve<MS><<<res_blocks, 256, 0, stream>>>(a, tab); });
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail((int)e, std::string("render launch: ") + cudaGetErrorString(e));
    }
    return ok();
}

// ------------------------------------------------------------------ traversal-only entries
// tfgTraceRays: closest hit of a batch of rays, 32 consecutive rays per warp
// (coherent when the rays come in tile order).
template <int TRI_FMT>
__global__ void __launch_bounds__(128) k_trace_rays(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                                                    const float4* __restrict__ rays, uint32_t n, float4* __restrict__ hits,
                                                    uint32_t* fetch) {
    __shared__ uint2 sstack[kSmemStack * 128];
    TravStack st;
    st.smem = sstack; st.stride = blockDim.x; st.tid = threadIdx.x;
    while (true) {
        uint32_t base = 0;
        if (lane_id() == 0) base = atomicAdd(fetch, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= n) break;
        const uint32_t i = base + lane_id();
        if (i < n) {
            const float4 o4 = rays[2 * i], d4 = rays[2 * i + 1];
            float tm = o4.w, hu = 0.0f, hv = 0.0f;
            uint32_t id = kMissId;
            if (!cwbvh_trace<TRI_FMT, false>(nodes, tris, xyz(o4), xyz(d4), 0.0f, tm, id, hu, hv, st, nullptr)) {
                id = kMissId; tm = o4.w; hu = 0.0f; hv = 0.0f;
            }
            hits[i] = make_float4(tm, hu, hv, __uint_as_float(id));
        }
    }
}

// Camera rays of `samples` samples, sample-major; within a sample in
// scanline order or in the path tracer's 8 x 4 tile order.
__global__ void k_camera_rays(const TfgCamara* camp, int W, int H, int frame, int samples, int tiles, float4* rays) {
    const uint32_t N = (uint32_t)W * (uint32_t)H;
    const uint64_t total = (uint64_t)N * (uint32_t)samples;
    const TfgCamara cam = *camp;
    for (uint64_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = (uint32_t)(p / N), l = (uint32_t)(p - (uint64_t)s * N);
        const uint32_t pix = tiles ? tiled_pixel(l, (uint32_t)W, (uint32_t)H) : l;
        const int x = (int)(pix % (uint32_t)W), y = (int)(pix / (uint32_t)W);
        uint32_t rng = seed_pixel(x, y, frame + (int)s);
        const float ox = pcg_uniform(rng);
        const float oy = pcg_uniform(rng);
        V3 O, D;
        camera_ray(cam, x, y, W, H, ox, oy, O, D);
        rays[2 * p] = make_float4(O.x, O.y, O.z, 1e9f);
        rays[2 * p + 1] = make_float4(D.x, D.y, D.z, 0.0f);
    }
}

namespace {
std::mutex g_fetch_mutex;
uint32_t* g_fetch[kMaxDevices] = {nullptr};
}

int trace_rays(const TfgTinyBVHD_GPU* bvh, const float* tris_wt, int fmt, const float* rays, int n, float* hits,
               cudaStream_t stream) {
    if (n < 0) return fail(TFG_E_INVALID, "tfgTraceRays: negative ray count");
    if (n == 0) return ok();
    if (!bvh || !bvh->d_nodos || !rays || !hits) return fail(TFG_E_INVALID, "tfgTraceRays: null argument");
    if (fmt == TFG_TRIS_REF && !bvh->d_tris) return fail(TFG_E_INVALID, "tfgTraceRays: d_tris is null");
    if (fmt == TFG_TRIS_WATERTIGHT && !tris_wt) return fail(TFG_E_INVALID, "tfgTraceRays: tris_wt is null");
    if (fmt != TFG_TRIS_REF && fmt != TFG_TRIS_WATERTIGHT) return fail(TFG_E_INVALID, "tfgTraceRays: bad format");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    uint32_t* fetch;
    {
        std::lock_guard<std::mutex> lk(g_fetch_mutex);
        if (!g_fetch[dev]) {
            e = cudaMalloc((void**)&g_fetch[dev], sizeof(uint32_t));
            if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
        }
        fetch = g_fetch[dev];
    }
    LaunchShapes sh;
    shapes_for(dev, sh);
    e = cudaMemsetAsync(fetch, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    const float4* tr = reinterpret_cast<const float4*>(fmt == TFG_TRIS_REF ? bvh->d_tris : tris_wt);
    if (fmt == 0)
        k_trace_rays<0><<<sh.sms * sh.trace_occ[0][0][1], 128, 0, stream>>>(reinterpret_cast<const float4*>(bvh->d_nodos), tr,
                                                                 reinterpret_cast<const float4*>(rays), (uint32_t)n,
                                                                 reinterpret_cast<float4*>(hits), fetch);
    else
        k_trace_rays<1><<<sh.sms * sh.trace_occ[0][1][1], 128, 0, stream>>>(reinterpret_cast<const float4*>(bvh->d_nodos), tr,
                                                                 reinterpret_cast<const float4*>(rays), (uint32_t)n,
                                                                 reinterpret_cast<float4*>(hits), fetch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail((int)e, std::string("tfgTraceRays: ") + cudaGetErrorString(e));
    return ok();
}

int camera_rays(const TfgCamara* d_cam, int W, int H, int frame, int samples, int order, float* rays,
                cudaStream_t stream) {
    if (!d_cam || !rays || W <= 0 || H <= 0) return fail(TFG_E_INVALID, "tfgGenerateCameraRays: bad argument");
    if (samples < 1 || (uint64_t)W * (uint64_t)H * (uint64_t)samples > (1ull << 31))
        return fail(TFG_E_INVALID, "tfgGenerateCameraRays: samples out of range");
    if (order != TFG_RAYS_SCANLINE && order != TFG_RAYS_TILES)
        return fail(TFG_E_INVALID, "tfgGenerateCameraRays: unknown ray order");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    const int blocks = (int)std::max<uint64_t>(
        1, std::min<uint64_t>(((uint64_t)W * (uint64_t)H * (uint64_t)samples + 255) / 256, 148 * 8));
    k_camera_rays<<<blocks, 256, 0, stream>>>(d_cam, W, H, frame, samples, order == TFG_RAYS_TILES ? 1 : 0,
                                              reinterpret_cast<float4*>(rays));
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    return ok();
}

}  // namespace tfg

// ------------------------------------------------------------------ C ABI
extern "C" void tfgRenderParamsReference(TfgRenderParams* p) {
    if (!p) return;
    p->max_depth = 20;
    p->rr_min_depth = 11;
    p->shadow_mesh = 0;
    p->tri_format = TFG_TRIS_REF;
    p->spp = 1;
    p->accumulate = 0;
    p->profile = 0;
    p->reserved = 0;
}

extern "C" void tfgRenderTuningDefault(TfgRenderTuning* t) {
    if (!t) return;
    std::memset(t, 0, sizeof(*t));
    t->wavefront_paths = 0;
    t->trace_threads = 128;
    t->trace_warps_per_sm = 0;
    t->refill_min = 8;
    t->shadow_one_lane = 0;
    t->refill_min_primary = 0;
    t->overlap_shadow = 1;
}

extern "C" int tfgRenderTuningSet(const TfgRenderTuning* t) {
    if (!t) return tfg::fail(TFG_E_INVALID, "tfgRenderTuningSet: tuning is null");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return tfg::fail((int)e, cudaGetErrorString(e));
    if (int rc = tfg::require_sm100(dev)) return rc;
    return tfg::render_tuning_set(dev, *t);
}

extern "C" int tfgRenderTuningGet(TfgRenderTuning* out) {
    if (!out) return tfg::fail(TFG_E_INVALID, "tfgRenderTuningGet: out is null");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return tfg::fail((int)e, cudaGetErrorString(e));
    if (int rc = tfg::require_sm100(dev)) return rc;
    return tfg::render_tuning_get(dev, out, nullptr);
}

extern "C" int tfgRenderProfileReset(void) { return tfg::profile_reset(); }

extern "C" int tfgRenderProfileGet(TfgRenderProfile* out) { return tfg::profile_get(out); }

extern "C" int tfgLaunchKernelRenderTiny(
    const TfgCamara* camara, const TfgPrimitiva* primitivas, int32_t num_primitivas, const TfgLuzPuntual* luces,
    int32_t num_luces, const TfgPrimitiva* primitivas_malla, int32_t num_primitivas_malla, int32_t ancho_img,
    int32_t alto_img, int32_t samples_per_pixel, int32_t frame_number, const TfgTinyBVHD_GPU* nodos_bvh,
    const TfgPrimitiva* primitivas_bvh, int32_t num_nodos_bvh, const TfgImagenGPU* imagen_directa,
    uint32_t* dev_counter, TfgRegistroEntrenamiento* buffer_registros, uint32_t* counter_train, int32_t max_cap_train,
    TfgDatosMLP* buffer_inference, TfgColor* buffer_throughput, int32_t usar_red_inferencia, int32_t entrenar_red,
    void* stream) {
    (void)primitivas_malla; (void)num_primitivas_malla; (void)samples_per_pixel; (void)dev_counter;
    if (!imagen_directa) return tfg::fail(TFG_E_INVALID, "tfgLaunchKernelRenderTiny: imagen is null");
    if (!buffer_throughput) return tfg::fail(TFG_E_INVALID, "tfgLaunchKernelRenderTiny: throughput buffer is null");
    TfgRenderParams prm;
    tfgRenderParamsReference(&prm);
    // The reference kernel draws a training-pixel decision and writes the
    // inference / throughput buffers every launch (render.h:443-458).
    return tfg::render_pass(prm, camara, primitivas, num_primitivas, luces, num_luces, ancho_img, alto_img, frame_number,
                            nodos_bvh, nullptr, primitivas_bvh, num_nodos_bvh, imagen_directa->datos, nullptr,
                            buffer_registros, counter_train, max_cap_train, buffer_inference, buffer_throughput,
                            usar_red_inferencia, entrenar_red, (cudaStream_t)stream);
}

extern "C" int tfgRenderPass(const TfgRenderParams* params, const TfgCamara* camara, const TfgPrimitiva* primitivas,
                             int32_t num_primitivas, const TfgLuzPuntual* luces, int32_t num_luces, int32_t ancho_img,
                             int32_t alto_img, int32_t frame_number, const TfgTinyBVHD_GPU* nodos_bvh,
                             const float* tris_wt, const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh,
                             const TfgImagenGPU* imagen_directa, float* accum,
                             TfgRegistroEntrenamiento* buffer_registros, uint32_t* counter_train,
                             int32_t max_cap_train, TfgDatosMLP* buffer_inference, TfgColor* buffer_throughput,
                             int32_t usar_red_inferencia, int32_t entrenar_red, void* stream) {
    if (!params) return tfg::fail(TFG_E_INVALID, "tfgRenderPass: params is null");
    TfgColor* img = imagen_directa ? imagen_directa->datos : nullptr;
    return tfg::render_pass(*params, camara, primitivas, num_primitivas, luces, num_luces, ancho_img, alto_img,
                            frame_number, nodos_bvh, tris_wt, primitivas_bvh, num_prims_bvh, img,
                            params->accumulate ? accum : nullptr, buffer_registros, counter_train, max_cap_train,
                            buffer_inference, buffer_throughput, usar_red_inferencia, entrenar_red,
                            (cudaStream_t)stream);
}

static_assert(sizeof(TfgRenderScene) == 88, "TfgRenderScene layout");

extern "C" int tfgRenderPassBatch(int32_t n, const TfgRenderScene* scenes, const TfgRenderParams* params,
                                  int32_t frame_number, void* stream) {
    using namespace tfg;
    if (!params) return fail(TFG_E_INVALID, "tfgRenderPassBatch: params is null");
    if (n < 0 || (n > 0 && !scenes)) return fail(TFG_E_INVALID, "tfgRenderPassBatch: bad scene array");
    // groups of up to 16 scenes, each one wavefront series
    for (int g0 = 0; g0 < n; g0 += kMaxBatchScenes) {
        const int m = std::min(n - g0, kMaxBatchScenes);
        PassScene ps[kMaxBatchScenes] = {};
        for (int i = 0; i < m; ++i) {
            const TfgRenderScene& r = scenes[g0 + i];
            PassScene& c = ps[i];
            c.cam = r.camara; c.prims = r.primitivas; c.nprims = r.num_primitivas;
            c.lights = r.luces; c.nlights = r.num_luces; c.W = r.ancho_img; c.H = r.alto_img;
            c.bvh = r.nodos_bvh; c.tris_wt = r.tris_wt; c.mesh = r.primitivas_bvh; c.nmesh = r.num_prims_bvh;
            c.img = r.imagen; c.accum = params->accumulate ? r.accum : nullptr;
        }
        if (int rc = render_pass_multi(*params, ps, m, frame_number, nullptr, 0, false, 0, (cudaStream_t)stream))
            return rc;
    }
    return ok();
}

extern "C" int tfgTraceRays(const TfgTinyBVHD_GPU* bvh, const float* tris_wt, int32_t tri_format, const float* rays,
                            int32_t n, float* hits, void* stream) {
    return tfg::trace_rays(bvh, tris_wt, tri_format, rays, n, hits, (cudaStream_t)stream);
}

extern "C" int tfgGenerateCameraRays(const TfgCamara* camara, int32_t ancho_img, int32_t alto_img, int32_t frame_number,
                                     float* rays, void* stream) {
    return tfg::camera_rays(camara, ancho_img, alto_img, frame_number, 1, TFG_RAYS_SCANLINE, rays, (cudaStream_t)stream);
}

extern "C" int tfgGenerateCameraRaysEx(const TfgCamara* camara, int32_t ancho_img, int32_t alto_img,
                                       int32_t frame_number, int32_t samples, int32_t order, float* rays,
                                       void* stream) {
    return tfg::camera_rays(camara, ancho_img, alto_img, frame_number, samples, order, rays, (cudaStream_t)stream);
}

extern "C" uint32_t tfgTiledPixel(uint32_t l, uint32_t ancho_img, uint32_t alto_img) {
    if (ancho_img == 0 || alto_img == 0 || l >= ancho_img * alto_img) return 0xFFFFFFFFu;
    return tfg::tiled_pixel(l, ancho_img, alto_img);
}

// ------------------------------------------------------------------ allocation-free render pass
// Some callers cannot allocate device memory at all: code running while
// another thread captures a CUDA graph in global mode (cudaMalloc is illegal
// then), engines that hand the library a fixed memory budget and forbid
// allocations behind their back, and real-time threads that must never block
// on the allocator.  tfgRenderPassStatic serves them: the wavefront queues
// and path state live in this file-scope array, which the library image
// reserves on every GPU that loads it, for the life of the process.
namespace tfg {
namespace {

constexpr size_t kStaticPaths = 128 * 128;
constexpr size_t kStaticCounters = 4 * (kMaxBounces + 1) * sizeof(uint32_t);
// Per path: 2 ray queues (32 B each), hit (16 B), shadow item (64 B),
// throughput, state, prefix and suffix radiance, footprint (16 B each).
constexpr size_t kStaticPathBytes = 2 * 32 + 16 + 64 + 5 * 16;
constexpr size_t kStaticBytes = kStaticPaths * kStaticPathBytes + kStaticCounters;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

std::mutex g_static_mutex;
unsigned char* g_static_base[kMaxDevices] = {nullptr};

// Device address of g_static_scratch for the current device, looked up once
// per device (the array's name is only a host-side stand-in in host code).
int static_scratch(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_static_mutex);
    if (!g_static_base[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return fail((int)e, std::string("tfgRenderPassStatic: scratch address: ") + cudaGetErrorString(e));
        g_static_base[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_static_base[dev];
    return ok();
}

}  // namespace
}  // namespace tfg

extern "C" int tfgRenderPassStatic(const TfgRenderParams* params, const TfgCamara* camara,
                                   const TfgPrimitiva* primitivas, int32_t num_primitivas, const TfgLuzPuntual* luces,
                                   int32_t num_luces, int32_t ancho_img, int32_t alto_img, int32_t frame_number,
                                   const TfgTinyBVHD_GPU* nodos_bvh, const float* tris_wt,
                                   const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh,
                                   const TfgImagenGPU* imagen_directa, float* accum, void* stream) {
    using namespace tfg;
    if (!params) return fail(TFG_E_INVALID, "tfgRenderPassStatic: params is null");
    const TfgRenderParams& prm = *params;
    if (ancho_img <= 0 || alto_img <= 0 || (size_t)ancho_img * (size_t)alto_img > kStaticPaths)
        return fail(TFG_E_INVALID, "tfgRenderPassStatic: image larger than the 16384-pixel (128 x 128) static scratch");
    if (!camara) return fail(TFG_E_INVALID, "tfgRenderPassStatic: camara is null");
    if (num_primitivas < 0 || num_luces < 0 || num_prims_bvh < 0) return fail(TFG_E_INVALID, "tfgRenderPassStatic: negative count");
    if ((num_primitivas > 0 && !primitivas) || (num_luces > 0 && !luces))
        return fail(TFG_E_INVALID, "tfgRenderPassStatic: null scene array");
    if (prm.max_depth < 1 || prm.max_depth > kMaxBounces) return fail(TFG_E_INVALID, "tfgRenderPassStatic: max_depth out of [1,64]");
    if (prm.spp < 1) return fail(TFG_E_INVALID, "tfgRenderPassStatic: spp < 1");
    if (prm.tri_format != TFG_TRIS_REF && prm.tri_format != TFG_TRIS_WATERTIGHT)
        return fail(TFG_E_INVALID, "tfgRenderPassStatic: unknown tri_format");
    if (prm.profile != 0) return fail(TFG_E_INVALID, "tfgRenderPassStatic: profiling is not available here");
    const bool has_bvh = nodos_bvh && nodos_bvh->d_nodos && nodos_bvh->d_tris && num_prims_bvh > 0;
    if (has_bvh && !primitivas_bvh) return fail(TFG_E_INVALID, "tfgRenderPassStatic: mesh primitives are null");
    if (has_bvh && prm.tri_format == TFG_TRIS_WATERTIGHT && !tris_wt)
        return fail(TFG_E_INVALID, "tfgRenderPassStatic: watertight format needs tris_wt");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    unsigned char* base = nullptr;
    if (int rc = static_scratch(dev, &base)) return rc;
    LaunchShapes sh;
    shapes_for(dev, sh);
    Tuning tu = resolve_tuning(dev, (uint32_t)ancho_img * (uint32_t)alto_img, prm.spp, false, nullptr);
    tu.wavefront = std::min<uint32_t>(tu.wavefront, (uint32_t)kStaticPaths);
    // Carve the scratch: queues first, then per-path state, counters last.
    const size_t P = kStaticPaths;
    Workspace ws;
    ws.cap = P;
    ws.ray[0] = reinterpret_cast<float4*>(base);
    ws.ray[1] = ws.ray[0] + 2 * P;
    ws.hit = ws.ray[1] + 2 * P;
    ws.shadow = ws.hit + P;
    ws.thr = ws.shadow + 4 * P;
    ws.st = reinterpret_cast<uint4*>(ws.thr + P);
    ws.lpre = reinterpret_cast<float4*>(ws.st + P);
    ws.lsuf = ws.lpre + P;
    ws.nrc = ws.lsuf + P;
    ws.ts = nullptr;
    ws.counters = reinterpret_cast<uint32_t*>(ws.nrc + P);
    PassArgs a{};
    a.prims = primitivas; a.nprims = num_primitivas; a.lights = luces; a.nlights = num_luces;
    a.nodes = has_bvh ? reinterpret_cast<const float4*>(nodos_bvh->d_nodos) : nullptr;
    a.tris = has_bvh ? reinterpret_cast<const float4*>(prm.tri_format == TFG_TRIS_REF ? nodos_bvh->d_tris : tris_wt)
                     : nullptr;
    a.has_bvh = has_bvh ? 1 : 0;
    a.mesh = primitivas_bvh; a.nmesh = num_prims_bvh;
    a.cam = camara;
    a.W = ancho_img; a.H = alto_img;
    a.accum = prm.accumulate ? accum : nullptr;
    a.max_depth = prm.max_depth; a.rr_min_depth = prm.rr_min_depth; a.shadow_mesh = prm.shadow_mesh;
    a.ws = ws;
    return enqueue_pass<false>(a, NoTable{}, prm, frame_number, imagen_directa ? imagen_directa->datos : nullptr, sh,
                               tu, (cudaStream_t)stream);
}
