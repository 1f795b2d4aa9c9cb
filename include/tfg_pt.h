/*
 * tfg_pt.h -- C ABI of the B200 path-tracing hot path (CWBVH traversal,
 * wavefront shading / next-event estimation / Russian roulette, neural
 * radiance cache kernels).
 *
 * Every struct below is byte-for-byte layout compatible with the structure
 * of the same (Spanish) name in the reference project, so a caller can pass
 * its existing device buffers by reinterpret_cast.  Sizes are checked with
 * static asserts in the implementation (tfg_b200/csrc/pt_common.cuh).
 *
 * Every entry point returns 0 on success or a non-zero code (a cudaError_t
 * value, or one of the TFG_E_* codes below).  tfgGetLastErrorString() gives
 * a readable message for the last failure on the calling thread.  The
 * reference's launch wrappers returned void and left error polling to the
 * caller (reference main.cpp:576-594); here each call checks its own launch.
 *
 * All device pointers are caller-owned unless a function says otherwise.
 * `stream` is a cudaStream_t passed as void* (0 = legacy default stream,
 * which is where the reference launched its render kernels,
 * RenderKernel.cu:270).
 */
#ifndef TFG_PT_H
#define TFG_PT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Scene value types (reference L0/L1 structs)                         */
/* ------------------------------------------------------------------ */

/* vector3d.h:14-16 -- three doubles, 24 B. */
typedef struct TfgVec3d { double x, y, z; } TfgVec3d;

/* color.h:13-15 -- three floats, 12 B. */
typedef struct TfgColor { float r, g, b; } TfgColor;

/* primitiva.h:17 enum TipoPrimitiva. */
enum { TFG_ESFERA = 0, TFG_PLANO = 1, TFG_TRIANGULO = 2 };

/* primitiva.h:19-41 -- tagged union, 200 B, union at offset 56. */
typedef struct TfgPrimitiva {
    int32_t  tipo;
    TfgColor emision;
    TfgColor difuso;
    TfgColor especular;
    TfgColor transmision;
    float    indice_refraccion;
    union {
        struct { TfgVec3d centro; float radio; } esfera;
        struct { TfgVec3d normal; float distancia; } plano;
        struct { TfgVec3d v0, v1, v2, v0_normal, v1_normal, v2_normal; } triangulo;
    } u;
} TfgPrimitiva;

/* luzPuntual.h:14-17 -- 40 B. */
typedef struct TfgLuzPuntual { TfgVec3d posicion; TfgColor intensidad; } TfgLuzPuntual;

/* camara.h:15-21 -- 112 B.  `izquierda` = frente x arriba (camera right). */
typedef struct TfgCamara {
    TfgVec3d posicion, frente, arriba, izquierda;
    float ancho_plano, alto_plano, distancia_focal;
} TfgCamara;

/* imagen_gpu.h:14-16 -- passed by value in the reference; 16 B. */
typedef struct TfgImagenGPU { int32_t anchura, altura; TfgColor* datos; } TfgImagenGPU;

/* mlp_types.h:14-23 -- 112 B. */
typedef struct TfgDatosMLP {
    TfgVec3d posicion, direccion, normal;
    TfgColor difuso, especular, color;
} TfgDatosMLP;

/* mlp_types.h:26-29 -- 48 B. */
typedef struct TfgSceneBounds { TfgVec3d min, max; } TfgSceneBounds;

/* mlp_types.h:32-38 -- 96 B. */
typedef struct TfgDatosGeometricos {
    TfgVec3d posicion, direccion, normal;
    TfgColor difuso, especular;
} TfgDatosGeometricos;

/* mlp_types.h:41-54 -- 232 B (bool at 228, padded). */
typedef struct TfgRegistroEntrenamiento {
    TfgDatosGeometricos head, tail;
    TfgColor luz_acumulada_sufijo, throughput_sufijo, factor_normalizacion;
    uint8_t  valido;
} TfgRegistroEntrenamiento;

/* tinybvh_wrapper.h:15-21 -- device descriptor of a CWBVH, passed by value
 * in the reference.  d_nodos: 5 float4 (80 B) per node; d_tris: 4 float4
 * (64 B) per triangle in the reference's transform layout. */
typedef struct TfgTinyBVHD_GPU {
    float*   d_nodos;
    float*   d_tris;
    uint32_t num_nodos;
    uint32_t num_tris;
} TfgTinyBVHD_GPU;

/* ------------------------------------------------------------------ */
/* Error handling                                                      */
/* ------------------------------------------------------------------ */

enum {
    TFG_OK = 0,
    TFG_E_INVALID = 10001,     /* bad argument (null pointer, size out of range) */
    TFG_E_UNSUPPORTED = 10002, /* device is not sm_100 or feature not built */
    TFG_E_TIMEOUT = 10003,     /* a bounded device-side wait ran out */
    TFG_E_BUILD = 10004        /* BVH build failed (e.g. out of memory) */
};

/* Message for the last non-zero return on this thread ("" if none). */
const char* tfgGetLastErrorString(void);

/* ------------------------------------------------------------------ */
/* CWBVH build hand-off (replaces TinyBVH::construirBVH,               */
/* tinybvh_wrapper.cpp:30-83)                                          */
/* ------------------------------------------------------------------ */

/* Host result of a CWBVH build.  Node and reference-triangle arrays use the
 * layout the reference traversal decodes (traverse_cwbvh.cuh:77-209):
 *   node  = 20 floats (80 B): p.xyz, {e.x,e.y,e.z,imask} bytes,
 *           child base (node units), triangle base (float4 units),
 *           meta[0..7], q_lo_x[8], q_lo_y[8], q_lo_z[8], q_hi_x[8], q_hi_y[8], q_hi_z[8]
 *   tris_ref = 16 floats (64 B) per triangle: rows u, v, plane of the
 *           world-to-triangle transform, then (0,0,0,prim id bits)
 *   tris_wt  = 12 floats (48 B) per triangle: v0.xyz, prim id bits,
 *           v1.xyz, 0, v2.xyz, 0  (watertight-test layout)
 * Triangle k of the BVH order lives at tris_*[k]; node field "triangle base"
 * is 4*k so both layouts are addressed from the same nodes. */
typedef struct TfgCWBVHHost {
    float*    nodes;
    float*    tris_ref;
    float*    tris_wt;
    uint32_t  num_nodes;
    uint32_t  num_tris;
    uint32_t  max_depth;  /* deepest node level (root = 1) */
    uint32_t  reserved;
} TfgCWBVHHost;

/* Build over `num_tris` triangles given as 9 floats each (v0,v1,v2).  The
 * prim id stored in each triangle is its index in `verts`.  Arrays in `out`
 * are malloc'ed by the library; release with tfgCWBVHFree.  Host only. */
int  tfgCWBVHBuild(const float* verts, uint32_t num_tris, TfgCWBVHHost* out);
void tfgCWBVHFree(TfgCWBVHHost* bvh);

/* Device-resident CWBVH plus the watertight triangle array.  `ref` is the
 * exact TinyBVHD_GPU a reference caller passes to launchKernelRenderTiny. */
typedef struct TfgTinyBVH {
    TfgTinyBVHD_GPU ref;
    float*          d_tris_wt;
    TfgPrimitiva*   d_primitivas;   /* triangles in input order, as the reference uploads them */
    uint32_t        num_primitivas;
    uint32_t        max_depth;
} TfgTinyBVH;

/* TinyBVH::construirBVH: filter TRIANGULO primitives (input order kept),
 * build, upload nodes / both triangle layouts / primitives with cudaMalloc. */
int  tfgTinyBVHConstruir(const TfgPrimitiva* primitivas_host, int32_t n, TfgTinyBVH* out);
/* The same hand-off built on the GPU from a DEVICE primitive array (the
 * reference builds on the host with tinybvh, tinybvh_wrapper.cpp:30-83):
 * TRIANGULO entries compacted in input order (their index is the prim id),
 * Morton-ordered binary tree (Karras 2012), collapsed to 8-wide nodes and
 * quantised on the device; same node / triangle layouts as
 * tfgTinyBVHConstruir, a lower-quality (LBVH) tree that builds in
 * milliseconds.  Synchronises `stream`; free with tfgTinyBVHLiberar. */
int  tfgTinyBVHConstruirGPU(const TfgPrimitiva* primitivas_device, int32_t n, TfgTinyBVH* out, void* stream);
/* Frees what tfgTinyBVHConstruir / tfgTinyBVHConstruirGPU allocated (TinyBVH::~TinyBVH). */
void tfgTinyBVHLiberar(TfgTinyBVH* bvh);

/* ------------------------------------------------------------------ */
/* Render entry points (RenderKernel.h:47-77)                          */
/* ------------------------------------------------------------------ */

/* Triangle test used against the CWBVH. */
enum {
    TFG_TRIS_REF = 0,        /* reference 64-B transform test (traverse_cwbvh.cuh:189-209) */
    TFG_TRIS_WATERTIGHT = 1  /* 48-B vertices, watertight FP32 test (Woop, Benthin, Wald 2013) */
};

/* Path-tracer settings that the reference hard-codes. */
typedef struct TfgRenderParams {
    int32_t max_depth;     /* bounces; reference 20 (render.h:63) */
    int32_t rr_min_depth;  /* Russian roulette when depth >= this; reference 11 (render.h:209: depth > 10) */
    int32_t shadow_mesh;   /* 1: shadow rays also test the CWBVH mesh; reference kernel 0 (escenario.h:65,168) */
    int32_t tri_format;    /* TFG_TRIS_REF or TFG_TRIS_WATERTIGHT */
    int32_t spp;           /* samples per pixel in this call: frame_number .. frame_number+spp-1 */
    int32_t accumulate;    /* 1: add each sample into `accum` (FP32 RGB per pixel) */
    int32_t profile;       /* TFG_PROFILE_* bits: stage timing / traversal work counters */
    int32_t reserved;
} TfgRenderParams;

enum {
    TFG_PROFILE_TIMES = 1,   /* CUDA events around every stage launch */
    TFG_PROFILE_COUNTS = 2   /* count rays, nodes visited and triangle tests (slower) */
};

/* Stage times and traversal work accumulated by passes run with `profile`
 * set, since the last tfgRenderProfileReset on this device. */
typedef struct TfgRenderProfile {
    double   ms[5];          /* generate, trace, shade, shadow, resolve (sum of launch durations) */
    uint64_t launches[5];
    uint64_t rays;           /* closest-hit rays traced */
    uint64_t nodes;          /* CWBVH nodes decoded by those rays */
    uint64_t tri_tests;      /* triangle tests by those rays */
    uint64_t shadow_rays;    /* shadow rays cast (one per light with cos > 0) */
    uint64_t shadow_nodes;
    uint64_t shadow_tri_tests;
} TfgRenderProfile;

int tfgRenderProfileReset(void);
/* Synchronises the device, then fills `out`. */
int tfgRenderProfileGet(TfgRenderProfile* out);

/* Reference settings: depth 20, RR from depth 11, mesh-free shadow rays,
 * reference triangle layout, 1 spp, no accumulation. */
void tfgRenderParamsReference(TfgRenderParams* p);

/* launchKernelRenderTiny (RenderKernel.h:55-61).  Same arguments and
 * meaning; the grid/block arguments of the reference are dropped because the
 * wavefront stages choose their own launch shapes.  `camara`, all arrays and
 * the counters are device pointers.  Uses the reference settings above and
 * the reference triangle layout in `nodos_bvh`, so a BVH built by either
 * builder works.  Unlike the reference, pixels outside W x H are never
 * written (RenderKernel.cu:35-46 had no bounds guard). */
int tfgLaunchKernelRenderTiny(
    const TfgCamara* camara, const TfgPrimitiva* primitivas, int32_t num_primitivas,
    const TfgLuzPuntual* luces, int32_t num_luces,
    const TfgPrimitiva* primitivas_malla, int32_t num_primitivas_malla,
    int32_t ancho_img, int32_t alto_img, int32_t samples_per_pixel, int32_t frame_number,
    const TfgTinyBVHD_GPU* nodos_bvh, const TfgPrimitiva* primitivas_bvh, int32_t num_nodos_bvh,
    const TfgImagenGPU* imagen_directa,
    uint32_t* dev_counter, TfgRegistroEntrenamiento* buffer_registros, uint32_t* counter_train,
    int32_t max_cap_train, TfgDatosMLP* buffer_inference, TfgColor* buffer_throughput,
    int32_t usar_red_inferencia, int32_t entrenar_red, void* stream);

/* Extended render: explicit settings, optional watertight triangles
 * (`tris_wt`, required when params->tri_format == TFG_TRIS_WATERTIGHT) and
 * optional accumulation buffer `accum` (W*H*3 floats).  Training / inference
 * capture arguments behave as in tfgLaunchKernelRenderTiny and may be null
 * when both NRC flags are 0.  `imagen_directa->datos` receives the last
 * sample's radiance. */
int tfgRenderPass(
    const TfgRenderParams* params,
    const TfgCamara* camara, const TfgPrimitiva* primitivas, int32_t num_primitivas,
    const TfgLuzPuntual* luces, int32_t num_luces,
    int32_t ancho_img, int32_t alto_img, int32_t frame_number,
    const TfgTinyBVHD_GPU* nodos_bvh, const float* tris_wt,
    const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh,
    const TfgImagenGPU* imagen_directa, float* accum,
    TfgRegistroEntrenamiento* buffer_registros, uint32_t* counter_train, int32_t max_cap_train,
    TfgDatosMLP* buffer_inference, TfgColor* buffer_throughput,
    int32_t usar_red_inferencia, int32_t entrenar_red, void* stream);

/* tfgRenderPass without any device allocation -- no counterpart in the
 * reference.  For callers that cannot allocate device memory (code running
 * while another thread captures a CUDA graph in global mode, engines that
 * give the library a fixed memory budget, real-time threads that must not
 * block on the allocator).  The wavefront queues and path state live in a
 * static device array of ~3.7 MB that the library reserves on every GPU that
 * loads it, until the process exits; images are limited to 16384 pixels
 * (e.g. 128 x 128) and plain path tracing (no cache queries or training
 * records) -- larger images return TFG_E_INVALID.  The first call on a device
 * looks up the array's device address; make that first call before any
 * stream capture.  All calls share the one array, which keeps the last call's
 * contents: calls that overlap on the GPU (different streams, or concurrent
 * host threads) race and must be serialised by the caller.  `accum` is used
 * when params->accumulate is set; params->profile must be 0. */
int tfgRenderPassStatic(
    const TfgRenderParams* params,
    const TfgCamara* camara, const TfgPrimitiva* primitivas, int32_t num_primitivas,
    const TfgLuzPuntual* luces, int32_t num_luces,
    int32_t ancho_img, int32_t alto_img, int32_t frame_number,
    const TfgTinyBVHD_GPU* nodos_bvh, const float* tris_wt,
    const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh,
    const TfgImagenGPU* imagen_directa, float* accum, void* stream);

/* One scene of tfgRenderPassBatch: the scene arguments of tfgRenderPass. */
typedef struct TfgRenderScene {
    const TfgCamara*       camara;
    const TfgPrimitiva*    primitivas;
    int32_t                num_primitivas;
    int32_t                num_luces;
    const TfgLuzPuntual*   luces;
    int32_t                ancho_img, alto_img;
    const TfgTinyBVHD_GPU* nodos_bvh;
    const float*           tris_wt;
    const TfgPrimitiva*    primitivas_bvh;
    int32_t                num_prims_bvh;
    int32_t                reserved;
    TfgColor*              imagen;   /* W*H: the last sample's radiance (may be null) */
    float*                 accum;    /* W*H*3 sums when params->accumulate (may be null) */
} TfgRenderScene;

/* No reference counterpart (the reference renders one scene per launch):
 * plain path tracing of `n` scenes of any sizes with the same settings, each
 * stage launched once for all of them (groups of up to 16 scenes share one
 * wavefront series).  Every scene's image equals what tfgRenderPass gives
 * for it alone, bit for bit. */
int tfgRenderPassBatch(int32_t n, const TfgRenderScene* scenes, const TfgRenderParams* params,
                       int32_t frame_number, void* stream);

/* Closest-hit traversal of `n` rays (primary-ray mode).  rays: 8 floats per
 * ray (O.x, O.y, O.z, t_max, D.x, D.y, D.z, unused).  hits: 4 floats per ray
 * (t, u, v, prim id bits); a miss returns t = t_max and id 0xFFFFFFFF.  This
 * is traverse_cwbvh (traverse_cwbvh.cuh:51) over a batch, with 1/D computed
 * per ray as the reference caller does (escenario.h:339-341). */
int tfgTraceRays(const TfgTinyBVHD_GPU* bvh, const float* tris_wt, int32_t tri_format,
                 const float* rays, int32_t n, float* hits, void* stream);

/* Camera rays for one sample of a W x H image, in the reference's order and
 * arithmetic (rng.h:25-35 seed, two jitter draws, camara.h:42-59), written
 * in the tfgTraceRays ray layout with t_max = 1e9 (escenario.h:318). */
int tfgGenerateCameraRays(const TfgCamara* camara, int32_t ancho_img, int32_t alto_img,
                          int32_t frame_number, float* rays, void* stream);

/* ------------------------------------------------------------------ */
/* Launch tuning and the autotuner -- no reference counterpart (the    */
/* reference launches one thread per pixel in fixed 16 x 16 blocks,    */
/* RenderKernel.cu:16-25)                                              */
/* ------------------------------------------------------------------ */

/* How the wavefront stages of the current device are sized and launched.
 * Every setting computes the same image from the same inputs (bit for bit);
 * only speed and memory change. */
typedef struct TfgRenderTuning {
    int32_t wavefront_paths;    /* queue capacity: paths per wavefront, 0 (default) = one sample of every
                                   pixel (W*H).  More runs several samples of the call per launch, less
                                   splits a sample into chunks; passes that query or train the cache
                                   stop at W*H.  0 or 1024 .. 2^26 (224 B of device memory per path) */
    int32_t trace_threads;      /* threads per traversal and shadow-ray CTA: 64, 128 (default) or 256 */
    int32_t trace_warps_per_sm; /* resident traversal warps per SM; 0 (default) = as many as fit */
    int32_t refill_min;         /* idle lanes that make a traversal warp fetch new rays, 1..32 (default 8) */
    int32_t shadow_one_lane;    /* threads per shadow query: 0 (default) = one lane per light (up to 32
                                   lights), 1 = one lane traces all lights of a shading point; both add
                                   the same terms in light order */
    int32_t refill_min_primary; /* refill threshold of the first bounce's traversal (camera rays, coherent
                                   in 8 x 4 pixel tiles; 32 = whole-warp batches), 0 (default) = refill_min */
    int32_t overlap_shadow;     /* 1 (default): each bounce's shadow rays run on a second stream beside the
                                   next bounce's closest-hit trace; 0: one stream */
    int32_t reserved[1];
} TfgRenderTuning;

void tfgRenderTuningDefault(TfgRenderTuning* t);
/* Applies to later passes on the current device, including frames captured
 * as CUDA graphs (they are re-captured on their next call). */
int  tfgRenderTuningSet(const TfgRenderTuning* t);
int  tfgRenderTuningGet(TfgRenderTuning* out);

/* One autotuner measurement: a candidate and its mean pass time. */
typedef struct TfgTuneRecord {
    TfgRenderTuning tuning;
    float ms;
    int32_t reserved;
} TfgTuneRecord;

/* The autotuner: times plain passes of this scene (no image written; the
 * call's spp capped at 16) under candidate tunings with CUDA events on
 * `stream`, one setting at a time starting from the current one (queue size,
 * then CTA size, warps per SM, refill threshold, shadow lanes, first-bounce
 * refill threshold, shadow / trace overlap), `repeats`
 * timed passes per candidate after one warm-up (0 = 3).  A candidate must be
 * at least 1% faster to replace the best.  Sets the winner on the current
 * device and returns it in `out`.  `num_records` (optional) gets the number
 * of candidates timed, the first `max_records` of them stored in `records`
 * (optional) in the order timed.  Synchronous; not during stream capture. */
int  tfgRenderAutotune(const TfgRenderParams* params, const TfgCamara* camara, const TfgPrimitiva* primitivas,
                       int32_t num_primitivas, const TfgLuzPuntual* luces, int32_t num_luces, int32_t ancho_img,
                       int32_t alto_img, const TfgTinyBVHD_GPU* nodos_bvh, const float* tris_wt,
                       const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh, int32_t repeats,
                       TfgRenderTuning* out, TfgTuneRecord* records, int32_t max_records, int32_t* num_records,
                       void* stream);

/* No reference counterpart: camera rays of `samples` consecutive samples
 * (frames frame_number .. frame_number + samples - 1), sample-major, each
 * sample's W*H rays in `order`: TFG_RAYS_SCANLINE (ray l starts at pixel l,
 * as tfgGenerateCameraRays) or TFG_RAYS_TILES, the path tracer's order (ray l
 * starts at pixel tfgTiledPixel(l, W, H): 8 x 4 pixel tiles, so a warp's 32
 * rays are coherent).  At most 2^31 rays. */
enum { TFG_RAYS_SCANLINE = 0, TFG_RAYS_TILES = 1 };
int tfgGenerateCameraRaysEx(const TfgCamara* camara, int32_t ancho_img, int32_t alto_img, int32_t frame_number,
                            int32_t samples, int32_t order, float* rays, void* stream);
/* Pixel index (y * W + x) of the l-th path or ray of a sample in tile
 * order: bands of 4 rows cut into 8 x 4 tiles left to right; 0xFFFFFFFF when
 * l >= W*H. */
uint32_t tfgTiledPixel(uint32_t l, uint32_t ancho_img, uint32_t alto_img);

/* launchInicializarCamara (RenderKernel.cu:68-90): default 45-degree camera
 * at (0,-0.75,4.25) looking down -z, written to device pointer d_camara. */
int tfgLaunchInicializarCamara(TfgCamara* d_camara, int32_t ancho_imagen, int32_t alto_imagen,
                               void* stream);

/* launchKernelComposite (RenderKernel.cu:49-66): img += thr * pred where thr != 0. */
int tfgLaunchKernelComposite(TfgColor* img_pt, const TfgColor* img_prediccion,
                             const TfgColor* throughput_map, int32_t ancho, int32_t alto,
                             void* stream);

/* launchKernelCalcularTargets (RenderKernel.cu:92-137). */
int tfgLaunchKernelCalcularTargets(const TfgRegistroEntrenamiento* buffer_registros,
                                   const TfgColor* buffer_prediccion_tail,
                                   TfgDatosMLP* buffer_training_final, int32_t num_elementos,
                                   void* stream);

/* launchKernelPrepararInferenciaTail (RenderKernel.cu:139-166). */
int tfgLaunchKernelPrepararInferenciaTail(const TfgRegistroEntrenamiento* source_registros,
                                          TfgDatosMLP* dest_inference_inputs,
                                          int32_t num_elements, void* stream);

/* ------------------------------------------------------------------ */
/* NRC data kernels (NrcKernel.h:24-41)                                */
/* ------------------------------------------------------------------ */

/* launchGenerarIndicesAleatorios (NrcKernel.cu:10-16): idx[i] = pcg32(seed ^ i) % max_range. */
int tfgLaunchGenerarIndicesAleatorios(int32_t* indices, int32_t max_range, int32_t count,
                                      uint32_t seed, void* stream);

/* launchPrepararDatosEntrenamiento (NrcKernel.cu:18-68): gather + 15-float rows
 * (position normalised to `bounds` and clamped to [0,1]) + 3-float targets clamped at 1e5. */
int tfgLaunchPrepararDatosEntrenamiento(const TfgDatosMLP* buffer, const int32_t* indices_aleatorios,
                                        int32_t batch_size, int32_t n_in, int32_t n_out,
                                        const TfgSceneBounds* bounds, float* input_matrix,
                                        float* target_matrix, void* stream);

/* launchPrepararDatosInferencia (NrcKernel.cu:70-97). */
int tfgLaunchPrepararDatosInferencia(const TfgDatosMLP* datos, uint32_t n_elements, uint32_t n_in,
                                     float* buffer_in, const TfgSceneBounds* bounds, void* stream);

/* launchGuardarSalidaInferencia (NrcKernel.cu:99-126): clamp to [0,1e5], NaN -> 0, Inf -> 1e5. */
int tfgLaunchGuardarSalidaInferencia(const float* network_output, TfgColor* buffer_color,
                                     int32_t n_elements, void* stream);

/* ------------------------------------------------------------------ */
/* Neural radiance cache MLP (ColorMLP, mlp.h:19-70)                   */
/* ------------------------------------------------------------------ */

/* Opaque cache model: FP32 master weights, Adam moments, an exponential
 * moving average of the weights (used for inference, as the reference's
 * EMA(Adam) optimizer, mlp.cpp:61-69) and packed FP16 / BF16 tensor-core
 * images of them. */
typedef struct TfgColorMLP TfgColorMLP;

/* ColorMLP(n_in=15, n_out=3, batch, config) (mlp.cpp:12-87): 12-band
 * frequency encoding of the position + the 12 other inputs + bias -> 5 x 64
 * ReLU -> 3.  `batch` (samples per train step, reference 16384) must be a
 * multiple of 128.  Weights are drawn from `seed`.  Adam lr 1e-2,
 * beta1 0.9, beta2 0.99, eps 1e-15, EMA decay 0.99. */
int  tfgMlpCreate(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed, TfgColorMLP** out);
/* No reference counterpart (the reference's network has a fixed shape): the
 * same model with 3, 5 (= tfgMlpCreate) or 7 hidden layers of 64 units. */
int  tfgMlpCreateEx(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed, int32_t hidden_layers,
                    TfgColorMLP** out);
/* The reference's own cache input (mlp.cpp:22-49): a multiresolution hash
 * grid on the position, one-blob on direction and normal, identity on the
 * albedos.  Reference settings (tfgHashGridConfigReference): 16 levels of 2
 * features, 2^19 entries per level, base resolution 16, per-level scale 1.5,
 * 4 one-blob bins. */
typedef struct TfgHashGridConfig {
    int32_t n_levels;            /* 1..16 */
    int32_t log2_hashmap_size;   /* 10..24: entries per level */
    float   base_resolution;     /* cells per axis at level 0 (>= 2) */
    float   per_level_scale;     /* >= 1 */
    int32_t reserved[4];
} TfgHashGridConfig;
void tfgHashGridConfigReference(TfgHashGridConfig* c);
/* tfgMlpCreateEx with the composite encoding instead of the frequency
 * encoding; the tables (2 features x n_levels x 2^log2_hashmap_size FP32
 * values, uniform in +-1e-4 from `seed`) train with the same Adam and weight
 * average as the layers.  Inference in FP16, BF16 or FP8 reads an FP16 image
 * of the tables' debiased average. */
int  tfgMlpCreateHashGrid(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed, int32_t hidden_layers,
                          const TfgHashGridConfig* config, TfgColorMLP** out);
/* The cache model with `width` = 64 or 128 units per hidden layer (3, 5 or 7
 * hidden layers; FP16, BF16 or FP8 inference at both widths) and the
 * frequency encoding (`config` null) or the composite encoding. */
int  tfgMlpCreateWide(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed, int32_t hidden_layers,
                      int32_t width, const TfgHashGridConfig* config, TfgColorMLP** out);
/* Length of the FP32 table arrays (0 for the frequency encoding). */
int64_t tfgMlpHashParamCount(const TfgColorMLP* mlp);
/* Table arrays [level][entry][feature]: which = 0 values, 1 average, 2 Adam m, 3 Adam v. */
int  tfgMlpGetHashParams(TfgColorMLP* mlp, int which, float* host, int64_t count);
/* Set the table values and restart the optimiser as tfgMlpSetParams does
 * (moments and averages of layers and tables cleared, step 0). */
int  tfgMlpSetHashParams(TfgColorMLP* mlp, const float* host, int64_t count);
/* tfgMlpComputeGradient that also returns the tables' gradient
 * (`host_table_grad`, tfgMlpHashParamCount floats; may be null). */
int  tfgMlpComputeGradientEx(TfgColorMLP* mlp, const TfgDatosMLP* buffer, uint32_t n_available, uint32_t seed,
                             float* host_grad, uint32_t count, float* host_table_grad, int64_t table_count,
                             float* loss_out);
/* One-blob encoding (the composite encoding's direction and normal input) of
 * `n` values in [0, 1] (device array): 4 bins each into `bins` (device, 4 n
 * floats), exactly as the cache kernels compute them. */
int  tfgOneBlobBins(const float* values, float* bins, int32_t n, void* stream);
/* The cache kernels' layer-0 input of `n` queries (device `DatosMLP`s): 96
 * floats per query (device `out`), each the exact FP16 / BF16 operand the
 * first GEMM reads -- frequency bands, direction, normal, albedos and the
 * constant 1, or the hash-grid, one-blob and albedo features of a composite
 * model.  `pass` TFG_ENCODE_TRAINING gives the training forward pass's FP16
 * features (FP32 tables), TFG_ENCODE_INFERENCE those of inference at the
 * model's precision (FP16 or BF16; FP8 is refused: its features are scaled
 * per call).  A test hook beside tfgOneBlobBins: it pins the GEMM chain of
 * the cache kernels against a model fed with these features.  No reference
 * counterpart (tiny-cuda-nn encodes inside its own kernels). */
#define TFG_ENCODE_TRAINING  0
#define TFG_ENCODE_INFERENCE 1
int  tfgMlpEncodeFeatures(TfgColorMLP* mlp, const TfgDatosMLP* in, uint32_t n, int32_t pass, float* out,
                          void* stream);
/* Length of the model's FP32 parameter arrays: 96 W + W^2 (hidden - 1) + 16 W
 * for width W (23552 for 5 hidden layers of 64, 79872 for 5 of 128). */
int32_t tfgMlpParamCount(const TfgColorMLP* mlp);
void tfgMlpDestroy(TfgColorMLP* mlp);
/* ColorMLP::setBounds (mlp.cpp:89-93): position normalisation box. */
int  tfgMlpSetBounds(TfgColorMLP* mlp, const TfgSceneBounds* bounds);
int  tfgMlpSetHyperparams(TfgColorMLP* mlp, float lr, float beta1, float beta2, float eps, float ema_decay);
/* ColorMLP::train_step (mlp.cpp:95-125): one Adam step on `batch` samples
 * drawn as pcg32(step ^ i) % n_available (NrcKernel.cu:10-16) from the
 * DatosMLP training buffer (targets in .color).  No step below 100 samples
 * (mlp.cpp:96).  When `loss_out` is not null the call synchronises the stream
 * and returns the batch loss there (the reference always did, mlp.cpp:122);
 * with null it stays asynchronous. */
int  tfgMlpTrainStep(TfgColorMLP* mlp, const TfgDatosMLP* buffer, uint32_t n_available, float* loss_out,
                     void* stream);
/* ColorMLP::inference (mlp.cpp:127-170): scrubbed predictions (clamped to
 * [0, 1e5], NaN -> 0) of `count` samples into `out`.  `in` must be 16-byte
 * aligned.  Asynchronous (the reference synchronised here). */
int  tfgMlpInference(TfgColorMLP* mlp, const TfgDatosMLP* in, TfgColor* out, uint32_t count, void* stream);
/* Inference fused with launchKernelComposite (RenderKernel.cu:49-66):
 * img[i] += throughput[i] * prediction where throughput[i] != 0. */
int  tfgMlpInferenceComposite(TfgColorMLP* mlp, const TfgDatosMLP* in, const TfgColor* throughput, TfgColor* img,
                              uint32_t count, void* stream);
/* No reference counterpart (tiny-cuda-nn runs its network in FP16): operand
 * precision of later inference calls -- TFG_MLP_FP16 (default), TFG_MLP_BF16,
 * or TFG_MLP_FP8 (E4M3 with per-layer scales).  Accumulation is FP32 in all
 * three and training is unchanged; the BF16 / FP8 weight images are re-packed
 * from the weight average before every such call. */
#define TFG_MLP_FP16 0
#define TFG_MLP_BF16 1
#define TFG_MLP_FP8  2
int  tfgMlpSetPrecision(TfgColorMLP* mlp, int32_t precision);
/* ColorMLP::save_model / load_model (mlp.cpp:173-276): a binary checkpoint of
 * the weights, weight average, Adam moments, step counters, bounds and
 * hyper-parameters (tiny-cuda-nn's JSON format is not reproduced).  Loading
 * needs a model of the same depth and restores training exactly where it
 * stopped. */
int  tfgMlpSave(TfgColorMLP* mlp, const char* path);
int  tfgMlpLoad(TfgColorMLP* mlp, const char* path);
/* No reference counterpart: FP8 input scales from the per-layer input amax of
 * `count` samples run through the FP16 path (scale = 448 / (2 amax)).  Needed
 * once before FP8 inference; afterwards every FP8 call re-derives the scales
 * from the amax it sees on the first tile of each slot (delayed scaling), so
 * they follow the model while it trains.  `in` must be 16-byte aligned. */
int  tfgMlpCalibrate(TfgColorMLP* mlp, const TfgDatosMLP* in, uint32_t count, void* stream);
/* FP32 parameter arrays (count = tfgMlpParamCount, padded [out][in] per layer):
 * which = 0 weights, 1 EMA, 2 Adam m, 3 Adam v. */
int  tfgMlpGetParams(TfgColorMLP* mlp, int which, float* host, uint32_t count);
/* Set the weights and restart the optimiser (Adam moments and the weight
 * average cleared, step 0, so inference uses these weights until the next
 * step); re-packs the tensor-core images. */
int  tfgMlpSetParams(TfgColorMLP* mlp, const float* host, uint32_t count);
/* d loss / d W for one batch drawn with `seed`, without updating anything
 * (synchronous; for gradient checks). */
int  tfgMlpComputeGradient(TfgColorMLP* mlp, const TfgDatosMLP* buffer, uint32_t n_available, uint32_t seed,
                           float* host_grad, uint32_t count, float* loss_out);
/* Diagnostic without a reference counterpart: runs one bounded wait that can
 * never complete (an mbarrier nothing arrives on) with a `timeout_us` limit
 * (at most 2 s) through the cache kernels' wait and error-flag path, and
 * returns what a stuck cache kernel would: TFG_E_TIMEOUT (the flag is cleared
 * and the context stays usable).  Every real wait gives up after 1 s. */
int  tfgMlpSelfTestWait(uint32_t timeout_us);
/* Roofline probe for the traversal stages (no reference counterpart): every
 * thread of `blocks` x 256 reads `reads_per_thread` records of 80 bytes (five
 * 16-byte loads, a CWBVH node's size) at hashed, independent indices of the
 * device `table` of `records` records (16-byte aligned), so that an
 * L2-resident table gives the random-gather bandwidth of L2.  `sink` is a
 * device word the kernel may write; time the call with events. */
int  tfgL2GatherPass(const void* table, uint32_t records, uint32_t reads_per_thread, uint32_t seed, uint32_t* sink,
                     int32_t blocks, void* stream);
/* How a model's kernels tile their batches (no reference counterpart).
 * Every setting computes the same values up to the order of FP32 gradient
 * additions. */
typedef struct TfgMlpTuning {
    int32_t wgrad_tiles_per_cta;  /* 128-sample tiles one weight-gradient CTA reduces before adding to the
                                     gradient; 0 (default) = max(2, tiles / 16) */
    int32_t infer_ctas;           /* CTAs of an inference launch (4 tiles of 128 in flight each);
                                     0 (default) = one per SM */
    int32_t reserved[2];
} TfgMlpTuning;
int  tfgMlpTuningSet(TfgColorMLP* mlp, const TfgMlpTuning* t);
int  tfgMlpTuningGet(TfgColorMLP* mlp, TfgMlpTuning* out);
/* The autotuner for the model's kernels: times the weight-gradient kernel of
 * one training batch for tiles-per-CTA in {1, 2, 4, ..., 64} and inference of
 * `count` samples of `in` (written to `out`) for CTA counts of 1/2, 3/4 and 1
 * per SM, `repeats` timed launches each after a warm-up (0 = 5), with CUDA
 * events on `stream`.  The model's weights, optimiser state, pending gradient
 * and FP8 scales are left as they were.  Sets and returns the winners;
 * `ms_out` (optional, 2 floats) gets their times.  Synchronous. */
int  tfgMlpAutotune(TfgColorMLP* mlp, const TfgDatosMLP* in, uint32_t count, TfgColor* out, int32_t repeats,
                    TfgMlpTuning* result, float* ms_out, void* stream);
/* TFG_E_TIMEOUT if a bounded tensor-core wait in an MLP kernel gave up since
 * the last call (synchronous). */
int  tfgMlpStatus(void);
/* Device training state (synchronous): [0] step counter, [1] Adam step,
 * [2] records used by the last step, [3] open cells of the gate grid after the last gated frame,
 * [4] running loss (float bits), [5..7] reserved. */
int  tfgMlpGetState(TfgColorMLP* mlp, uint32_t* out8);

/* ------------------------------------------------------------------ */
/* One cache frame (main.cpp:995-1061) without host synchronisation    */
/* ------------------------------------------------------------------ */

typedef struct TfgNrcFrameConfig {
    int32_t  train_steps;     /* train_step calls per frame; reference 1 (main.cpp:1056) */
    uint32_t max_records;     /* records used per frame; reference 65536 (main.cpp:1036) */
    uint32_t min_records;     /* train only above this count; reference 1024 (main.cpp:1043) */
    int32_t  warmup;          /* 1: no cache queries, every path is a training path (main.cpp:997) */
    float    gate_threshold;  /* > 0: per-cell gate judged by the path tracer.  Training records whose
                                 suffix ran to its end (unbiased estimates of the radiance at their head)
                                 are compared with the cache's answer there, per cell of a 32^3 grid over
                                 the model's scene bounds, in running sums decayed by 0.8 per frame; a
                                 cell opens once it holds 8 samples' weight and the cache's running
                                 relative error there (|mean error| over sqrt(mean target^2 + 0.01)) is
                                 below this value, and closes again when it rises.  Paths query the
                                 cache, training paths record bootstrapped heads and cut their suffixes
                                 into it only in open cells; elsewhere they go on as plain paths, so with
                                 every cell closed a frame renders plain path tracing.  The training and
                                 unbiased draws then come from a per-pixel stream of their own, which
                                 leaves each path the random numbers of a plain pass.
                                 0: no gate, the reference's behaviour (render.h:182) */
    int32_t  use_graph;       /* 1: capture the frame as a CUDA graph on first use and replay it
                                 (needs a non-default stream) */
    float    footprint;       /* a path queries (or records a training head) once its footprint
                                 a_suffix >= footprint * a_0; reference 0.01 (render.h:86-102).  0: at
                                 the first diffuse, non-specular vertex, the primary hit included */
    float    train_fraction;  /* share of paths traced for training while queries are on; reference
                                 0.05 (render.h:443) */
} TfgNrcFrameConfig;

/* Reference frame settings: 1 step, 65536 records, train above 1024, footprint 0.01,
 * 5 % training paths, no gate, no graph. */
void tfgNrcFrameConfigReference(TfgNrcFrameConfig* cfg);

/* Caller-owned device buffers of a cache frame (main.cpp:908-930). */
typedef struct TfgNrcBuffers {
    TfgColor*                 img;        /* W*H: frame radiance (prefix + cache) */
    float*                    accum;      /* W*H*3 running sum, or null */
    TfgDatosMLP*              infer;      /* W*H cache queries */
    TfgColor*                 thr;        /* W*H throughput at the query vertex */
    TfgRegistroEntrenamiento* regs;       /* training-record ring */
    uint32_t*                 counter;    /* ring counter (1 word) */
    uint32_t                  ring_cap;   /* ring capacity, >= max_records */
    uint32_t                  reserved;
    TfgDatosMLP*              tail_in;    /* max_records */
    TfgColor*                 tail_pred;  /* max_records */
    TfgDatosMLP*              train_buf;  /* max_records */
} TfgNrcBuffers;

/* Render one sample per pixel with cache queries and training records, answer
 * the queries with the cache and composite into buffers->img (accumulating
 * into buffers->accum if set), then bootstrap targets and take
 * cfg->train_steps Adam steps -- all enqueued on `stream` with the record
 * count kept in device memory.  `params` sets depth / roulette / shadows /
 * triangle test (spp is forced to 1).  `frame` seeds the RNG
 * (rng.h:25-35). */
int tfgNrcFrame(TfgColorMLP* mlp, const TfgNrcFrameConfig* cfg, const TfgRenderParams* params,
                const TfgCamara* camara, const TfgPrimitiva* primitivas, int32_t num_primitivas,
                const TfgLuzPuntual* luces, int32_t num_luces, int32_t ancho_img, int32_t alto_img,
                const TfgTinyBVHD_GPU* bvh, const float* tris_wt, const TfgPrimitiva* primitivas_bvh,
                int32_t num_prims_bvh, const TfgNrcBuffers* buffers, int32_t frame, void* stream);

/* The reference's reconstruction mode (main.cpp:454-668): `spp` samples
 * (frames first_frame ..) rendered with cache queries and no training, each
 * answered by the cache, composited into `img` and summed into `accum`
 * (W*H*3 floats, cleared first) -- all enqueued on `stream`, no host
 * synchronisation.  `img`, `infer`, `thr`: W*H scratch buffers.  Finish with
 * tfgToneMapFilmic(accum, spp, ...). */
int tfgNrcReconstruct(TfgColorMLP* mlp, const TfgRenderParams* params, const TfgCamara* camara,
                      const TfgPrimitiva* primitivas, int32_t num_primitivas, const TfgLuzPuntual* luces,
                      int32_t num_luces, int32_t ancho_img, int32_t alto_img, const TfgTinyBVHD_GPU* bvh,
                      const float* tris_wt, const TfgPrimitiva* primitivas_bvh, int32_t num_prims_bvh, int32_t spp,
                      int32_t first_frame, TfgColor* img, TfgDatosMLP* infer, TfgColor* thr, float* accum,
                      void* stream);

/* Final image (main.cpp:1108-1115): accum / frames into `hdr_out` (W*H*3
 * floats, optional) and the reference's filmic curve (imagen.h:193-214) as
 * 8-bit RGB, round(clamp(v, 0, 1) * 255) (imagen_utils.h:59-62), into
 * `rgb8_out` (W*H*3 bytes, optional).  Device buffers. */
int tfgToneMapFilmic(const float* accum, int32_t frames, int32_t ancho_img, int32_t alto_img, float* hdr_out,
                     uint8_t* rgb8_out, void* stream);
/* Headless image files from host buffers (the reference writes PNG through
 * libpng, absent here): binary PPM (8-bit RGB, top row first) and PFM (float
 * RGB, little-endian, bottom row first as the format requires). */
int tfgWritePPM(const char* path, const uint8_t* rgb8, int32_t ancho_img, int32_t alto_img);
int tfgWritePFM(const char* path, const float* rgb, int32_t ancho_img, int32_t alto_img);

/* One scene of a batched cache frame: the arguments of tfgNrcFrame (104 B). */
typedef struct TfgNrcSceneFrame {
    TfgColorMLP*             mlp;
    const TfgNrcFrameConfig* cfg;
    const TfgRenderParams*   params;
    const TfgCamara*         camara;
    const TfgPrimitiva*      primitivas;
    const TfgLuzPuntual*     luces;
    const TfgTinyBVHD_GPU*   bvh;
    const float*             tris_wt;
    const TfgPrimitiva*      primitivas_bvh;
    const TfgNrcBuffers*     buffers;
    int32_t                  num_primitivas;
    int32_t                  num_luces;
    int32_t                  num_prims_bvh;
    int32_t                  ancho_img;
    int32_t                  alto_img;
    int32_t                  reserved;
} TfgNrcSceneFrame;

/* No reference counterpart (the reference renders one scene per process).
 * One cache frame of each of `n` independent scenes -- each with its own
 * cache model, configuration and buffers, all distinct -- as tfgNrcFrame
 * would run it, enqueued on `stream` as up to four concurrent branches
 * (scenes assigned largest first, one render workspace per branch).  With
 * `use_graph` set and a non-default `stream`, the whole batch is captured
 * once as a single CUDA graph (re-captured when any argument changes) and
 * replayed.  `frame` seeds every scene's RNG; cfg->use_graph is ignored. */
int tfgNrcFrameBatch(int32_t n, const TfgNrcSceneFrame* scenes, int32_t frame, int32_t use_graph, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TFG_PT_H */
