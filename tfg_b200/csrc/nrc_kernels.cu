// Element-wise kernels around the radiance cache: the reference's
// NrcKernel.cu:5-126 (batch indices, 15-float feature rows, output scrub) and
// RenderKernel.cu:49-166 (composite, bootstrapped targets, tail queries,
// default camera).  Each computes exactly what the reference kernel computes,
// in the same FP32 operation order, so results are bit-identical when built
// with the same compiler settings.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/tfg_pt.h"
#include "pt_common.cuh"
#include "tfg_errors.h"
#include "tfg_runtime.h"

namespace tfg {

namespace {

__device__ __forceinline__ float unit_clamp(float v, float lo, float hi) {   // NrcKernel.cu:5-8
    float n = (v - lo) / (hi - lo);
    return fminf(fmaxf(n, 0.0f), 1.0f);
}

__device__ __forceinline__ void feature_row(const TfgDatosMLP& d, const TfgSceneBounds& b, float* row) {
    row[0] = unit_clamp((float)d.posicion.x, (float)b.min.x, (float)b.max.x);
    row[1] = unit_clamp((float)d.posicion.y, (float)b.min.y, (float)b.max.y);
    row[2] = unit_clamp((float)d.posicion.z, (float)b.min.z, (float)b.max.z);
    row[3] = (float)d.direccion.x; row[4] = (float)d.direccion.y; row[5] = (float)d.direccion.z;
    row[6] = (float)d.normal.x; row[7] = (float)d.normal.y; row[8] = (float)d.normal.z;
    row[9] = d.difuso.r; row[10] = d.difuso.g; row[11] = d.difuso.b;
    row[12] = d.especular.r; row[13] = d.especular.g; row[14] = d.especular.b;
}

__global__ void k_indices(int* idx, int max_range, int count, uint32_t seed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        uint32_t s = seed ^ (uint32_t)i;
        idx[i] = (int)(pcg_next(s) % (uint32_t)max_range);
    }
}

__global__ void k_train_rows(const TfgDatosMLP* __restrict__ buf, const int* __restrict__ idx, int batch, int n_in,
                             int n_out, TfgSceneBounds b, float* __restrict__ in, float* __restrict__ tgt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    const TfgDatosMLP d = buf[idx[i]];
    feature_row(d, b, in + (size_t)i * n_in);
    float r = d.color.r, g = d.color.g, bl = d.color.b;
    const float mx = 100000.0f;
    if (r > mx) r = mx;
    if (g > mx) g = mx;
    if (bl > mx) bl = mx;
    float* t = tgt + (size_t)i * n_out;
    t[0] = r; t[1] = g; t[2] = bl;
}

__global__ void k_infer_rows(const TfgDatosMLP* __restrict__ d, uint32_t n, uint32_t n_in, float* __restrict__ out,
                             TfgSceneBounds b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int)n) return;
    feature_row(d[i], b, out + (size_t)i * n_in);
}

__global__ void k_scrub(const float* __restrict__ net, TfgColor* __restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float c[3] = {net[3 * i], net[3 * i + 1], net[3 * i + 2]};
    const float mx = 100000.0f;
    for (int k = 0; k < 3; ++k) {
        if (c[k] < 0.0f) c[k] = 0.0f;
        if (isnan(c[k])) c[k] = 0.0f;
        if (c[k] > mx) c[k] = mx;
        if (isinf(c[k])) c[k] = mx;
    }
    out[i] = TfgColor{c[0], c[1], c[2]};
}

__global__ void k_composite(TfgColor* img, const TfgColor* pred, const TfgColor* thr, int W, int H) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const int i = y * W + x;
    TfgColor f = img[i];
    const TfgColor t = thr[i], p = pred[i];
    if (t.r > 0 || t.g > 0 || t.b > 0) {
        f.r = f.r + t.r * p.r;
        f.g = f.g + t.g * p.g;
        f.b = f.b + t.b * p.b;
    }
    img[i] = f;
}

__global__ void k_targets(const TfgRegistroEntrenamiento* regs, const TfgColor* tail, TfgDatosMLP* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const TfgRegistroEntrenamiento r = regs[i];
    if (!r.valido) {
        out[i].color = TfgColor{0.0f, 0.0f, 0.0f};
        return;
    }
    const TfgColor tl = tail[i];
    const float rr = r.luz_acumulada_sufijo.r + r.throughput_sufijo.r * tl.r;
    const float rg = r.luz_acumulada_sufijo.g + r.throughput_sufijo.g * tl.g;
    const float rb = r.luz_acumulada_sufijo.b + r.throughput_sufijo.b * tl.b;
    const float eps = 1e-8f;
    float c[3] = {rr / fmaxf(r.factor_normalizacion.r, eps), rg / fmaxf(r.factor_normalizacion.g, eps),
                  rb / fmaxf(r.factor_normalizacion.b, eps)};
    for (int k = 0; k < 3; ++k) {
        c[k] = fminf(c[k], 100000.0f);
        if (isnan(c[k]) || isinf(c[k])) c[k] = 0.0f;
    }
    TfgDatosMLP d;
    d.posicion = r.head.posicion; d.direccion = r.head.direccion; d.normal = r.head.normal;
    d.difuso = r.head.difuso; d.especular = r.head.especular;
    d.color = TfgColor{c[0], c[1], c[2]};
    out[i] = d;
}

__global__ void k_tail(const TfgRegistroEntrenamiento* __restrict__ regs, TfgDatosMLP* __restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const TfgRegistroEntrenamiento& r = regs[i];
    TfgDatosMLP d;
    memset(&d, 0, sizeof(d));
    if (r.valido) {
        d.posicion = r.tail.posicion; d.direccion = r.tail.direccion; d.normal = r.tail.normal;
        d.difuso = r.tail.difuso; d.especular = r.tail.especular;
    }
    out[i] = d;
}

// RenderKernel.cu:68-90: focal 1, vertical FOV 45 deg, pose (0,-0.75,4.25) -> -z;
// camara.h:29-40 orthonormalises the frame.
__global__ void k_default_camera(TfgCamara* c, int W, int H) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const float focal = 1.0f;
    const float fov = 45.0f * 3.14159265358979323846 / 180.0f;
    const float alto = 2.0f * focal * tanf(fov / 2.0f);
    const float ancho = alto * (static_cast<float>(W) / H);
    auto norm = [](double& x, double& y, double& z) {
        double l = sqrt(x * x + y * y + z * z);
        if (l > 0.0) { double il = 1.0 / l; x *= il; y *= il; z *= il; }
    };
    double fx = 0, fy = 0, fz = -1, ax = 0, ay = 1, az = 0;
    norm(fx, fy, fz);
    norm(ax, ay, az);
    double lx = fy * az - fz * ay, ly = fz * ax - fx * az, lz = fx * ay - fy * ax;
    norm(lx, ly, lz);
    double ux = ly * fz - lz * fy, uy = lz * fx - lx * fz, uz = lx * fy - ly * fx;
    norm(ux, uy, uz);
    TfgCamara r;
    r.posicion = TfgVec3d{0.0, -0.75, 4.25};
    r.frente = TfgVec3d{fx, fy, fz};
    r.arriba = TfgVec3d{ux, uy, uz};
    r.izquierda = TfgVec3d{lx, ly, lz};
    r.ancho_plano = ancho; r.alto_plano = alto; r.distancia_focal = focal;
    *c = r;
}

// Device-count forms for the frame driver: the record count lives in device
// memory (no host read between render and training).
// GATED: a complete record (its suffix ran to the end: zero suffix
// throughput, so the targets ignore its tail prediction) queries its head
// instead, which gives the gate update the cache's prediction there.
template <bool GATED>
__global__ void k_tail_dev(const TfgRegistroEntrenamiento* __restrict__ regs, TfgDatosMLP* __restrict__ out,
                           const uint32_t* n_dev, uint32_t min_n) {
    const uint32_t n = *n_dev;
    if (n < min_n) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const TfgRegistroEntrenamiento& r = regs[i];
        TfgDatosMLP d;
        memset(&d, 0, sizeof(d));
        if (r.valido) {
            const TfgColor ts = r.throughput_sufijo;
            const bool complete = GATED && ts.r == 0.0f && ts.g == 0.0f && ts.b == 0.0f;
            const TfgDatosGeometricos& v = complete ? r.head : r.tail;
            d.posicion = v.posicion; d.direccion = v.direccion; d.normal = v.normal;
            d.difuso = v.difuso; d.especular = v.especular;
        }
        out[i] = d;
    }
}

__global__ void k_targets_dev(const TfgRegistroEntrenamiento* regs, const TfgColor* tail, TfgDatosMLP* out,
                              const uint32_t* n_dev, uint32_t min_n) {
    const uint32_t n = *n_dev;
    if (n < min_n) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const TfgRegistroEntrenamiento r = regs[i];
        if (!r.valido) { out[i].color = TfgColor{0.0f, 0.0f, 0.0f}; continue; }
        const TfgColor tl = tail[i];
        const float rr = r.luz_acumulada_sufijo.r + r.throughput_sufijo.r * tl.r;
        const float rg = r.luz_acumulada_sufijo.g + r.throughput_sufijo.g * tl.g;
        const float rb = r.luz_acumulada_sufijo.b + r.throughput_sufijo.b * tl.b;
        float c[3] = {rr / fmaxf(r.factor_normalizacion.r, 1e-8f), rg / fmaxf(r.factor_normalizacion.g, 1e-8f),
                      rb / fmaxf(r.factor_normalizacion.b, 1e-8f)};
        for (int k = 0; k < 3; ++k) {
            c[k] = fminf(c[k], 100000.0f);
            if (isnan(c[k]) || isinf(c[k])) c[k] = 0.0f;
        }
        TfgDatosMLP d;
        d.posicion = r.head.posicion; d.direccion = r.head.direccion; d.normal = r.head.normal;
        d.difuso = r.head.difuso; d.especular = r.head.especular;
        d.color = TfgColor{c[0], c[1], c[2]};
        out[i] = d;
    }
}

// main.cpp:1033-1039: records appended this frame, capped and rounded down
// to a multiple of 4.
__global__ void k_record_count(const uint32_t* counter, uint32_t* n_out, uint32_t cap) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        uint32_t n = min(*counter, cap);
        *n_out = (n / 4u) * 4u;
    }
}

__global__ void k_accumulate(float* __restrict__ accum, const TfgColor* __restrict__ img, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const TfgColor c = img[i];
        accum[3 * (size_t)i] += c.r;
        accum[3 * (size_t)i + 1] += c.g;
        accum[3 * (size_t)i + 2] += c.b;
    }
}

int launch_check(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail((int)e, std::string(what) + ": " + cudaGetErrorString(e));
    return ok();
}

int device_ok() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    return require_sm100(dev);
}

inline int blocks_for(long n) { return (int)std::max(1L, (n + 255) / 256); }

}  // namespace

int launch_nrc_frame_small(int which, const void* a, void* b, const void* c, const uint32_t* n_dev, uint32_t cap,
                           uint32_t min_n, cudaStream_t s) {
    const int blocks = std::max(1, std::min((int)((cap + 255) / 256), 148 * 4));
    switch (which) {
        case 0:
            k_tail_dev<false><<<blocks, 256, 0, s>>>(static_cast<const TfgRegistroEntrenamiento*>(a),
                                                     static_cast<TfgDatosMLP*>(b), n_dev, min_n);
            return launch_check("nrc tail queries");
        case 4:
            k_tail_dev<true><<<blocks, 256, 0, s>>>(static_cast<const TfgRegistroEntrenamiento*>(a),
                                                    static_cast<TfgDatosMLP*>(b), n_dev, min_n);
            return launch_check("nrc gated tail queries");
        case 1:
            k_targets_dev<<<blocks, 256, 0, s>>>(static_cast<const TfgRegistroEntrenamiento*>(a),
                                                 static_cast<const TfgColor*>(c), static_cast<TfgDatosMLP*>(b), n_dev,
                                                 min_n);
            return launch_check("nrc targets");
        case 2:
            k_record_count<<<1, 32, 0, s>>>(static_cast<const uint32_t*>(a), static_cast<uint32_t*>(b), cap);
            return launch_check("nrc record count");
        case 3:
            k_accumulate<<<blocks, 256, 0, s>>>(static_cast<float*>(b), static_cast<const TfgColor*>(a), cap);
            return launch_check("accumulate");
        default:
            return fail(TFG_E_INVALID, "unknown frame kernel");
    }
}

}  // namespace tfg

using namespace tfg;

extern "C" int tfgLaunchGenerarIndicesAleatorios(int32_t* indices, int32_t max_range, int32_t count, uint32_t seed,
                                                 void* stream) {
    if (!indices || count < 0 || max_range <= 0) return fail(TFG_E_INVALID, "tfgLaunchGenerarIndicesAleatorios: bad argument");
    if (int rc = device_ok()) return rc;
    if (count == 0) return ok();
    k_indices<<<blocks_for(count), 256, 0, (cudaStream_t)stream>>>(indices, max_range, count, seed);
    return launch_check("tfgLaunchGenerarIndicesAleatorios");
}

extern "C" int tfgLaunchPrepararDatosEntrenamiento(const TfgDatosMLP* buffer, const int32_t* idx, int32_t batch,
                                                   int32_t n_in, int32_t n_out, const TfgSceneBounds* bounds,
                                                   float* in, float* tgt, void* stream) {
    if (!buffer || !idx || !bounds || !in || !tgt || batch < 0 || n_in < 15 || n_out < 3)
        return fail(TFG_E_INVALID, "tfgLaunchPrepararDatosEntrenamiento: bad argument");
    if (int rc = device_ok()) return rc;
    if (batch == 0) return ok();
    k_train_rows<<<blocks_for(batch), 256, 0, (cudaStream_t)stream>>>(buffer, idx, batch, n_in, n_out, *bounds, in, tgt);
    return launch_check("tfgLaunchPrepararDatosEntrenamiento");
}

extern "C" int tfgLaunchPrepararDatosInferencia(const TfgDatosMLP* datos, uint32_t n, uint32_t n_in, float* out,
                                                const TfgSceneBounds* bounds, void* stream) {
    if (!datos || !out || !bounds || n_in < 15 || n > 0x7FFFFFFFu)
        return fail(TFG_E_INVALID, "tfgLaunchPrepararDatosInferencia: bad argument");
    if (int rc = device_ok()) return rc;
    if (n == 0) return ok();
    k_infer_rows<<<blocks_for((long)n), 256, 0, (cudaStream_t)stream>>>(datos, n, n_in, out, *bounds);
    return launch_check("tfgLaunchPrepararDatosInferencia");
}

extern "C" int tfgLaunchGuardarSalidaInferencia(const float* net, TfgColor* out, int32_t n, void* stream) {
    if (!net || !out || n < 0) return fail(TFG_E_INVALID, "tfgLaunchGuardarSalidaInferencia: bad argument");
    if (int rc = device_ok()) return rc;
    if (n == 0) return ok();
    k_scrub<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(net, out, n);
    return launch_check("tfgLaunchGuardarSalidaInferencia");
}

extern "C" int tfgLaunchKernelComposite(TfgColor* img, const TfgColor* pred, const TfgColor* thr, int32_t W, int32_t H,
                                        void* stream) {
    if (!img || !pred || !thr || W < 0 || H < 0) return fail(TFG_E_INVALID, "tfgLaunchKernelComposite: bad argument");
    if (int rc = device_ok()) return rc;
    if (W == 0 || H == 0) return ok();
    dim3 blk(16, 16), grd((W + 15) / 16, (H + 15) / 16);
    k_composite<<<grd, blk, 0, (cudaStream_t)stream>>>(img, pred, thr, W, H);
    return launch_check("tfgLaunchKernelComposite");
}

extern "C" int tfgLaunchKernelCalcularTargets(const TfgRegistroEntrenamiento* regs, const TfgColor* tail,
                                              TfgDatosMLP* out, int32_t n, void* stream) {
    if (!regs || !tail || !out || n < 0) return fail(TFG_E_INVALID, "tfgLaunchKernelCalcularTargets: bad argument");
    if (int rc = device_ok()) return rc;
    if (n == 0) return ok();
    k_targets<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(regs, tail, out, n);
    return launch_check("tfgLaunchKernelCalcularTargets");
}

extern "C" int tfgLaunchKernelPrepararInferenciaTail(const TfgRegistroEntrenamiento* regs, TfgDatosMLP* out, int32_t n,
                                                     void* stream) {
    if (!regs || !out || n < 0) return fail(TFG_E_INVALID, "tfgLaunchKernelPrepararInferenciaTail: bad argument");
    if (int rc = device_ok()) return rc;
    if (n == 0) return ok();
    k_tail<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(regs, out, n);
    return launch_check("tfgLaunchKernelPrepararInferenciaTail");
}

extern "C" int tfgLaunchInicializarCamara(TfgCamara* d_camara, int32_t W, int32_t H, void* stream) {
    if (!d_camara || W <= 0 || H <= 0) return fail(TFG_E_INVALID, "tfgLaunchInicializarCamara: bad argument");
    if (int rc = device_ok()) return rc;
    k_default_camera<<<1, 1, 0, (cudaStream_t)stream>>>(d_camara, W, H);
    return launch_check("tfgLaunchInicializarCamara");
}
