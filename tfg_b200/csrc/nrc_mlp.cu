// Neural radiance cache MLP on sm_100a tensor cores: the replacement for the
// reference's ColorMLP over tiny-cuda-nn (mlp.h:19-70, mlp.cpp:22-275).
//
// Network: 15 reference inputs (NrcKernel.cu:18-97 layout: position
// normalised to the scene bounds, view direction and normal mapped to [0,1],
// diffuse and specular albedo) -> 12-band frequency encoding of the position
// (sin, cos of 2^b*pi*p, b = 0..11: 72 features) + the 12 other inputs + a
// constant 1 (first-layer bias) -> 96 features -> 5 hidden layers of 64 ReLU
// -> 3 outputs (no output activation).  FP16 weights and activations with FP32
// accumulation for inference and the training forward pass; BF16 for the
// backward pass (gradients exceed the FP16 range); FP32 master weights, Adam
// and an exponential moving average of the weights (used for inference), as
// the reference's EMA(Adam) configuration (mlp.cpp:61-69).
// Loss: relative L2 on luminance (the reference's RelativeL2Luminance):
// mean over samples and channels of (y_hat - y)^2 / (lum(y_hat)^2 + 0.01), the
// denominator treated as a constant.
//
// Kernels (one CTA = one warpgroup of 128 threads, one thread per sample row
// of a 128-sample tile, TMEM accumulators, SW128 K-major operands in shared
// memory, one elected thread issues tcgen05.mma):
//   k_infer   inputs by bulk (TMA) copy, encode, 6 chained layer GEMMs,
//             output scrub (NrcKernel.cu:99-126) and optionally the
//             composite img += throughput * prediction (RenderKernel.cu:49-66)
//   k_train   gather (NrcKernel.cu:10-68 sample selection), forward, loss
//             gradient, backward through the layers; writes transposed
//             activation / gradient tiles for the weight gradients
//   k_wgrad   dW = dZ^T H per layer, reduced over the batch with tcgen05
//   k_adam    Adam + EMA on FP32 masters, re-packs the three weight images
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tfg_pt.h"
#include "pt_common.cuh"
#include "tfg_errors.h"
#include "tfg_runtime.h"
#include "umma.cuh"

namespace tfg {
namespace mlp {

constexpr int kTile = 128;
constexpr int kHid = 64;
constexpr int kOutPad = 16;
constexpr int kBands = 12;
constexpr int kMaxLayers = 8;    // up to 7 hidden layers

// A network of `nl` layers: 96 -> 64, (nl - 2) x 64 -> 64, 64 -> 16 (3
// outputs used); nl = 4, 6 (the default: 5 hidden layers of 64) or 8.  The
// runtime forms serve the host; kernels use the template forms kRows<NL> etc.
//
// FP32 master parameters, row-major [out][in] per layer with padded shapes
// 64x96, (nl - 2) x 64x64, 16x64 (rows 3..15 of the last layer stay zero).
__host__ __device__ constexpr int rows_of(int nl, int l) { return l == nl - 1 ? 16 : 64; }
__host__ __device__ constexpr int cols_of(int l) { return l == 0 ? 96 : 64; }
__host__ __device__ constexpr int poff_of(int nl, int l) {
    return l == 0 ? 0 : (l <= nl - 1 ? 6144 + (l - 1) * 4096 : 6144 + (nl - 2) * 4096 + 1024);
}
__host__ __device__ constexpr int params_of(int nl) { return poff_of(nl, nl); }
// Forward / inference weight image (FP16 or BF16, SW128 K-major): layer 0 uses
// two K regions (64 rows x 128 B each), hidden layers one region, the last
// layer 16 rows.
__host__ __device__ constexpr int foff_of(int nl, int l) {
    return l == 0 ? 0 : (l <= nl - 1 ? 16384 + (l - 1) * 8192 : 16384 + (nl - 2) * 8192 + 2048);
}
__host__ __device__ constexpr int fwd_bytes_of(int nl) { return foff_of(nl, nl); }
// Backward image (BF16, W^T: [in rows][out K]) for layers 1..nl-1; the last
// layer's K = 16 occupies the first two chunks of each row.
__host__ __device__ constexpr int bwd_bytes_of(int nl) { return (nl - 1) * 8192; }
// FP8 inference image: one SW128 region per layer (K <= 128 bytes per row).
__host__ __device__ constexpr int f8_bytes_of(int nl) { return (nl - 1) * 8192 + 2048; }

template <int NL> __host__ __device__ constexpr int kRows(int l) { return rows_of(NL, l); }
template <int NL> __host__ __device__ constexpr int kCols(int l) { return cols_of(l); }
template <int NL> __host__ __device__ constexpr int kPOff(int l) { return poff_of(NL, l); }
template <int NL> __host__ __device__ constexpr int kFOff(int l) { return foff_of(NL, l); }
template <int NL> __host__ __device__ constexpr int kBOff(int l) { return (l - 1) * 8192; }
template <int NL> __host__ __device__ constexpr int kF8Off(int l) { return l * 8192; }
// Transposed per-tile layouts written by k_train for k_wgrad: feature rows x
// 128 samples, two 64-sample K regions of F*128 bytes.
template <int NL> __host__ __device__ constexpr int kHTFeat(int l) { return l == 0 ? 96 : 64; }        // input of layer l
template <int NL> __host__ __device__ constexpr int kZTFeat(int l) { return l == NL - 1 ? 16 : 64; }   // output gradient
template <int NL> constexpr int kParams = params_of(NL);
template <int NL> constexpr int kFwdBytes = fwd_bytes_of(NL);
template <int NL> constexpr int kBwdBytes = bwd_bytes_of(NL);
template <int NL> constexpr int kF8Bytes = f8_bytes_of(NL);
// Shared-memory layouts are sized for the deepest network.
constexpr int kFwdBytesMax = fwd_bytes_of(kMaxLayers);            // 67584
constexpr int kWeightRegion = (kFwdBytesMax + 1023) / 1024 * 1024;  // 68608
static_assert(fwd_bytes_of(6) == 51200 && bwd_bytes_of(6) == 40960 && params_of(6) == 23552, "default layout");

// The same layouts for hidden width HID (64 or 128; 3, 5 or 7 hidden
// layers): 96 -> HID, (nl - 2) x HID -> HID, HID -> 16.  Weight images keep
// 64-feature (128-byte) SW128 K regions: layer 0 two regions of HID rows,
// hidden layers HID/64 regions of HID rows, the last layer HID/64 regions of
// 16 rows; the backward image W^T of layer l >= 1 has HID rows (input units)
// and HID/64 regions of K (one for the last layer's K = 16).
template <int HID> __host__ __device__ constexpr int rows_h(int nl, int l) { return l == nl - 1 ? 16 : HID; }
template <int HID> __host__ __device__ constexpr int cols_h(int l) { return l == 0 ? 96 : HID; }
// FP8 images: one 128-byte K row per output (K <= 128 features of one byte).
template <int HID> __host__ __device__ constexpr int f8_off_h(int l) { return l * HID * 128; }
template <int HID> __host__ __device__ constexpr int f8_bytes_h(int nl) { return (nl - 1) * HID * 128 + 16 * 128; }
template <int HID> __host__ __device__ constexpr int poff_h(int nl, int l) {
    return l == 0 ? 0 : (l <= nl - 1 ? 96 * HID + (l - 1) * HID * HID : 96 * HID + (nl - 2) * HID * HID + 16 * HID);
}
template <int HID> __host__ __device__ constexpr int params_h(int nl) { return poff_h<HID>(nl, nl); }
template <int HID> __host__ __device__ constexpr int foff_h(int nl, int l) {
    return l == 0 ? 0
                  : (l <= nl - 1 ? 2 * HID * 128 + (l - 1) * (HID / 64) * HID * 128
                                 : 2 * HID * 128 + (nl - 2) * (HID / 64) * HID * 128 + (HID / 64) * 16 * 128);
}
template <int HID> __host__ __device__ constexpr int fwd_bytes_h(int nl) { return foff_h<HID>(nl, nl); }
template <int HID> __host__ __device__ constexpr int boff_h(int, int l) { return (l - 1) * (HID / 64) * HID * 128; }
template <int HID> __host__ __device__ constexpr int bwd_bytes_h(int nl) { return (nl - 2) * (HID / 64) * HID * 128 + HID * 128; }
static_assert(params_h<64>(6) == params_of(6) && fwd_bytes_h<64>(6) == fwd_bytes_of(6) &&
              bwd_bytes_h<64>(6) == bwd_bytes_of(6) && foff_h<64>(6, 5) == foff_of(6, 5) &&
              poff_h<64>(8, 7) == poff_of(8, 7) && boff_h<64>(6, 3) == 2 * 8192, "width 64 keeps its layout");
static_assert(rows_h<64>(6, 2) == rows_of(6, 2) && rows_h<64>(6, 5) == rows_of(6, 5) && cols_h<64>(0) == cols_of(0) &&
                  cols_h<64>(3) == cols_of(3) && f8_off_h<64>(3) == 3 * 8192 && f8_bytes_h<64>(6) == f8_bytes_of(6),
              "width 64 keeps its FP8 layout");
static_assert(params_h<128>(6) == 79872 && fwd_bytes_h<128>(6) == 167936 && bwd_bytes_h<128>(6) == 147456,
              "width 128 layout");
// Runtime forms for the host.
constexpr int params_rt(int nl, int hid) { return hid == 128 ? params_h<128>(nl) : params_h<64>(nl); }
constexpr int rows_rt(int nl, int l, int hid) { return hid == 128 ? rows_h<128>(nl, l) : rows_h<64>(nl, l); }
constexpr int cols_rt(int l, int hid) { return hid == 128 ? cols_h<128>(l) : cols_h<64>(l); }
constexpr int poff_rt(int nl, int l, int hid) { return hid == 128 ? poff_h<128>(nl, l) : poff_h<64>(nl, l); }
constexpr int fwd_bytes_rt(int nl, int hid) { return hid == 128 ? fwd_bytes_h<128>(nl) : fwd_bytes_h<64>(nl); }
constexpr int bwd_bytes_rt(int nl, int hid) { return hid == 128 ? bwd_bytes_h<128>(nl) : bwd_bytes_h<64>(nl); }

// Every wait on a bulk copy or an MMA gives up after this long (a stuck
// wait sets g_mlp_error; the host reports TFG_E_TIMEOUT), far above any
// legitimate wait (microseconds).
constexpr uint64_t kSpinLimit = 1000000000ull;   // 1 s

struct Bounds {
    float lo[3], hi[3];
};

// Device state words of a cache model.
enum : int {
    S_STEP = 0,      // ColorMLP::step_counter (mlp.cpp:103), seed of the sample indices
    S_ADAM_T = 1,    // Adam time step
    S_NAVAIL = 2,    // training records available to this step
    S_GATE = 3,      // open cells of the gate grid after the last gated frame
    S_LOSS_EMA = 4,  // running loss (float bits)
    S_F8_VER = 5,    // S_ADAM_T + 1 of the weights in the FP8 image (0: not packed)
    S_WORDS = 8
};


__device__ int g_mlp_error;   // set when a bounded wait gives up (TFG_E_TIMEOUT)

// ------------------------------------------------------------------ small helpers
__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ uint32_t pack_bf2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ float unit_clamp(float v, float lo, float hi) {   // NrcKernel.cu:5-8
    float n = (v - lo) / (hi - lo);
    return fminf(fmaxf(n, 0.0f), 1.0f);
}

// ------------------------------------------------------------------ composite encoding
// The reference's own cache input (mlp.cpp:22-49, tiny-cuda-nn "Composite"):
// a multiresolution hash grid on the normalised position (Mueller, Evans,
// Schied, Keller 2022: level l has N_l = floor(N_min * b^l) cells per axis,
// trilinear interpolation of 2 features stored at the 8 cell corners; a
// level whose (N_l + 1)^3 corners fit in the table is indexed densely, the
// others by the spatial hash x * 1 ^ y * 2654435761 ^ z * 805459861 mod T),
// one-blob encoding of the view direction and the normal (Mueller et al.
// 2019: k bins per input, each the mass of a Gaussian of sigma 1/k centred at
// the input that falls in the bin) and the albedos as they are.  Feature
// layout of layer 0: 0..2L-1 hash grid (level-major), 32..55 one-blob (6
// inputs x 4 bins), 56..61 albedos, 62 the constant 1, the rest zero.
constexpr int kHashMaxLevels = 16;
constexpr int kBlobBins = 4;
constexpr int kHashLive = 63;     // live input columns of layer 0 with the composite encoding
constexpr int kFreqLive = 85;     // ... with the frequency encoding

struct HashGrid {
    const float2* master;    // FP32 tables [level][T], read by the training forward pass
    const __half2* infer;    // FP16 tables of the debiased weight average, read by inference
    uint32_t T;              // entries per level (a power of two)
    int levels;              // 0: frequency encoding
    uint32_t dense;          // bit l: level l indexed densely
    float res[kHashMaxLevels];
};

// Index of corner (x, y, z) of level l in its table.
__host__ __device__ __forceinline__ uint32_t hash_index(uint32_t x, uint32_t y, uint32_t z, uint32_t n_cells,
                                                        bool dense, uint32_t T) {
    if (dense) {
        const uint32_t st = n_cells + 1u;
        return x + st * (y + st * z);
    }
    return (x ^ (y * 2654435761u) ^ (z * 805459861u)) & (T - 1u);
}

// Cell of position p (in [0, 1]) at level l: integer corner and weights.
__device__ __forceinline__ void hash_cell(const float (&p)[3], float n, uint32_t (&i)[3], float (&f)[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float x = p[k] * n;
        const float c = fminf(floorf(x), n - 1.0f);
        i[k] = (uint32_t)c;
        f[k] = x - c;
    }
}

// Byte offsets, within its level's table, of the x pair (cx, cx + 1) of each
// of a cell's four (y, z) corner rows (row r: y + (r & 1), z + (r >> 1)),
// for entries of E bytes (a power of two).  Scaling by E distributes over the
// hash's XOR and mask (both primes and the mask are pre-scaled, the mask stays
// below 2^32 for T <= 2^24), so each corner costs one logic op.
template <uint32_t E>
__device__ __forceinline__ void level_rows(const uint32_t (&i)[3], uint32_t n_cells, bool dense, uint32_t T,
                                           uint32_t (&o0)[4], uint32_t (&o1)[4]) {
    if (dense) {
        const uint32_t st = n_cells + 1u;
        const uint32_t b = (i[0] + st * (i[1] + st * i[2])) * E, sy = st * E, sz = st * st * E;
        o0[0] = b; o0[1] = b + sy; o0[2] = b + sz; o0[3] = b + sz + sy;
#pragma unroll
        for (int r = 0; r < 4; ++r) o1[r] = o0[r] + E;
    } else {
        constexpr uint32_t P1 = 2654435761u * E, P2 = 805459861u * E;
        const uint32_t m = (T - 1u) * E;
        const uint32_t y0 = i[1] * P1, y1 = y0 + P1, z0 = i[2] * P2, z1 = z0 + P2;
        const uint32_t x0 = i[0] * E, x1 = x0 + E;
        const uint32_t yz[4] = {y0 ^ z0, y1 ^ z0, y0 ^ z1, y1 ^ z1};
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            o0[r] = (x0 ^ yz[r]) & m;
            o1[r] = (x1 ^ yz[r]) & m;
        }
    }
}

// The 2L hash-grid features of position p from the FP32 tables (the training
// forward pass).  A level's trilinear sum runs over its four (y, z) corner
// rows: each row's x pair is blended with the x weights, then the row with
// its (y, z) weight.
__device__ __forceinline__ void hash_features(const float (&p)[3], const HashGrid& g, float (&h)[2 * kHashMaxLevels]) {
#pragma unroll
    for (int l = 0; l < kHashMaxLevels; ++l) {
        h[2 * l] = 0.0f;
        h[2 * l + 1] = 0.0f;
        if (l >= g.levels) continue;
        const float n = g.res[l];
        uint32_t i[3], o0[4], o1[4];
        float f[3];
        hash_cell(p, n, i, f);
        level_rows<8>(i, (uint32_t)n, (g.dense >> l) & 1u, g.T, o0, o1);
        const char* lvl = reinterpret_cast<const char*>(g.master + (size_t)l * g.T);
        const float wx0 = 1.0f - f[0], wy0 = 1.0f - f[1], wz0 = 1.0f - f[2];
        float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float2 v0 = __ldg(reinterpret_cast<const float2*>(lvl + o0[r]));
            const float2 v1 = __ldg(reinterpret_cast<const float2*>(lvl + o1[r]));
            const float wyz = ((r & 1) ? f[1] : wy0) * ((r & 2) ? f[2] : wz0);
            a0 = fmaf(wyz, fmaf(f[0], v1.x, wx0 * v0.x), a0);
            a1 = fmaf(wyz, fmaf(f[0], v1.y, wx0 * v0.y), a1);
        }
        h[2 * l] = a0;
        h[2 * l + 1] = a1;
    }
}

// The same features from the FP16 image of the averaged tables (inference),
// interpolated in FP16 pair arithmetic: word l holds level l's two features,
// in the FP16 operand format layer 0 reads.  Levels go in pairs whose 16
// corner loads are all issued before either level is combined, so a thread
// keeps twice the gathers in flight.
constexpr int kHashLevelBatch = 2;

__device__ __forceinline__ void hash_words_f16(const float (&p)[3], const HashGrid& g, __half2 (&h)[kHashMaxLevels]) {
#pragma unroll
    for (int l0 = 0; l0 < kHashMaxLevels; l0 += kHashLevelBatch) {
        __half2 v[kHashLevelBatch][8];
        float f[kHashLevelBatch][3];
#pragma unroll
        for (int b = 0; b < kHashLevelBatch; ++b) {
            const int l = l0 + b;
            if (l >= g.levels) continue;
            const float n = g.res[l];
            uint32_t i[3], o0[4], o1[4];
            hash_cell(p, n, i, f[b]);
            level_rows<4>(i, (uint32_t)n, (g.dense >> l) & 1u, g.T, o0, o1);
            const char* lvl = reinterpret_cast<const char*>(g.infer + (size_t)l * g.T);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                v[b][2 * r] = __ldg(reinterpret_cast<const __half2*>(lvl + o0[r]));
                v[b][2 * r + 1] = __ldg(reinterpret_cast<const __half2*>(lvl + o1[r]));
            }
        }
#pragma unroll
        for (int b = 0; b < kHashLevelBatch; ++b) {
            const int l = l0 + b;
            h[l] = __float2half2_rn(0.0f);
            if (l >= g.levels) continue;
            const __half2 hx0 = __float2half2_rn(1.0f - f[b][0]), hx1 = __float2half2_rn(f[b][0]);
            const float wy0 = 1.0f - f[b][1], wz0 = 1.0f - f[b][2];
            __half2 acc = __float2half2_rn(0.0f);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const __half2 wyz = __float2half2_rn(((r & 1) ? f[b][1] : wy0) * ((r & 2) ? f[b][2] : wz0));
                acc = __hfma2(wyz, __hfma2(hx1, v[b][2 * r + 1], __hmul2(hx0, v[b][2 * r])), acc);
            }
            h[l] = acc;
        }
    }
}

// Standard normal CDF by Abramowitz & Stegun, Handbook of Mathematical
// Functions, formula 26.2.17 (Hastings' rational approximation, absolute
// error below 7.5e-8): Phi(x) = 1 - phi(x) (b1 t + ... + b5 t^5) with
// t = 1 / (1 + p |x|) for x >= 0, and Phi(x) = 1 - Phi(-x).  About half
// the instructions of the library's normcdff; the one-blob bins are its only
// user.
__device__ __forceinline__ float std_normal_cdf(float x) {
    const float ax = fabsf(x);
    const float t = __fdividef(1.0f, fmaf(0.2316419f, ax, 1.0f));
    float poly = fmaf(t, 1.330274429f, -1.821255978f);
    poly = fmaf(t, poly, 1.781477937f);
    poly = fmaf(t, poly, -0.356563782f);
    poly = fmaf(t, poly, 0.319381530f);
    poly *= t;
    const float tail = 0.3989422804f * __expf(-0.5f * ax * ax) * poly;   // phi(|x|) * poly
    return x >= 0.0f ? 1.0f - tail : tail;
}

// One-blob bins of an input in [0, 1]: Phi((b+1)/k - s; 1/k) - Phi(b/k - s; 1/k).
__device__ __forceinline__ void one_blob(float s, float (&o)[kBlobBins]) {
    float prev = std_normal_cdf((0.0f - s) * (float)kBlobBins);
#pragma unroll
    for (int b = 0; b < kBlobBins; ++b) {
        const float next = std_normal_cdf(((float)(b + 1) / (float)kBlobBins - s) * (float)kBlobBins);
        o[b] = next - prev;
        prev = next;
    }
}

// Features 32..63 of layer 0 with the composite encoding: one-blob bins of
// direction and normal, the albedos, the constant 1 and a zero.
__device__ __forceinline__ void composite_tail(const TfgDatosMLP& d, float (&x)[32]) {
    const float dirn[6] = {(float)d.direccion.x, (float)d.direccion.y, (float)d.direccion.z,
                           (float)d.normal.x,    (float)d.normal.y,    (float)d.normal.z};
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        float o[kBlobBins];
        one_blob(dirn[j], o);
#pragma unroll
        for (int k = 0; k < kBlobBins; ++k) x[kBlobBins * j + k] = o[k];
    }
    x[24] = d.difuso.r; x[25] = d.difuso.g; x[26] = d.difuso.b;
    x[27] = d.especular.r; x[28] = d.especular.g; x[29] = d.especular.b;
    x[30] = 1.0f;
    x[31] = 0.0f;
}

__device__ __forceinline__ void unit_position(const TfgDatosMLP& d, const Bounds& b, float (&p)[3]) {
    p[0] = unit_clamp((float)d.posicion.x, b.lo[0], b.hi[0]);
    p[1] = unit_clamp((float)d.posicion.y, b.lo[1], b.hi[1]);
    p[2] = unit_clamp((float)d.posicion.z, b.lo[2], b.hi[2]);
}

// The 64 features of layer 0 with the composite encoding (63 live + one zero)
// from the FP32 tables (training forward pass).
__device__ __forceinline__ void composite_features(const TfgDatosMLP& d, const Bounds& b, const HashGrid& g,
                                                   float (&x)[64]) {
    float p[3];
    unit_position(d, b, p);
    float h[2 * kHashMaxLevels], t[32];
    hash_features(p, g, h);
    composite_tail(d, t);
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        x[k] = h[k];
        x[32 + k] = t[k];
    }
}

// Encoded features of one training sample, packed as 48 FP16 pairs (96
// features); the composite encoding reads the FP32 tables.
__device__ __forceinline__ void encode(const TfgDatosMLP& d, const Bounds& b, const HashGrid& g, uint32_t (&w)[48]) {
    if (g.levels > 0) {
        float x[64];
        composite_features(d, b, g, x);
#pragma unroll
        for (int k = 0; k < 32; ++k) w[k] = pack_h2(x[2 * k], x[2 * k + 1]);
#pragma unroll
        for (int k = 32; k < 48; ++k) w[k] = 0u;
        return;
    }
    const float p[3] = {unit_clamp((float)d.posicion.x, b.lo[0], b.hi[0]),
                        unit_clamp((float)d.posicion.y, b.lo[1], b.hi[1]),
                        unit_clamp((float)d.posicion.z, b.lo[2], b.hi[2])};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        float s, c;
        sincospif(p[j], &s, &c);
#pragma unroll
        for (int k = 0; k < kBands; ++k) {
            w[12 * j + k] = pack_h2(s, c);
            const float s2 = 2.0f * s * c;
            const float c2 = (c - s) * (c + s);
            s = s2;
            c = c2;
        }
    }
    w[36] = pack_h2((float)d.direccion.x, (float)d.direccion.y);
    w[37] = pack_h2((float)d.direccion.z, (float)d.normal.x);
    w[38] = pack_h2((float)d.normal.y, (float)d.normal.z);
    w[39] = pack_h2(d.difuso.r, d.difuso.g);
    w[40] = pack_h2(d.difuso.b, d.especular.r);
    w[41] = pack_h2(d.especular.g, d.especular.b);
    w[42] = pack_h2(1.0f, 0.0f);
#pragma unroll
    for (int k = 43; k < 48; ++k) w[k] = 0u;
}

// Store the 96 encoded features of row r into the two-region A buffer.
__device__ __forceinline__ void store_encoded(uint8_t* a0, int r, const uint32_t (&w)[48]) {
#pragma unroll
    for (int c = 0; c < 12; ++c) {
        uint8_t* region = a0 + (c >> 3) * (kTile * 128);
        *reinterpret_cast<uint4*>(region + umma::sw128_offset(r, c & 7)) =
            make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
    }
}

// Store 64 values of row r (ReLU'd by the caller) as FP16 or BF16.
template <bool BF16>
__device__ __forceinline__ void store_row64(uint8_t* a, int r, const float (&v)[64]) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint32_t q[4];
#pragma unroll
        for (int e = 0; e < 4; ++e)
            q[e] = BF16 ? pack_bf2(v[8 * c + 2 * e], v[8 * c + 2 * e + 1]) : pack_h2(v[8 * c + 2 * e], v[8 * c + 2 * e + 1]);
        *reinterpret_cast<uint4*>(a + umma::sw128_offset(r, c)) = make_uint4(q[0], q[1], q[2], q[3]);
    }
}

__device__ __forceinline__ void tmem_row64(uint32_t tmem, int warp, int col0, float (&v)[64]) {
    float a[32], b[32];
    const uint32_t base = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)col0;
    umma::tmem_ld32(base, a);
    umma::tmem_ld32(base + 32, b);
#pragma unroll
    for (int i = 0; i < 32; ++i) { v[i] = a[i]; v[32 + i] = b[i]; }
}

// Issue the MMAs of one layer: D[128 x N] = A[128 x K] * W^T, K in 16-steps.
__device__ __forceinline__ void issue_layer(uint32_t d_tmem, const uint8_t* a, int a_region_bytes, const uint8_t* w,
                                            int w_region_bytes, int K, int N, bool bf16) {
    const uint32_t id = umma::idesc_f16(kTile, N, bf16);
    const int steps = K / 16;
    for (int s = 0; s < steps; ++s) {
        const int reg = s >> 2, kk = s & 3;
        const uint64_t ad = umma::sdesc_sw128(umma::smem_u32(a + reg * a_region_bytes + kk * 32));
        const uint64_t bd = umma::sdesc_sw128(umma::smem_u32(w + reg * w_region_bytes + kk * 32));
        umma::mma_f16(d_tmem, ad, bd, id, s > 0);
    }
}

// Scrub a prediction as guardarSalidaInferencia (NrcKernel.cu:99-126).
__device__ __forceinline__ float scrub(float c) {
    if (c < 0.0f) c = 0.0f;
    if (isnan(c)) c = 0.0f;
    if (c > 100000.0f) c = 100000.0f;
    if (isinf(c)) c = 100000.0f;
    return c;
}

__device__ __forceinline__ bool all_ok(bool ok) { return __syncthreads_and(ok ? 1 : 0) != 0; }

// ------------------------------------------------------------------ inference
// Persistent kernel, one CTA per SM.  The CTA runs kSlots tiles of 128
// queries at a time; each tile ("slot") is one warpgroup with its own 128
// TMEM columns (64 FP32 accumulator columns, then the A operand of the next
// layer), its own input staging buffer, MMA mbarrier and named barrier;
// thread t owns row t (TMEM lane t).  Only the weights (bulk-copied once) and
// the staged inputs live in shared memory: the tensor pipe reads B from
// shared memory and A from TMEM.  Per layer: MMAs (issued from a converged
// warp through elect.sync) -> commit -> TMEM load -> scale / ReLU / pack ->
// TMEM store of the next A operand -> barrier.
//
// Precisions (template PREC): FP16 and BF16 operands (kind::f16, K = 16 per
// MMA, two features per TMEM column) or FP8 E4M3 with per-layer scales
// (kind::f8f6f4, K = 32 per MMA, four features per column): inputs of layer
// l are quantised as x * q[l] (q = 448 / (2 * amax of the layer's input)),
// weights as w * wq[l] (wq = 448 / amax|W_l|), and the accumulator is
// rescaled by 1 / (q[l] * wq[l]).  All accumulate in FP32.
enum : int { kPrecF16 = 0, kPrecBF16 = 1, kPrecF8 = 2 };
constexpr int kSlots = 4;
constexpr int kInferThreads = 128 * kSlots;
constexpr int kRowBytes = (int)sizeof(TfgDatosMLP);              // 112
constexpr int kStageBytes = kTile * kRowBytes;                   // 14336
constexpr int kInferSmemStage = kWeightRegion;
constexpr int kInferSmem = kInferSmemStage + kSlots * kStageBytes;
static_assert(kSlots * 128 <= 512, "TMEM: 128 columns per slot");
static_assert(kInferSmem + 1024 <= 227 * 1024, "inference shared memory");
// Scale words of the FP8 path (device floats): q[l], wq[l] and the running
// amax of each layer's input observed by the last inference calls.
constexpr int kF8Q = 0, kF8WQ = 8, kF8Amax = 16, kF8Words = 24;
constexpr float kF8Max = 448.0f;

__device__ __forceinline__ void slot_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// AND of `p` over the slot's 128 threads (all of them get the result).
__device__ __forceinline__ bool slot_all(int id, bool p) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred pi, po;\n\t"
        "setp.ne.u32 pi, %1, 0;\n\t"
        "bar.red.and.pred po, %2, 128, pi;\n\t"
        "selp.u32 %0, 1, 0, po;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(id)
        : "memory");
    return r != 0;
}

// max(x, 0) of two floats packed as FP16x2 / BF16x2 (ReLU fused into the
// conversion); lo in the low half.
__device__ __forceinline__ uint32_t relu_h2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ uint32_t relu_bf2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
// Four floats as E4M3 (round to nearest, saturating), element a in the lowest
// byte; the RELU form clamps negatives to zero.
template <bool RELU>
__device__ __forceinline__ uint32_t pack_e4m3x4(float a, float b, float c, float d) {
    uint16_t lo, hi;
    if (RELU) {
        asm("cvt.rn.satfinite.relu.e4m3x2.f32 %0, %1, %2;" : "=h"(lo) : "f"(b), "f"(a));
        asm("cvt.rn.satfinite.relu.e4m3x2.f32 %0, %1, %2;" : "=h"(hi) : "f"(d), "f"(c));
    } else {
        asm("cvt.rn.satfinite.e4m3x2.f32 %0, %1, %2;" : "=h"(lo) : "f"(b), "f"(a));
        asm("cvt.rn.satfinite.e4m3x2.f32 %0, %1, %2;" : "=h"(hi) : "f"(d), "f"(c));
    }
    return (uint32_t)lo | ((uint32_t)hi << 16);
}
// Two lanes of an IEEE round-to-nearest multiply in one packed instruction
// (sm_100 f32x2): each lane equals the scalar product exactly.
__device__ __forceinline__ void mul2(float& a, float& b, float s) {
    uint64_t x, y;
    asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "f"(a), "f"(b));
    asm("mov.b64 %0, {%1, %1};" : "=l"(y) : "f"(s));
    asm("mul.rn.f32x2 %0, %0, %1;" : "+l"(x) : "l"(y));
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x));
}
// Four accumulator values scaled by s, then ReLU and E4M3 as pack_e4m3x4.
__device__ __forceinline__ uint32_t scale_relu_e4m3x4(float a, float b, float c, float d, float s) {
    mul2(a, b, s);
    mul2(c, d, s);
    return pack_e4m3x4<true>(a, b, c, d);
}

template <int PREC>
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    return PREC == kPrecBF16 ? pack_bf2(a, b) : pack_h2(a, b);
}

// Packed words of the composite encoding: the hash-grid pairs (FP16 from
// the interpolation, or re-rounded to BF16), then the one-blob / albedo tail.
template <int PREC>
__device__ __forceinline__ void composite_words(const __half2 (&hw)[kHashMaxLevels], const float (&t)[32],
                                                uint32_t (&w)[48]) {
#pragma unroll
    for (int k = 0; k < kHashMaxLevels; ++k) {
        if constexpr (PREC == kPrecBF16) {
            const float2 v = __half22float2(hw[k]);
            w[k] = pack_bf2(v.x, v.y);
        } else {
            w[k] = *reinterpret_cast<const uint32_t*>(&hw[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) w[16 + k] = pack2<PREC>(t[2 * k], t[2 * k + 1]);
#pragma unroll
    for (int k = 32; k < 48; ++k) w[k] = 0u;
}

// Packed words of the frequency encoding of the unit position p and the 13
// other inputs (direction, normal, albedos, the constant 1).
template <int PREC>
__device__ __forceinline__ void frequency_words(const float (&p)[3], const float (&misc)[13], uint32_t (&w)[48]) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        float s, c;
        __sincosf(kPiF * p[j], &s, &c);
#pragma unroll
        for (int k = 0; k < kBands; ++k) {
            w[12 * j + k] = pack2<PREC>(s, c);
            const float s2 = 2.0f * s * c;
            const float c2 = (c - s) * (c + s);
            s = s2;
            c = c2;
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) w[36 + k] = pack2<PREC>(misc[2 * k], misc[2 * k + 1]);
    w[42] = pack2<PREC>(1.0f, 0.0f);
#pragma unroll
    for (int k = 43; k < 48; ++k) w[k] = 0u;
}

// Encoded features of one staged row as 96 floats' worth of packed words:
// features 0..71 are (sin, cos)(2^k pi p) of the x, y, z bands (double-angle
// recurrence from a hardware sin/cos of the base band), 72..84 direction,
// normal, albedos and the constant 1, 85..95 zero.  FP16 / BF16 write 48 TMEM
// columns (two features each), FP8 24 columns (four each, scaled by q0).
// Returns the largest |feature| of 72..84 (the bands are within [-1, 1]).
template <int PREC, bool HASH>
__device__ __forceinline__ float encode_to_tmem(const TfgDatosMLP* r, const Bounds& b, const HashGrid& g, float q0,
                                                uint32_t ta) {
    if constexpr (HASH) {
        // composite encoding: the hash-grid pairs straight from the FP16
        // interpolation, then the one-blob / albedo features; the largest
        // |feature| for the FP8 scale
        float p[3];
        unit_position(*r, b, p);
        __half2 hw[kHashMaxLevels];
        hash_words_f16(p, g, hw);
        float t[32];
        composite_tail(*r, t);
        float x[32];
#pragma unroll
        for (int k = 0; k < kHashMaxLevels; ++k) {
            const float2 v = __half22float2(hw[k]);
            x[2 * k] = v.x;
            x[2 * k + 1] = v.y;
        }
        float amax = 1.0f;
#pragma unroll
        for (int k = 0; k < 32; ++k) amax = fmaxf(amax, fabsf(x[k]));
#pragma unroll
        for (int k = 0; k < 30; ++k) amax = fmaxf(amax, fabsf(t[k]));
        if constexpr (PREC == kPrecF8) {
            uint32_t w[24];
#pragma unroll
            for (int k = 0; k < 8; ++k)
                w[k] = pack_e4m3x4<false>(x[4 * k] * q0, x[4 * k + 1] * q0, x[4 * k + 2] * q0, x[4 * k + 3] * q0);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                w[8 + k] = pack_e4m3x4<false>(t[4 * k] * q0, t[4 * k + 1] * q0, t[4 * k + 2] * q0, t[4 * k + 3] * q0);
#pragma unroll
            for (int k = 16; k < 24; ++k) w[k] = 0u;
            umma::tmem_st16(ta, *reinterpret_cast<const uint32_t(*)[16]>(w));
            umma::tmem_st8(ta + 16u, w + 16);
        } else {
            uint32_t w[48];
            composite_words<PREC>(hw, t, w);
#pragma unroll
            for (int c = 0; c < 3; ++c)
                umma::tmem_st16(ta + 16u * c, *reinterpret_cast<const uint32_t(*)[16]>(w + 16 * c));
        }
        return amax;
    } else {
    const float misc[13] = {(float)r->direccion.x, (float)r->direccion.y, (float)r->direccion.z,
                            (float)r->normal.x,    (float)r->normal.y,    (float)r->normal.z,
                            r->difuso.r,           r->difuso.g,           r->difuso.b,
                            r->especular.r,        r->especular.g,        r->especular.b, 1.0f};
    float amax = 1.0f;
#pragma unroll
    for (int k = 0; k < 12; ++k) amax = fmaxf(amax, fabsf(misc[k]));
    const float p[3] = {unit_clamp((float)r->posicion.x, b.lo[0], b.hi[0]),
                        unit_clamp((float)r->posicion.y, b.lo[1], b.hi[1]),
                        unit_clamp((float)r->posicion.z, b.lo[2], b.hi[2])};
    if constexpr (PREC == kPrecF8) {
        uint32_t w[24];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float s, c;
            __sincosf(kPiF * p[j], &s, &c);
#pragma unroll
            for (int k = 0; k < kBands; k += 2) {
                const float s1 = 2.0f * s * c, c1 = (c - s) * (c + s);
                w[6 * j + k / 2] = pack_e4m3x4<false>(s * q0, c * q0, s1 * q0, c1 * q0);
                s = 2.0f * s1 * c1;
                c = (c1 - s1) * (c1 + s1);
            }
        }
        w[18] = pack_e4m3x4<false>(misc[0] * q0, misc[1] * q0, misc[2] * q0, misc[3] * q0);
        w[19] = pack_e4m3x4<false>(misc[4] * q0, misc[5] * q0, misc[6] * q0, misc[7] * q0);
        w[20] = pack_e4m3x4<false>(misc[8] * q0, misc[9] * q0, misc[10] * q0, misc[11] * q0);
        w[21] = pack_e4m3x4<false>(q0, 0.0f, 0.0f, 0.0f);
        w[22] = 0u;
        w[23] = 0u;
        umma::tmem_st16(ta, *reinterpret_cast<const uint32_t(*)[16]>(w));
        umma::tmem_st8(ta + 16u, w + 16);
    } else {
        uint32_t w[48];
        frequency_words<PREC>(p, misc, w);
#pragma unroll
        for (int c = 0; c < 3; ++c) umma::tmem_st16(ta + 16u * c, *reinterpret_cast<const uint32_t(*)[16]>(w + 16 * c));
    }
    return amax;
    }
}

// The 48 packed FP16 / BF16 words of one query row (both encodings), for
// kernels whose layer-0 operand lives in shared memory; returns the largest
// |feature| as encode_to_tmem does.
template <int PREC, bool HASH>
__device__ __forceinline__ float encode_words(const TfgDatosMLP& d, const Bounds& b, const HashGrid& g,
                                              uint32_t (&w)[48]) {
    float p[3];
    unit_position(d, b, p);
    float amax = 1.0f;
    if constexpr (HASH) {
        __half2 hw[kHashMaxLevels];
        hash_words_f16(p, g, hw);
        float t[32];
        composite_tail(d, t);
        composite_words<PREC>(hw, t, w);
#pragma unroll
        for (int k = 0; k < kHashMaxLevels; ++k) {
            const float2 v = __half22float2(hw[k]);
            amax = fmaxf(amax, fmaxf(fabsf(v.x), fabsf(v.y)));
        }
#pragma unroll
        for (int k = 0; k < 30; ++k) amax = fmaxf(amax, fabsf(t[k]));
    } else {
        const float misc[13] = {(float)d.direccion.x, (float)d.direccion.y, (float)d.direccion.z,
                                (float)d.normal.x,    (float)d.normal.y,    (float)d.normal.z,
                                d.difuso.r,           d.difuso.g,           d.difuso.b,
                                d.especular.r,        d.especular.g,        d.especular.b, 1.0f};
        frequency_words<PREC>(p, misc, w);
#pragma unroll
        for (int k = 0; k < 12; ++k) amax = fmaxf(amax, fabsf(misc[k]));
    }
    return amax;
}

// Largest value over the warp, folded into *dst (values are >= 0, so their
// bit patterns order like the floats).
__device__ __forceinline__ void warp_amax(float v, float* dst) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.0f) atomicMax(reinterpret_cast<int*>(dst), __float_as_int(v));
}

// `f8` (FP8 only): scale words.  TRACK: the per-layer input amax is folded
// into amax[0..5]; with `amax_all` every tile contributes, otherwise only the
// first tile of each slot (the delayed-scaling estimate).
template <int PREC, bool TRACK, int NL, bool HASH>
__global__ void __launch_bounds__(kInferThreads, 1) k_infer(const TfgDatosMLP* __restrict__ in, uint32_t n_max,
                                                            const uint32_t* __restrict__ n_dev, Bounds bounds,
                                                            HashGrid hg,
                                                            const uint8_t* __restrict__ wimg,
                                                            TfgColor* __restrict__ out, TfgColor* __restrict__ img,
                                                            const TfgColor* __restrict__ thr,
                                                            const float* __restrict__ f8, float* amax, int amax_all) {
    constexpr bool kF8 = PREC == kPrecF8;
    constexpr uint32_t kWBytes = kF8 ? kF8Bytes<NL> : kFwdBytes<NL>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sw = smem;
    __shared__ uint64_t mb_w, mb_mma[kSlots], mb_in[kSlots], mb_drain[kSlots];
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, q = warp & 3, t = tid & 127;
    const int slot = tid / 128;
    const bool leader = t == 0;
    const bool issuer_warp = t < 32;                               // first warp of the slot issues its MMAs
    const int bar = 1 + slot;
    uint8_t* stage = smem + kInferSmemStage + slot * kStageBytes;
    const uint32_t n = n_dev ? min(*n_dev, n_max) : n_max;
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    if (blockIdx.x * kSlots >= ntiles) return;
    // FP8 scales: input quantisation of each layer and the accumulator rescale.
    float qs[NL], deq[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        qs[l] = kF8 ? f8[kF8Q + l] : 1.0f;
        deq[l] = kF8 ? 1.0f / (f8[kF8Q + l] * f8[kF8WQ + l]) : 1.0f;
    }
    if (warp == 0) umma::tmem_alloc(&tslot, 512);
    if (tid == 0) {
        umma::mbar_init(&mb_w, 1);
        for (int k = 0; k < kSlots; ++k) {
            umma::mbar_init(&mb_mma[k], 1);
            umma::mbar_init(&mb_in[k], 1);
            umma::mbar_init(&mb_drain[k], 1);
        }
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tlane = (uint32_t)(32 * q) << 16;
    const uint32_t tmem = tslot + 128u * (uint32_t)slot;          // accumulator: columns 0..63 of the slot
    const uint32_t tmem_a = tmem + 64u;                            // A operand: columns 64..111
    const uint32_t tstride = gridDim.x * kSlots;
    const uint64_t wdesc = umma::sdesc_sw128(umma::smem_u32(sw));
    // Bulk copy of tile `tl`'s rows (a multiple of 16 bytes from a 16-byte
    // aligned source) into the slot's staging buffer.
    auto fetch = [&](uint32_t tl) {
        const uint32_t rows = min((uint32_t)kTile, n - tl * kTile);
        umma::mbar_expect_tx(&mb_in[slot], rows * kRowBytes);
        umma::bulk_g2s(stage, reinterpret_cast<const uint8_t*>(in) + (size_t)tl * kStageBytes, rows * kRowBytes,
                       &mb_in[slot]);
    };
    if (tid == 0) {
        umma::mbar_expect_tx(&mb_w, kWBytes);
        umma::bulk_g2s(sw, wimg, kWBytes, &mb_w);
    }
    uint32_t tile = blockIdx.x * kSlots + slot;
    bool pending = tile < ntiles;
    if (pending && leader) fetch(tile);
    bool ok = umma::mbar_wait(&mb_w, 0, kSpinLimit);
    ok = __syncthreads_and(ok ? 1 : 0) != 0;
    uint32_t mph = 0, iph = 0;
    bool first = true;
    for (; tile < ntiles && ok; tile += tstride, first = false) {
        const uint32_t row = tile * kTile + (uint32_t)t;
        const bool valid = row < n;
        const bool track = TRACK && (amax_all || first);
        ok = slot_all(bar, umma::mbar_wait(&mb_in[slot], iph, kSpinLimit));
        if (!ok) break;
        pending = false;
        iph ^= 1u;
        // rows past the end of a partial tile encode stale staging bytes; the
        // rows of the MLP are independent and those outputs are never stored
        const float a0 = encode_to_tmem<PREC, HASH>(reinterpret_cast<const TfgDatosMLP*>(stage + t * kRowBytes), bounds, hg,
                                              qs[0], tmem_a + tlane);
        if (track) warp_amax(valid ? a0 : 0.0f, &amax[0]);
        umma::tmem_wait_st();
        umma::fence_before_sync();
        slot_sync(bar);   // staging buffer consumed, A operand of layer 0 in TMEM
        if (tile + tstride < ntiles) {
            if (leader) {
                umma::fence_smem_to_async();
                fetch(tile + tstride);
            }
            pending = true;
        }
        // Fully unrolled: every descriptor is the weights' base descriptor plus
        // an immediate (the start-address field holds address / 16), so the
        // issuing thread runs no descriptor arithmetic between MMAs.
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            const bool last = l == NL - 1;
            if (issuer_warp) {
                umma::fence_after_sync();
                constexpr uint32_t id_hid = umma::idesc_f16(kTile, kHid, PREC == kPrecBF16);
                constexpr uint32_t id_out = umma::idesc_f16(kTile, kOutPad, PREC == kPrecBF16);
                if (umma::elect_one()) {
                    if constexpr (kF8) {
#pragma unroll
                        for (int s = 0; s < kCols<NL>(l) / 32; ++s)
                            umma::mma_f8_ta(tmem, tmem_a + 8u * s, wdesc + (uint64_t)((kF8Off<NL>(l) + s * 32) >> 4),
                                            last ? id_out : id_hid, s > 0);
                    } else {
#pragma unroll
                        for (int s = 0; s < kCols<NL>(l) / 16; ++s) {
                            const uint64_t bd =
                                wdesc + (uint64_t)((kFOff<NL>(l) + (s >> 2) * (kRows<NL>(l) * 128) + (s & 3) * 32) >> 4);
                            umma::mma_f16_ta(tmem, tmem_a + 8u * s, bd, last ? id_out : id_hid, s > 0);
                        }
                    }
                    umma::mma_commit(&mb_mma[slot]);
                }
                __syncwarp();
            }
            ok = slot_all(bar, umma::mbar_wait(&mb_mma[slot], mph, kSpinLimit));
            mph ^= 1u;
            if (!ok) break;
            umma::fence_after_sync();
            if (!last) {
                float lmax = 0.0f;   // max of the raw accumulator; x deq[l] > 0 keeps the order
                // FP8 keeps the column chunks rolled: unrolled, with the amax
                // tracking, the kernel outgrows the instruction cache
#pragma unroll(kF8 ? 1 : 2)
                for (int h = 0; h < 2; ++h) {
                    float v[32];
                    umma::tmem_ld32(tmem + tlane + 32u * h, v);
                    if constexpr (kF8) {
                        // dequantise, ReLU, requantise for the next layer
                        const float sc = deq[l] * qs[l + 1];
                        uint32_t r[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i)
                            r[i] = scale_relu_e4m3x4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3], sc);
                        umma::tmem_st8(tmem_a + tlane + 8u * h, r);
                        if (track) {
#pragma unroll
                            for (int i = 0; i < 32; ++i) lmax = fmaxf(lmax, v[i]);
                        }
                    } else {
                        uint32_t r[16];
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                            r[i] = PREC == kPrecBF16 ? relu_bf2(v[2 * i], v[2 * i + 1]) : relu_h2(v[2 * i], v[2 * i + 1]);
                        umma::tmem_st16(tmem_a + tlane + 16u * h, r);
                        if (track) {
#pragma unroll
                            for (int i = 0; i < 32; ++i) lmax = fmaxf(lmax, v[i]);
                        }
                    }
                }
                if (track) warp_amax(valid ? lmax * deq[l] : 0.0f, &amax[l + 1]);
                umma::tmem_wait_st();
                umma::fence_before_sync();
                slot_sync(bar);
            } else {
                float v[16];
                umma::tmem_ld16(tmem + tlane, v);
                if (valid && (out || img)) {
                    const float cr = scrub(v[0] * deq[l]), cg = scrub(v[1] * deq[l]), cb = scrub(v[2] * deq[l]);
                    if (img) {
                        const TfgColor th = thr[row];
                        if (th.r > 0 || th.g > 0 || th.b > 0) {
                            TfgColor f = img[row];
                            f.r = f.r + th.r * cr;
                            f.g = f.g + th.g * cg;
                            f.b = f.b + th.b * cb;
                            img[row] = f;
                        }
                    } else {
                        out[row] = TfgColor{cr, cg, cb};
                    }
                }
                umma::fence_before_sync();
                slot_sync(bar);   // accumulator read before the next tile's first MMA
            }
        }
    }
    if (pending) umma::mbar_wait(&mb_in[slot], iph, kSpinLimit);   // no copy may land after exit
    if (!ok && issuer_warp) {   // after a timeout: every MMA this slot issued must finish before TMEM is freed
        if (umma::elect_one()) {
            umma::mma_commit(&mb_drain[slot]);
            umma::mbar_wait(&mb_drain[slot], 0, kSpinLimit);
        }
        __syncwarp();
    }
    if (!ok && leader) atomicExch(&g_mlp_error, 1);
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tslot, 512);
}

// Width-128 inference (3 or 5 hidden layers, whose weights stay resident in
// shared memory; 7 layers use k_infer128s; FP16 or BF16): the same
// pipeline as k_infer with two 128-query slots per SM, each with 256 TMEM
// columns (128 FP32 accumulator columns, then up to 64 columns of the next
// layer's A operand), and the 164 KB weight image in shared memory.
constexpr int kSlots128 = 2;
constexpr int kInfer128Threads = 128 * kSlots128;
constexpr int kInfer128Stage = fwd_bytes_h<128>(6);                       // 167936, 1024-aligned
constexpr int kInfer128Smem = kInfer128Stage + kSlots128 * kStageBytes;   // 196608
static_assert(kInfer128Stage % 1024 == 0 && kInfer128Smem + 1024 <= 227 * 1024, "width-128 inference shared memory");

// FP8 (E4M3, kind::f8f6f4, four features per TMEM column) and amax tracking
// follow k_infer: `f8` holds the per-layer input and weight scales, TRACK
// folds each layer's input amax into amax[] (every tile with `amax_all`,
// otherwise the first tile of each slot).
template <int PREC, bool TRACK, int NL, bool HASH>
__global__ void __launch_bounds__(kInfer128Threads, 1)
    k_infer128(const TfgDatosMLP* __restrict__ in, uint32_t n_max, const uint32_t* __restrict__ n_dev, Bounds bounds,
               HashGrid hg, const uint8_t* __restrict__ wimg, TfgColor* __restrict__ out, TfgColor* __restrict__ img,
               const TfgColor* __restrict__ thr, const float* __restrict__ f8, float* amax, int amax_all) {
    constexpr bool kF8 = PREC == kPrecF8;
    static_assert(NL == 4 || NL == 6 || (kF8 && NL == 8),
                  "width 128 with resident weights: 3 or 5 hidden layers (7 in FP8, whose image fits)");
    constexpr uint32_t kWBytes = kF8 ? f8_bytes_h<128>(NL) : fwd_bytes_h<128>(NL);
    static_assert(kWBytes <= kInfer128Stage, "weights fit before the staging buffers");
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sw = smem;
    __shared__ uint64_t mb_w, mb_mma[kSlots128], mb_in[kSlots128], mb_drain[kSlots128];
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, q = warp & 3, t = tid & 127;
    const int slot = tid / 128;
    const bool leader = t == 0;
    const bool issuer_warp = t < 32;
    const int bar = 1 + slot;
    uint8_t* stage = smem + kInfer128Stage + slot * kStageBytes;
    const uint32_t n = n_dev ? min(*n_dev, n_max) : n_max;
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    if (blockIdx.x * kSlots128 >= ntiles) return;
    float qs[NL], deq[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        qs[l] = kF8 ? f8[kF8Q + l] : 1.0f;
        deq[l] = kF8 ? 1.0f / (f8[kF8Q + l] * f8[kF8WQ + l]) : 1.0f;
    }
    if (warp == 0) umma::tmem_alloc(&tslot, 512);
    if (tid == 0) {
        umma::mbar_init(&mb_w, 1);
        for (int k = 0; k < kSlots128; ++k) {
            umma::mbar_init(&mb_mma[k], 1);
            umma::mbar_init(&mb_in[k], 1);
            umma::mbar_init(&mb_drain[k], 1);
        }
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tlane = (uint32_t)(32 * q) << 16;
    const uint32_t tmem = tslot + 256u * (uint32_t)slot;          // accumulator: columns 0..127 of the slot
    const uint32_t tmem_a = tmem + 128u;                           // A operand: columns 128..191
    const uint32_t tstride = gridDim.x * kSlots128;
    const uint64_t wdesc = umma::sdesc_sw128(umma::smem_u32(sw));
    auto fetch = [&](uint32_t tl) {
        const uint32_t rows = min((uint32_t)kTile, n - tl * kTile);
        umma::mbar_expect_tx(&mb_in[slot], rows * kRowBytes);
        umma::bulk_g2s(stage, reinterpret_cast<const uint8_t*>(in) + (size_t)tl * kStageBytes, rows * kRowBytes,
                       &mb_in[slot]);
    };
    if (tid == 0) {
        umma::mbar_expect_tx(&mb_w, kWBytes);
        umma::bulk_g2s(sw, wimg, kWBytes, &mb_w);
    }
    uint32_t tile = blockIdx.x * kSlots128 + slot;
    bool pending = tile < ntiles;
    if (pending && leader) fetch(tile);
    bool ok = umma::mbar_wait(&mb_w, 0, kSpinLimit);
    ok = __syncthreads_and(ok ? 1 : 0) != 0;
    uint32_t mph = 0, iph = 0;
    bool first = true;
    for (; tile < ntiles && ok; tile += tstride, first = false) {
        const uint32_t row = tile * kTile + (uint32_t)t;
        const bool valid = row < n;
        const bool track = TRACK && (amax_all || first);
        ok = slot_all(bar, umma::mbar_wait(&mb_in[slot], iph, kSpinLimit));
        if (!ok) break;
        pending = false;
        iph ^= 1u;
        const float a0 = encode_to_tmem<PREC, HASH>(reinterpret_cast<const TfgDatosMLP*>(stage + t * kRowBytes), bounds,
                                                    hg, qs[0], tmem_a + tlane);
        if (track) warp_amax(valid ? a0 : 0.0f, &amax[0]);
        umma::tmem_wait_st();
        umma::fence_before_sync();
        slot_sync(bar);
        if (tile + tstride < ntiles) {
            if (leader) {
                umma::fence_smem_to_async();
                fetch(tile + tstride);
            }
            pending = true;
        }
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            const bool last = l == NL - 1;
            if (issuer_warp) {
                umma::fence_after_sync();
                constexpr uint32_t id_hid = umma::idesc_f16(kTile, 128, PREC == kPrecBF16);
                constexpr uint32_t id_out = umma::idesc_f16(kTile, kOutPad, PREC == kPrecBF16);
                if (umma::elect_one()) {
                    if constexpr (kF8) {
                        // K = 32 one-byte features per MMA: one 128-byte row holds a layer's K
#pragma unroll
                        for (int s = 0; s < cols_h<128>(l) / 32; ++s)
                            umma::mma_f8_ta(tmem, tmem_a + 8u * s, wdesc + (uint64_t)((f8_off_h<128>(l) + s * 32) >> 4),
                                            last ? id_out : id_hid, s > 0);
                    } else {
#pragma unroll
                        for (int s = 0; s < cols_h<128>(l) / 16; ++s) {
                            const uint64_t bd = wdesc + (uint64_t)((foff_h<128>(NL, l) + (s >> 2) * (rows_h<128>(NL, l) * 128) +
                                                                    (s & 3) * 32) >> 4);
                            umma::mma_f16_ta(tmem, tmem_a + 8u * s, bd, last ? id_out : id_hid, s > 0);
                        }
                    }
                    umma::mma_commit(&mb_mma[slot]);
                }
                __syncwarp();
            }
            ok = slot_all(bar, umma::mbar_wait(&mb_mma[slot], mph, kSpinLimit));
            mph ^= 1u;
            if (!ok) break;
            umma::fence_after_sync();
            if (!last) {
                float lmax = 0.0f;   // max of the raw accumulator; x deq[l] > 0 keeps the order
                // FP8 keeps the column chunks rolled: unrolled, with the amax
                // tracking, the kernel outgrows the instruction cache
#pragma unroll(kF8 ? 1 : 4)
                for (int h = 0; h < 4; ++h) {
                    float v[32];
                    umma::tmem_ld32(tmem + tlane + 32u * h, v);
                    if constexpr (kF8) {
                        // dequantise, ReLU, requantise for the next layer
                        const float sc = deq[l] * qs[l + 1];
                        uint32_t r[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i)
                            r[i] = scale_relu_e4m3x4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3], sc);
                        umma::tmem_st8(tmem_a + tlane + 8u * h, r);
                        if (track) {
#pragma unroll
                            for (int i = 0; i < 32; ++i) lmax = fmaxf(lmax, v[i]);
                        }
                    } else {
                        uint32_t r[16];
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                            r[i] = PREC == kPrecBF16 ? relu_bf2(v[2 * i], v[2 * i + 1]) : relu_h2(v[2 * i], v[2 * i + 1]);
                        umma::tmem_st16(tmem_a + tlane + 16u * h, r);
                        if (track) {
#pragma unroll
                            for (int i = 0; i < 32; ++i) lmax = fmaxf(lmax, v[i]);
                        }
                    }
                }
                if (track) warp_amax(valid ? lmax * deq[l] : 0.0f, &amax[l + 1]);
                umma::tmem_wait_st();
                umma::fence_before_sync();
                slot_sync(bar);
            } else {
                float v[16];
                umma::tmem_ld16(tmem + tlane, v);
                if (valid && (out || img)) {
                    const float cr = scrub(v[0] * deq[l]), cg = scrub(v[1] * deq[l]), cb = scrub(v[2] * deq[l]);
                    if (img) {
                        const TfgColor th = thr[row];
                        if (th.r > 0 || th.g > 0 || th.b > 0) {
                            TfgColor f = img[row];
                            f.r = f.r + th.r * cr;
                            f.g = f.g + th.g * cg;
                            f.b = f.b + th.b * cb;
                            img[row] = f;
                        }
                    } else {
                        out[row] = TfgColor{cr, cg, cb};
                    }
                }
                umma::fence_before_sync();
                slot_sync(bar);
            }
        }
    }
    if (pending) umma::mbar_wait(&mb_in[slot], iph, kSpinLimit);
    if (!ok && issuer_warp) {
        if (umma::elect_one()) {
            umma::mma_commit(&mb_drain[slot]);
            umma::mbar_wait(&mb_drain[slot], 0, kSpinLimit);
        }
        __syncwarp();
    }
    if (!ok && leader) atomicExch(&g_mlp_error, 1);
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tslot, 512);
}

// FP8 inference image from the debiased weight average, one block per
// layer: the layer's weight scale wq = 448 / amax|W| goes to f8[kF8WQ + l].
// Skipped when the image already holds the weights of this Adam step.
template <int NL, int HID = 64>
__global__ void __launch_bounds__(1024) k_pack_f8(const float* __restrict__ w, const float* __restrict__ ema,
                                                  const uint32_t* __restrict__ state, float decay,
                                                  uint8_t* __restrict__ img, float* f8) {
    __shared__ float smax[32];
    const uint32_t t_adam = state[S_ADAM_T];
    if (state[S_F8_VER] == t_adam + 1u) return;
    const int l = blockIdx.x;
    const float debias = t_adam > 0u ? 1.0f - powf(decay, (float)t_adam) : 0.0f;
    const int rows = rows_h<HID>(NL, l), cols = cols_h<HID>(l), poff = poff_h<HID>(NL, l);
    const int cnt = rows * cols;
    float m = 0.0f;
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
        const int i = poff + j;
        m = fmaxf(m, fabsf(debias > 0.0f ? ema[i] / debias : w[i]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = m;
    __syncthreads();
    m = 0.0f;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = fmaxf(m, smax[k]);
    const float wq = m > 0.0f ? kF8Max / m : 1.0f;
    if (threadIdx.x == 0) f8[kF8WQ + l] = wq;
    // every byte of the layer's 128-byte rows: K index c (zero past kCols)
    for (int j = threadIdx.x; j < rows * 128; j += blockDim.x) {
        const int r = j / 128, c = j % 128;
        float x = 0.0f;
        if (c < cols) {
            const int i = poff + r * cols + c;
            x = (debias > 0.0f ? ema[i] / debias : w[i]) * wq;
        }
        __nv_fp8_e4m3 e(x);
        img[f8_off_h<HID>(l) + umma::sw128_offset(r, c >> 4) + (c & 15)] = *reinterpret_cast<uint8_t*>(&e);
    }
}

// After an FP8 inference call: new input scales from the observed amax (with
// a factor-2 margin; a layer that saw nothing keeps its scale), amax cleared,
// and the FP8 image marked current for this Adam step.
__global__ void k_f8_update(float* f8, uint32_t* state, int mark_packed) {
    const int l = threadIdx.x;
    if (l == 0 && mark_packed) state[S_F8_VER] = state[S_ADAM_T] + 1u;
    if (l >= kMaxLayers) return;
    const float a = f8[kF8Amax + l];
    if (a > 0.0f) f8[kF8Q + l] = kF8Max / (2.0f * a);
    f8[kF8Amax + l] = 0.0f;
}

// ------------------------------------------------------------------ training forward + backward
// Shared memory: fwd weights 51200 | bwd weights 40960 | A 32768.
constexpr int kTrainSmemF = 0;
constexpr int kTrainSmemB = kWeightRegion;                          // 68608, 1024-aligned
constexpr int kTrainSmemA = kTrainSmemB + bwd_bytes_of(kMaxLayers);   // 125952
constexpr int kTrainSmem = kTrainSmemA + 2 * kTile * 128;           // 158720

// Device-resident training state (one per model): read by the kernels so a
// whole frame can be enqueued (and captured in a CUDA graph) without reading
// anything back to the host.
struct TrainArgs {
    const TfgDatosMLP* buf;      // training records (targets in .color)
    const uint32_t* state;       // S_NAVAIL records available, S_STEP seed
    uint32_t min_n;              // no step below this many records
    uint32_t batch;              // samples in this step (multiple of kTile)
    Bounds bounds;
    const uint8_t* fwd;          // FP16 forward image
    const uint8_t* bwd;          // BF16 backward image
    uint8_t* hT[kMaxLayers];  // transposed inputs of each layer, per tile
    uint8_t* zT[kMaxLayers];  // transposed output gradients of each layer, per tile
    float* loss;                 // sum of per-sample losses (unnormalised)
    uint32_t navail;             // records available when given by the host (written to S_NAVAIL by
                                 // CTA 0 for the later kernels of the step); 0: read S_NAVAIL
    HashGrid hg;                 // composite encoding (levels 0: frequency encoding)
};

// Records available to a training step: given by the host (CTA 0 publishes the
// count in S_NAVAIL for the step's later kernels) or left there by the frame.
__device__ __forceinline__ uint32_t train_navail(const TrainArgs& a) {
    if (a.navail == 0u) return a.state[S_NAVAIL];
    if (blockIdx.x == 0 && threadIdx.x == 0) const_cast<uint32_t*>(a.state)[S_NAVAIL] = a.navail;
    return a.navail;
}

// Write 64 (or 16) values of sample s into the transposed BF16 tile layout.
template <int F>
__device__ __forceinline__ void store_T(uint8_t* tile, int s, const float* v) {
    uint8_t* region = tile + (s >> 6) * (F * 128);
    const int c = (s & 63) >> 3, e = s & 7;
#pragma unroll
    for (int f = 0; f < F; ++f) {
        __nv_bfloat16 h = __float2bfloat16_rn(v[f]);
        *reinterpret_cast<__nv_bfloat16*>(region + umma::sw128_offset(f, c) + 2 * e) = h;
    }
}

// 32 values of row r, features f0 .. f0 + 31 (f0 a multiple of 32), into the
// two-region A buffer as FP16 or BF16.
template <bool BF16>
__device__ __forceinline__ void store_row32(uint8_t* a, int r, int f0, const float* v) {
    uint8_t* region = a + (f0 >> 6) * (kTile * 128);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        uint32_t q[4];
#pragma unroll
        for (int e = 0; e < 4; ++e)
            q[e] = BF16 ? pack_bf2(v[8 * j + 2 * e], v[8 * j + 2 * e + 1]) : pack_h2(v[8 * j + 2 * e], v[8 * j + 2 * e + 1]);
        *reinterpret_cast<uint4*>(region + umma::sw128_offset(r, ((f0 & 63) >> 3) + j)) = make_uint4(q[0], q[1], q[2], q[3]);
    }
}

// 32 features f0 .. f0 + 31 of sample s into a transposed tile of F features.
template <int F>
__device__ __forceinline__ void store_T32(uint8_t* tile, int s, int f0, const float* v) {
    uint8_t* region = tile + (s >> 6) * (F * 128);
    const int c = (s & 63) >> 3, e = s & 7;
#pragma unroll
    for (int i = 0; i < 32; ++i)
        *reinterpret_cast<__nv_bfloat16*>(region + umma::sw128_offset(f0 + i, c) + 2 * e) = __float2bfloat16_rn(v[i]);
}

// Two warpgroups share a tile: thread t serves row (sample) t % 128, and
// warpgroup t / 128 handles 32 of each layer's 64 columns (TMEM lane quarter
// warp % 4, columns 32 * half ..), so every layer's epilogue -- TMEM load,
// ReLU and mask, the FP16 / BF16 row for the next MMA, the transposed BF16
// copy for the weight gradients -- is split over twice the warps, which the
// chain of dependent layer rounds is bound by.  The weight images are copied
// while the first tile is gathered and encoded.
constexpr int kTrainThreads = 256;

template <int NL>
__global__ void __launch_bounds__(kTrainThreads) k_train(TrainArgs a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sf = smem + kTrainSmemF;
    uint8_t* sb = smem + kTrainSmemB;
    uint8_t* sa = smem + kTrainSmemA;
    __shared__ uint64_t mb_w, mb_mma, mb_drain;
    __shared__ uint32_t tslot;
    const int t = threadIdx.x, warp = t >> 5;
    const int r = t & (kTile - 1);              // the row (sample) of the tile
    const int half = t >> 7;                    // columns 32 * half .. 32 * half + 31 of a layer
    const uint32_t lanes = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t ntiles = a.batch / kTile;
    const uint32_t n_avail = train_navail(a);
    const uint32_t seed = a.state[S_STEP];
    if (blockIdx.x >= ntiles || n_avail < a.min_n || n_avail == 0) return;
    if (warp == 0) umma::tmem_alloc(&tslot, 128);
    if (t == 0) {
        umma::mbar_init(&mb_w, 1);
        umma::mbar_init(&mb_mma, 1);
        umma::mbar_init(&mb_drain, 1);
        umma::mbar_fence_init();
    }
    for (int i = t; i < kTile * 4; i += blockDim.x) {
        const int rr = i >> 2, c = 4 + (i & 3);
        *reinterpret_cast<uint4*>(sa + kTile * 128 + umma::sw128_offset(rr, c)) = make_uint4(0, 0, 0, 0);
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    if (t == 0) {
        umma::mbar_expect_tx(&mb_w, kFwdBytes<NL> + kBwdBytes<NL>);
        umma::bulk_g2s(sf, a.fwd, kFwdBytes<NL>, &mb_w);
        umma::bulk_g2s(sb, a.bwd, kBwdBytes<NL>, &mb_w);
    }
    bool ok = true, weights_in = false;
    uint32_t mph = 0;
    float lsum = 0.0f;
    for (uint32_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        uint8_t* h0 = a.hT[0] + (size_t)tile * (2 * 96 * 128);
        float tgt[3] = {0.0f, 0.0f, 0.0f};
        if (half == 0) {
            const uint32_t s = tile * kTile + (uint32_t)r;
            // Sample selection as generarIndicesAleatorios (NrcKernel.cu:10-16).
            uint32_t st = seed ^ s;
            const uint32_t idx = pcg_next(st) % n_avail;
            const TfgDatosMLP d = a.buf[idx];
            tgt[0] = d.color.r; tgt[1] = d.color.g; tgt[2] = d.color.b;
#pragma unroll
            for (int k = 0; k < 3; ++k) if (tgt[k] > 100000.0f) tgt[k] = 100000.0f;   // NrcKernel.cu:52-57
            uint32_t w[48];
            encode(d, a.bounds, a.hg, w);
            store_encoded(sa, r, w);
            // transposed copy of the layer-0 input for dW0: features 0..63 here,
            // 64..95 by the other warpgroup once the row is in shared memory
            float f[64];
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float2 ff = __half22float2(*reinterpret_cast<__half2*>(&w[k]));
                f[2 * k] = ff.x; f[2 * k + 1] = ff.y;
            }
            store_T32<96>(h0, r, 0, f);
            store_T32<96>(h0, r, 32, f + 32);
        }
        umma::fence_smem_to_async();
        if (!weights_in) {
            ok = all_ok(umma::mbar_wait(&mb_w, 0, kSpinLimit));
            weights_in = ok;
            if (!ok) break;
        } else {
            __syncthreads();
        }
        if (half == 1) {
            const uint8_t* reg1 = sa + kTile * 128;
            float f[32];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const uint4 q = *reinterpret_cast<const uint4*>(reg1 + umma::sw128_offset(r, c));
                const uint32_t qq[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float2 ff = __half22float2(*reinterpret_cast<const __half2*>(&qq[e]));
                    f[8 * c + 2 * e] = ff.x; f[8 * c + 2 * e + 1] = ff.y;
                }
            }
            store_T32<96>(h0, r, 64, f);
        }
        uint32_t mask[NL - 1];
        // forward
        for (int l = 0; l < NL && ok; ++l) {
            const int K = kCols<NL>(l), N = (l == NL - 1) ? kOutPad : kHid;
            const uint32_t dcol = (l == NL - 1) ? 64u : 0u;
            if (warp == 0) {   // converged warp, one elected lane issues (see k_infer)
                umma::fence_after_sync();
                if (umma::elect_one()) {
                    issue_layer(tmem + dcol, sa, kTile * 128, sf + kFOff<NL>(l), kRows<NL>(l) * 128, K, N, false);
                    umma::mma_commit(&mb_mma);
                }
                __syncwarp();
            }
            ok = all_ok(umma::mbar_wait(&mb_mma, mph, kSpinLimit));
            mph ^= 1u;
            if (!ok) break;
            umma::fence_after_sync();
            if (l < NL - 1) {
                float v[32];
                umma::tmem_ld32(tmem + lanes + (uint32_t)(32 * half), v);
                uint32_t m = 0;
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const bool on = v[i] > 0.0f;
                    v[i] = on ? v[i] : 0.0f;
                    m |= (on ? 1u : 0u) << i;
                }
                mask[l] = m;
                store_row32<false>(sa, r, 32 * half, v);
                store_T32<64>(a.hT[l + 1] + (size_t)tile * (2 * 64 * 128), r, 32 * half, v);
            } else if (half == 0) {
                float v[16];
                umma::tmem_ld16(tmem + lanes + 64u, v);
                // Relative L2 on luminance: the denominator is held constant.
                const float lum = 0.299f * v[0] + 0.587f * v[1] + 0.114f * v[2];
                const float den = lum * lum + 0.01f;
                float g[64];
#pragma unroll
                for (int k = 0; k < 64; ++k) g[k] = 0.0f;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float diff = v[k] - tgt[k];
                    lsum += diff * diff / den;
                    g[k] = 2.0f * diff / den;
                }
                store_row64<true>(sa, r, g);
                store_T<16>(a.zT[NL - 1] + (size_t)tile * (2 * 16 * 128), r, g);
            }
            umma::fence_before_sync();
            umma::fence_smem_to_async();
            __syncthreads();
        }
        // backward: dH_{l-1} = dZ_l * W_l, masked by the ReLU of layer l-1
        for (int l = NL - 1; l >= 1 && ok; --l) {
            const int K = (l == NL - 1) ? kOutPad : kHid;
            if (warp == 0) {
                umma::fence_after_sync();
                if (umma::elect_one()) {
                    issue_layer(tmem, sa, kTile * 128, sb + kBOff<NL>(l), 64 * 128, K, kHid, true);
                    umma::mma_commit(&mb_mma);
                }
                __syncwarp();
            }
            ok = all_ok(umma::mbar_wait(&mb_mma, mph, kSpinLimit));
            mph ^= 1u;
            if (!ok) break;
            umma::fence_after_sync();
            float v[32];
            umma::tmem_ld32(tmem + lanes + (uint32_t)(32 * half), v);
            const uint32_t m = mask[l - 1];
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = ((m >> i) & 1u) ? v[i] : 0.0f;
            if (l > 1) store_row32<true>(sa, r, 32 * half, v);
            store_T32<64>(a.zT[l - 1] + (size_t)tile * (2 * 64 * 128), r, 32 * half, v);
            umma::fence_before_sync();
            umma::fence_smem_to_async();
            __syncthreads();
        }
    }
    // loss reduction (the loss lives in the first warpgroup)
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xFFFFFFFFu, lsum, o);
    if ((t & 31) == 0 && half == 0) atomicAdd(a.loss, lsum);
    if (!ok && warp == 0) {   // after a timeout: the weight copy and every issued MMA finish first
        if (umma::elect_one()) {
            if (!weights_in) umma::mbar_wait(&mb_w, 0, kSpinLimit);
            umma::mma_commit(&mb_drain);
            umma::mbar_wait(&mb_drain, 0, kSpinLimit);
        }
        __syncwarp();
    }
    if (!ok && t == 0) atomicExch(&g_mlp_error, 1);
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

// ------------------------------------------------------------------ width-128 training
// k_train for 128-wide layers.  The whole network's forward and backward
// images (308 KB) do not fit in shared memory, so they are streamed: the
// NL forward images and then the NL - 1 backward images of each tile pass
// through two 32 KB buffers, each bulk-copied as soon as the MMAs that read
// the buffer's previous image have completed (one layer ahead).
constexpr int kT128Buf = 32768;
constexpr int kT128SmemA = 2 * kT128Buf;                    // activations: 2 regions x 16 KB
constexpr int kT128Smem = kT128SmemA + 2 * kTile * 128;    // 98304

template <int NL>
__global__ void __launch_bounds__(128) k_train128(TrainArgs a) {
    static_assert(NL == 4 || NL == 6 || NL == 8, "width 128: 3, 5 or 7 hidden layers");
    constexpr int kItems = 2 * NL - 1;   // weight images per tile: NL forward, then NL - 1 backward
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sa = smem + kT128SmemA;
    __shared__ uint64_t mb_w[2], mb_mma, mb_drain;
    __shared__ uint32_t tslot;
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t ntiles = a.batch / kTile;
    const uint32_t n_avail = train_navail(a);
    const uint32_t seed = a.state[S_STEP];
    if (blockIdx.x >= ntiles || n_avail < a.min_n || n_avail == 0) return;
    const uint32_t total = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x * kItems;   // images this CTA loads
    if (warp == 0) umma::tmem_alloc(&tslot, 256);
    if (t == 0) {
        umma::mbar_init(&mb_w[0], 1);
        umma::mbar_init(&mb_w[1], 1);
        umma::mbar_init(&mb_mma, 1);
        umma::mbar_init(&mb_drain, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t tlane = (uint32_t)(32 * warp) << 16;
    // image g % kItems of the per-tile sequence, into buffer g & 1
    bool wpend[2] = {false, false};
    auto load = [&](uint32_t g) {
        const int k = (int)(g % (uint32_t)kItems), b = (int)(g & 1u);
        wpend[b] = true;   // every thread tracks it; thread 0 issues the copy
        if (t != 0) return;
        uint32_t bytes;
        const uint8_t* src;
        if (k < NL) {
            bytes = k == NL - 1 ? 2 * 16 * 128 : 2 * 128 * 128;
            src = a.fwd + foff_h<128>(NL, k);
        } else {
            const int l = NL - 1 - (k - NL);   // backward layers NL - 1 down to 1
            bytes = l == NL - 1 ? 128 * 128 : 2 * 128 * 128;
            src = a.bwd + boff_h<128>(NL, l);
        }
        umma::mbar_expect_tx(&mb_w[b], bytes);
        umma::bulk_g2s(smem + b * kT128Buf, src, bytes, &mb_w[b]);
    };
    load(0);
    if (total > 1) load(1);
    uint32_t wph[2] = {0, 0}, g = 0, mph = 0;
    bool ok = true;
    float lsum = 0.0f;
    // Wait for image g, issue one layer's MMAs from it, wait for them, then
    // reuse its buffer for image g + 2.
    auto run_layer = [&](uint32_t dcol, int K, int N, int w_region_bytes, bool bf16) {
        const int b = (int)(g & 1u);
        ok = all_ok(umma::mbar_wait(&mb_w[b], wph[b], kSpinLimit));
        if (!ok) return;   // the copy stays pending: the exit path waits for it
        wph[b] ^= 1u;
        wpend[b] = false;
        umma::fence_after_sync();
        if (warp == 0) {
            if (umma::elect_one()) {
                issue_layer(tmem + dcol, sa, kTile * 128, smem + b * kT128Buf, w_region_bytes, K, N, bf16);
                umma::mma_commit(&mb_mma);
            }
            __syncwarp();
        }
        ok = all_ok(umma::mbar_wait(&mb_mma, mph, kSpinLimit));
        mph ^= 1u;
        if (ok && g + 2 < total) load(g + 2);
        ++g;
        umma::fence_after_sync();
    };
    for (uint32_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const uint32_t s = tile * kTile + (uint32_t)t;
        uint32_t st = seed ^ s;
        const uint32_t idx = pcg_next(st) % n_avail;
        const TfgDatosMLP d = a.buf[idx];
        float tgt[3] = {d.color.r, d.color.g, d.color.b};
#pragma unroll
        for (int k = 0; k < 3; ++k) if (tgt[k] > 100000.0f) tgt[k] = 100000.0f;
        {
            uint32_t w[48];
            encode(d, a.bounds, a.hg, w);
            store_encoded(sa, t, w);
            float f[96];
#pragma unroll
            for (int k = 0; k < 48; ++k) {
                const float2 ff = __half22float2(*reinterpret_cast<__half2*>(&w[k]));
                f[2 * k] = ff.x; f[2 * k + 1] = ff.y;
            }
            store_T<96>(a.hT[0] + (size_t)tile * (2 * 96 * 128), t, f);
        }
        umma::fence_smem_to_async();
        __syncthreads();
        uint32_t mask[NL - 1][4];
        // forward
        for (int l = 0; l < NL && ok; ++l) {
            const bool last = l == NL - 1;
            run_layer(last ? 128u : 0u, cols_h<128>(l), last ? kOutPad : 128, rows_h<128>(NL, l) * 128, false);
            if (!ok) break;
            if (!last) {
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    float v[32];
                    umma::tmem_ld32(tmem + tlane + 32u * h, v);
                    uint32_t m = 0;
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        const bool on = v[i] > 0.0f;
                        v[i] = on ? v[i] : 0.0f;
                        m |= (on ? 1u : 0u) << i;
                    }
                    mask[l][h] = m;
                    store_row32<false>(sa, t, 32 * h, v);
                    store_T32<128>(a.hT[l + 1] + (size_t)tile * (2 * 128 * 128), t, 32 * h, v);
                }
            } else {
                float v[16];
                umma::tmem_ld16(tmem + tlane + 128u, v);
                const float lum = 0.299f * v[0] + 0.587f * v[1] + 0.114f * v[2];
                const float den = lum * lum + 0.01f;
                float gr[32];
#pragma unroll
                for (int k = 0; k < 32; ++k) gr[k] = 0.0f;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float diff = v[k] - tgt[k];
                    lsum += diff * diff / den;
                    gr[k] = 2.0f * diff / den;
                }
                store_row32<true>(sa, t, 0, gr);    // K = 16: the backward reads the first two chunks
                store_T<16>(a.zT[NL - 1] + (size_t)tile * (2 * 16 * 128), t, gr);
            }
            umma::fence_before_sync();
            umma::fence_smem_to_async();
            __syncthreads();
        }
        // backward: dH_{l-1} = dZ_l * W_l, masked by the ReLU of layer l-1
        for (int l = NL - 1; l >= 1 && ok; --l) {
            run_layer(0u, l == NL - 1 ? kOutPad : 128, 128, 128 * 128, true);
            if (!ok) break;
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                float v[32];
                umma::tmem_ld32(tmem + tlane + 32u * h, v);
                const uint32_t m = mask[l - 1][h];
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] = ((m >> i) & 1u) ? v[i] : 0.0f;
                if (l > 1) store_row32<true>(sa, t, 32 * h, v);
                store_T32<128>(a.zT[l - 1] + (size_t)tile * (2 * 128 * 128), t, 32 * h, v);
            }
            umma::fence_before_sync();
            umma::fence_smem_to_async();
            __syncthreads();
        }
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xFFFFFFFFu, lsum, o);
    if ((t & 31) == 0) atomicAdd(a.loss, lsum);
    if (!ok && warp == 0) {   // after a timeout: pending copies and issued MMAs finish first
        if (umma::elect_one()) {
            for (int b = 0; b < 2; ++b)
                if (wpend[b]) umma::mbar_wait(&mb_w[b], wph[b], kSpinLimit);
            umma::mma_commit(&mb_drain);
            umma::mbar_wait(&mb_drain, 0, kSpinLimit);
        }
        __syncwarp();
    }
    if (!ok && t == 0) atomicExch(&g_mlp_error, 1);
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, 256);
}

// ------------------------------------------------------------------ width-128 streamed inference
// Inference for width-128 networks whose forward image does not fit in shared
// memory (7 hidden layers: 233,472 B).  One 128-query tile per CTA at a time;
// the NL layer images of each tile pass through two 32 KB buffers, each
// bulk-copied as soon as the MMAs that read the buffer's previous image have
// completed (one layer ahead), as in k_train128's forward pass; the
// activations are the A operand in shared memory.  Same output rule as
// k_infer / k_infer128 (NrcKernel.cu:99-126; RenderKernel.cu:49-66).
template <int PREC, bool TRACK, int NL, bool HASH>
__global__ void __launch_bounds__(128) k_infer128s(const TfgDatosMLP* __restrict__ in, uint32_t n_max,
                                                   const uint32_t* __restrict__ n_dev, Bounds bounds, HashGrid hg,
                                                   const uint8_t* __restrict__ wimg, TfgColor* __restrict__ out,
                                                   TfgColor* __restrict__ img, const TfgColor* __restrict__ thr,
                                                   float* amax) {
    static_assert(PREC != kPrecF8 && NL >= 2 && NL <= kMaxLayers, "width 128 streamed: FP16 / BF16");
    constexpr bool kBF = PREC == kPrecBF16;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sa = smem + kT128SmemA;
    __shared__ uint64_t mb_w[2], mb_mma, mb_drain;
    __shared__ uint32_t tslot;
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t n = n_dev ? min(*n_dev, n_max) : n_max;
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    if (blockIdx.x >= ntiles) return;
    const uint32_t total = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x * NL;   // images this CTA loads
    if (warp == 0) umma::tmem_alloc(&tslot, 256);
    if (t == 0) {
        umma::mbar_init(&mb_w[0], 1);
        umma::mbar_init(&mb_w[1], 1);
        umma::mbar_init(&mb_mma, 1);
        umma::mbar_init(&mb_drain, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t tlane = (uint32_t)(32 * warp) << 16;
    bool wpend[2] = {false, false};
    auto load = [&](uint32_t g) {   // layer image g % NL into buffer g & 1
        const int k = (int)(g % (uint32_t)NL), b = (int)(g & 1u);
        wpend[b] = true;
        if (t != 0) return;
        const uint32_t bytes = k == NL - 1 ? 2 * 16 * 128 : 2 * 128 * 128;
        umma::mbar_expect_tx(&mb_w[b], bytes);
        umma::bulk_g2s(smem + b * kT128Buf, wimg + foff_h<128>(NL, k), bytes, &mb_w[b]);
    };
    load(0);
    if (total > 1) load(1);
    uint32_t wph[2] = {0, 0}, g = 0, mph = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const uint32_t row = tile * kTile + (uint32_t)t;
        const bool valid = row < n;
        {
            // rows past the end encode the last row again; their outputs are never stored
            uint32_t w[48];
            const float a0 = encode_words<PREC, HASH>(in[valid ? row : n - 1], bounds, hg, w);
            if (TRACK) warp_amax(valid ? a0 : 0.0f, &amax[0]);   // every tile: the calibration pass
            store_encoded(sa, t, w);
        }
        umma::fence_smem_to_async();
        __syncthreads();
        for (int l = 0; l < NL && ok; ++l) {
            const bool last = l == NL - 1;
            const int b = (int)(g & 1u);
            ok = all_ok(umma::mbar_wait(&mb_w[b], wph[b], kSpinLimit));
            if (!ok) break;   // the copy stays pending: the exit path waits for it
            wph[b] ^= 1u;
            wpend[b] = false;
            umma::fence_after_sync();
            if (warp == 0) {
                if (umma::elect_one()) {
                    issue_layer(tmem + (last ? 128u : 0u), sa, kTile * 128, smem + b * kT128Buf,
                                rows_h<128>(NL, l) * 128, cols_h<128>(l), last ? kOutPad : 128, kBF);
                    umma::mma_commit(&mb_mma);
                }
                __syncwarp();
            }
            ok = all_ok(umma::mbar_wait(&mb_mma, mph, kSpinLimit));
            mph ^= 1u;
            if (ok && g + 2 < total) load(g + 2);
            ++g;
            umma::fence_after_sync();
            if (!ok) break;
            if (!last) {
                float lmax = 0.0f;
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    float v[32];
                    umma::tmem_ld32(tmem + tlane + 32u * h, v);
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        v[i] = fmaxf(v[i], 0.0f);
                        if (TRACK) lmax = fmaxf(lmax, v[i]);
                    }
                    store_row32<kBF>(sa, t, 32 * h, v);
                }
                if (TRACK) warp_amax(valid ? lmax : 0.0f, &amax[l + 1]);
            } else {
                float v[16];
                umma::tmem_ld16(tmem + tlane + 128u, v);
                if (valid && (out || img)) {
                    const float cr = scrub(v[0]), cg = scrub(v[1]), cb = scrub(v[2]);
                    if (img) {
                        const TfgColor th = thr[row];
                        if (th.r > 0 || th.g > 0 || th.b > 0) {
                            TfgColor f = img[row];
                            f.r = f.r + th.r * cr;
                            f.g = f.g + th.g * cg;
                            f.b = f.b + th.b * cb;
                            img[row] = f;
                        }
                    } else {
                        out[row] = TfgColor{cr, cg, cb};
                    }
                }
            }
            umma::fence_before_sync();
            umma::fence_smem_to_async();
            __syncthreads();
        }
    }
    if (!ok && warp == 0) {   // after a timeout: pending copies and issued MMAs finish first
        if (umma::elect_one()) {
            for (int b = 0; b < 2; ++b)
                if (wpend[b]) umma::mbar_wait(&mb_w[b], wph[b], kSpinLimit);
            umma::mma_commit(&mb_drain);
            umma::mbar_wait(&mb_drain, 0, kSpinLimit);
        }
        __syncwarp();
    }
    if (!ok && t == 0) atomicExch(&g_mlp_error, 1);
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, 256);
}

// ------------------------------------------------------------------ weight gradients
// dW_l[out][in] = sum_s dZ_l[s][out] * H_l[s][in].  A = dZ^T (out rows padded
// to 128 with zeros), B = H^T (in rows), K = samples.  One CTA reduces
// `tiles_per_cta` sample tiles of one layer into TMEM and stores its partial
// sums in its own slice of `part` (the Adam step adds the slices in order).
//
// Tiles stream through kWgStages shared-memory stages.  (Four stages at
// width 64, as many as fit, measured no faster than two: 11.0 against
// 10.8 us per 16,384-sample step.)
template <int HID> constexpr int kWgStages = 2;
constexpr int kWgSmemA = 0;                                             // stages x 2 regions x 16 KB
template <int HID> constexpr int kWgSmemB = kWgStages<HID> * 32768;    // stages x 2 x FH x 128
template <int HID> constexpr int kWgStageB = 2 * (HID > 96 ? HID : 96) * 128;
template <int HID> constexpr int kWgSmemH = kWgSmemB<HID> + kWgStages<HID> * kWgStageB<HID>;
constexpr int kWgSmem = kWgSmemH<64>;                                   // 114688
static_assert(kWgSmemH<64> + 1024 <= 232448 && kWgSmemH<128> + 1024 <= 232448, "k_wgrad shared memory");

struct WgradArgs {
    const uint8_t* zT[kMaxLayers];
    const uint8_t* hT[kMaxLayers];
    float* part;                 // per-CTA partial sums, [gridDim.x][params]
    const uint32_t* state;
    uint32_t min_n;
    uint32_t ntiles;
    uint32_t tiles_per_cta;
    // When set, CTA (0, 0) ends the step (step counter, Adam time, running
    // loss, as k_tick): the forward / backward kernel that read the step's
    // seed has finished, and nothing later in a step without hash tables
    // reads the seed.
    int tick;
    const float* loss_sum;
    float inv_count;
};

// Ends a step: advance the step counter and Adam time, keep a running loss.
__device__ __forceinline__ void tick_state(uint32_t* state, const float* loss_sum, float inv_count, uint32_t min_n) {
    const uint32_t n = state[S_NAVAIL];
    if (n < min_n || n == 0) return;
    state[S_STEP] += 1u;
    state[S_ADAM_T] += 1u;
    const float loss = *loss_sum * inv_count;
    float ema = __uint_as_float(state[S_LOSS_EMA]);
    ema = (state[S_ADAM_T] == 1u) ? loss : 0.9f * ema + 0.1f * loss;
    state[S_LOSS_EMA] = __float_as_uint(ema);
}

template <int NL, int HID>
__global__ void __launch_bounds__(128) k_wgrad(WgradArgs a) {
    constexpr int S = kWgStages<HID>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ uint64_t mb_ld[S], mb_mma[S], mb_done;
    __shared__ uint32_t tslot;
    const int t = threadIdx.x, warp = t >> 5;
    const int l = blockIdx.y;
    const int FZ = l == NL - 1 ? 16 : HID, FH = l == 0 ? 96 : HID;
    const uint32_t t0 = blockIdx.x * a.tiles_per_cta;
    if (t0 >= a.ntiles || a.state[S_NAVAIL] < a.min_n || a.state[S_NAVAIL] == 0) return;
    const uint32_t t1 = min(a.ntiles, t0 + a.tiles_per_cta);
    if (a.tick && t == 0 && blockIdx.x == 0 && blockIdx.y == 0)
        tick_state(const_cast<uint32_t*>(a.state), a.loss_sum, a.inv_count, a.min_n);
    if (warp == 0) umma::tmem_alloc(&tslot, 128);
    if (t == 0) {
        for (int k = 0; k < S; ++k) { umma::mbar_init(&mb_ld[k], 1); umma::mbar_init(&mb_mma[k], 1); }
        umma::mbar_init(&mb_done, 1);
        umma::mbar_fence_init();
    }
    // Zero every A stage: rows >= FZ stay zero (padding of M to 128).
    for (int i = t; i < S * 32768 / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(smem + kWgSmemA)[i] = make_uint4(0, 0, 0, 0);
    umma::fence_smem_to_async();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t zbytes = (uint32_t)FZ * 128, hbytes = 2u * FH * 128;
    bool ld_pending[S];
    uint32_t ldph[S], mmph[S];
#pragma unroll
    for (int k = 0; k < S; ++k) { ld_pending[k] = false; ldph[k] = 0; mmph[k] = 0; }
    auto load = [&](uint32_t tile, int stage) {
        ld_pending[stage] = true;
        uint8_t* sA = smem + kWgSmemA + stage * 32768;
        uint8_t* sB = smem + kWgSmemB<HID> + stage * kWgStageB<HID>;
        const uint8_t* gz = a.zT[l] + (size_t)tile * 2 * zbytes;
        const uint8_t* gh = a.hT[l] + (size_t)tile * hbytes;
        umma::mbar_expect_tx(&mb_ld[stage], 2 * zbytes + hbytes);
        umma::bulk_g2s(sA, gz, zbytes, &mb_ld[stage]);
        umma::bulk_g2s(sA + 16384, gz + zbytes, zbytes, &mb_ld[stage]);
        umma::bulk_g2s(sB, gh, hbytes, &mb_ld[stage]);
    };
    bool ok = true;
    if (t == 0) {
        for (int k = 0; k < S && t0 + (uint32_t)k < t1; ++k) load(t0 + (uint32_t)k, k);
        const uint32_t id = umma::idesc_f16(kTile, FH, true);
        for (uint32_t tile = t0; tile < t1 && ok; ++tile) {
            const int stage = (int)((tile - t0) % (uint32_t)S);
            ok = umma::mbar_wait(&mb_ld[stage], ldph[stage], kSpinLimit);
            if (!ok) break;
            ldph[stage] ^= 1u;
            ld_pending[stage] = false;
            umma::fence_after_sync();
            const uint8_t* sA = smem + kWgSmemA + stage * 32768;
            const uint8_t* sB = smem + kWgSmemB<HID> + stage * kWgStageB<HID>;
            for (int s = 0; s < 8; ++s) {
                const int reg = s >> 2, kk = s & 3;
                const uint64_t ad = umma::sdesc_sw128(umma::smem_u32(sA + reg * 16384 + kk * 32));
                const uint64_t bd = umma::sdesc_sw128(umma::smem_u32(sB + reg * (FH * 128) + kk * 32));
                umma::mma_f16(tmem, ad, bd, id, tile > t0 || s > 0);
            }
            umma::mma_commit(&mb_mma[stage]);
            if (tile + S < t1) {
                // Refill this stage once its MMAs have read it.
                ok = umma::mbar_wait(&mb_mma[stage], mmph[stage], kSpinLimit);
                mmph[stage] ^= 1u;
                if (!ok) break;
                load(tile + S, stage);
            }
        }
        // One more commit tracks every MMA issued above; after a timeout the
        // loads still in flight are waited for as well (no copy lands after exit).
        umma::mma_commit(&mb_done);
        ok = umma::mbar_wait(&mb_done, 0, kSpinLimit) && ok;
        for (int k = 0; k < S; ++k)
            if (ld_pending[k]) umma::mbar_wait(&mb_ld[k], ldph[k], kSpinLimit);
    }
    ok = all_ok(ok);
    umma::fence_after_sync();
    if (ok && 32 * warp < FZ) {
        // This CTA's sum over its tiles, stored (no atomics) in its own slice;
        // the Adam step adds the slices in a fixed order.
        const int row = 32 * warp + (t & 31);
        for (int c0 = 0; c0 < FH; c0 += 32) {
            float v[32];
            umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            if (row < FZ) {
                float4* g = reinterpret_cast<float4*>(a.part + (size_t)blockIdx.x * params_h<HID>(NL) +
                                                      poff_h<HID>(NL, l) + row * cols_h<HID>(l) + c0);
#pragma unroll
                for (int i = 0; i < 8; ++i) g[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            }
        }
    }
    if (!ok && t == 0) atomicExch(&g_mlp_error, 1);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

// The gradient of a step that does not update (tfgMlpComputeGradient): the
// weight-gradient CTAs' partial sums added in the order the Adam step adds
// them, so both see the same gradient bit for bit.
template <int NL, int HID>
__global__ void k_wgrad_sum(const float* __restrict__ part, uint32_t groups, float* __restrict__ grad,
                            const uint32_t* __restrict__ state, uint32_t min_n) {
    if (state[S_NAVAIL] < min_n || state[S_NAVAIL] == 0) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (uint32_t)params_h<HID>(NL);
         i += gridDim.x * blockDim.x) {
        float gs = 0.0f;
        for (uint32_t k = 0; k < groups; ++k) gs += part[(size_t)k * params_h<HID>(NL) + i];
        grad[i] = gs;
    }
}

// ------------------------------------------------------------------ Adam + EMA + packing
struct AdamArgs {
    float* w;        // FP32 master
    float* m;
    float* v;
    float* ema;      // running EMA (not debiased)
    float* grad;     // summed gradient (written here when `part` is set)
    const float* part;   // weight-gradient partial sums [groups][params], or null
    uint32_t groups;
    uint8_t* fwd;    // FP16 forward image of w
    uint8_t* bwd;    // BF16 W^T image of w
    uint8_t* inf;    // FP16 image of the debiased EMA
    uint8_t* inf_bf; // BF16 image of the debiased EMA (same layout)
    float lr, beta1, beta2, eps, decay;
    float grad_scale;              // 1 / (batch * 3)
    const uint32_t* state;         // S_ADAM_T before this step, S_NAVAIL
    uint32_t min_n;
    int update;                    // 0: only re-pack (after loading parameters)
    int live0;                     // live input columns of layer 0 (the rest stay zero)
    int ticked;                    // the step's end already advanced S_ADAM_T (k_wgrad)
};

template <int NL, int HID>
__device__ __forceinline__ void layer_of(int i, int& l, int& r, int& c) {
    l = 0;
    while (i >= poff_h<HID>(NL, l + 1)) ++l;
    const int j = i - poff_h<HID>(NL, l);
    r = j / cols_h<HID>(l);
    c = j % cols_h<HID>(l);
}


template <int NL, int HID>
__global__ void k_adam(AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= params_h<HID>(NL)) return;
    int l, r, c;
    layer_of<NL, HID>(i, l, r, c);
    // Padded entries (output rows 3..15, input columns past the encoding of layer 0) stay zero.
    const bool live = !(l == NL - 1 && r >= 3) && !(l == 0 && c >= a.live0);
    float w = a.w[i];
    float e = a.ema[i];
    const bool update = a.update && a.state[S_NAVAIL] >= a.min_n && a.state[S_NAVAIL] > 0;
    const float tn = (float)(a.state[S_ADAM_T] + ((update && !a.ticked) ? 1u : 0u));
    if (update && live) {
        const float bc1 = 1.0f - powf(a.beta1, tn), bc2 = 1.0f - powf(a.beta2, tn);
        float gs = 0.0f;
        for (uint32_t k = 0; k < a.groups; ++k) gs += a.part[(size_t)k * params_h<HID>(NL) + i];
        const float g = gs * a.grad_scale;
        const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * g;
        const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * g * g;
        a.m[i] = m;
        a.v[i] = v;
        w -= a.lr * (m / bc1) / (sqrtf(v / bc2) + a.eps);
        e = a.decay * e + (1.0f - a.decay) * w;
        a.w[i] = w;
        a.ema[i] = e;
    }
    if (!live) { w = 0.0f; e = 0.0f; }
    const float ema_debias = tn > 0.0f ? 1.0f - powf(a.decay, tn) : 0.0f;
    const float ew = ema_debias > 0.0f ? e / ema_debias : w;
    // forward / inference images: row r, K index c
    const int rows = rows_h<HID>(NL, l);
    const uint32_t off = (uint32_t)foff_h<HID>(NL, l) + (uint32_t)(c >> 6) * rows * 128 +
                         umma::sw128_offset(r, (c & 63) >> 3) + 2 * (c & 7);
    *reinterpret_cast<__half*>(a.fwd + off) = __float2half_rn(w);
    *reinterpret_cast<__half*>(a.inf + off) = __float2half_rn(ew);
    *reinterpret_cast<__nv_bfloat16*>(a.inf_bf + off) = __float2bfloat16_rn(ew);
    if (l >= 1) {
        // backward image: W^T, row = c (input unit), K index = r (output unit)
        const uint32_t boff = (uint32_t)boff_h<HID>(NL, l) + (uint32_t)(r >> 6) * (HID * 128) +
                              umma::sw128_offset(c, (r & 63) >> 3) + 2 * (r & 7);
        *reinterpret_cast<__nv_bfloat16*>(a.bwd + boff) = __float2bfloat16_rn(w);
    }
}

// ------------------------------------------------------------------ hash-grid tables
// Gradient of the hash-grid tables for one training batch.  dZ_0 (the
// gradient at layer 0's pre-activation, written by k_train as transposed BF16
// tiles) times the FP16-rounded layer-0 weights gives the gradient of the 2L
// hash features; each is spread over its cell's 8 corners with the
// trilinear weights (float2 atomics into the FP32 table gradient).
struct HashGradArgs {
    const TfgDatosMLP* buf;
    const uint32_t* state;
    uint32_t min_n, batch;
    Bounds bounds;
    const uint8_t* zT0;          // dZ_0 tiles (hid features)
    const float* w0;             // FP32 master weights of layer 0, [hid][96]
    float2* grad;                // table gradient [level][T]
    HashGrid hg;
    int hid;                     // hidden width: 64 or 128
};

// One thread per (sample, level): 16 samples x 16 levels per 256-thread
// block.  The thread forms its level's two feature gradients from the
// sample's layer-0 output gradient and the FP16-rounded layer-0 weights the
// forward pass used, then scatters them to the level's 8 corners.
constexpr int kHashGradThreads = 256;
constexpr int kHashGradSamples = kHashGradThreads / kHashMaxLevels;

__global__ void __launch_bounds__(kHashGradThreads) k_hash_grad(HashGradArgs a) {
    __shared__ float sw[128][2 * kHashMaxLevels];
    __shared__ float sdz[kHashGradSamples][128 + 1];
    const int L2 = 2 * a.hg.levels;
    for (int i = threadIdx.x; i < a.hid * 2 * kHashMaxLevels; i += blockDim.x) {
        const int o = i / (2 * kHashMaxLevels), j = i % (2 * kHashMaxLevels);
        sw[o][j] = j < L2 ? __half2float(__float2half_rn(a.w0[o * 96 + j])) : 0.0f;
    }
    // dZ_0 of the block's samples (rows of the transposed BF16 tiles), all
    // loads in flight at once
    const uint32_t s0 = blockIdx.x * kHashGradSamples;
    for (int i = threadIdx.x; i < kHashGradSamples * a.hid; i += blockDim.x) {
        const uint32_t j = (uint32_t)i % kHashGradSamples, o = (uint32_t)i / kHashGradSamples, s = s0 + j;
        float v = 0.0f;
        if (s < a.batch) {
            const uint32_t tile = s / kTile, t = s % kTile;
            const uint8_t* region = a.zT0 + (size_t)tile * (2 * a.hid * 128) + (t >> 6) * (a.hid * 128);
            v = __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(
                region + umma::sw128_offset(o, (t & 63u) >> 3) + 2 * (t & 7u)));
        }
        sdz[j][o] = v;
    }
    __syncthreads();
    const uint32_t js = threadIdx.x / kHashMaxLevels, s = s0 + js;
    const int l = (int)(threadIdx.x % kHashMaxLevels);
    const uint32_t n_avail = a.state[S_NAVAIL];
    if (s >= a.batch || l >= a.hg.levels || n_avail < a.min_n || n_avail == 0) return;
    // the sample k_train drew for row s (NrcKernel.cu:10-16)
    uint32_t st = a.state[S_STEP] ^ s;
    const uint32_t idx = pcg_next(st) % n_avail;
    const TfgDatosMLP* d = a.buf + idx;
    float dx0 = 0.0f, dx1 = 0.0f;
    for (int o = 0; o < a.hid; ++o) {
        const float dz = sdz[js][o];
        dx0 = fmaf(dz, sw[o][2 * l], dx0);
        dx1 = fmaf(dz, sw[o][2 * l + 1], dx1);
    }
    if (dx0 == 0.0f && dx1 == 0.0f) return;
    const float p[3] = {unit_clamp((float)d->posicion.x, a.bounds.lo[0], a.bounds.hi[0]),
                        unit_clamp((float)d->posicion.y, a.bounds.lo[1], a.bounds.hi[1]),
                        unit_clamp((float)d->posicion.z, a.bounds.lo[2], a.bounds.hi[2])};
    const float n = a.hg.res[l];
    uint32_t i[3];
    float f[3];
    hash_cell(p, n, i, f);
    const bool dense = (a.hg.dense >> l) & 1u;
    float2* grad = a.grad + (size_t)l * a.hg.T;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t cx = i[0] + (k & 1), cy = i[1] + ((k >> 1) & 1), cz = i[2] + (k >> 2);
        const float w = ((k & 1) ? f[0] : 1.0f - f[0]) * ((k & 2) ? f[1] : 1.0f - f[1]) *
                        ((k & 4) ? f[2] : 1.0f - f[2]);
        const uint32_t q = hash_index(cx, cy, cz, (uint32_t)n, dense, a.hg.T);
        atomicAdd(&grad[q], make_float2(w * dx0, w * dx1));
    }
}

// Adam + weight average over the tables (the same optimiser and step as the
// layer weights, updated in the same step), the FP16 image of the debiased
// average for inference, and the gradient reset.
struct HashAdamArgs {
    float* w; float* m; float* v; float* ema; float* grad;
    __half* infer;
    size_t count;
    float lr, beta1, beta2, eps, decay, grad_scale;
    const uint32_t* state;
    uint32_t min_n;
    int update;
};

// Adam step of one table value: updates w, m, v, e in place and returns the
// inference value (the debiased average, or w before the first step).
// The bias corrections enter as reciprocals (one division per value left).
struct HashAdamStep {
    float lr, beta1, beta2, eps, decay, grad_scale, inv_bc1, inv_bc2, inv_debias;
    bool update;
    __device__ __forceinline__ float operator()(float& w, float& m, float& v, float& e, float g) const {
        if (update) {
            g *= grad_scale;
            m = beta1 * m + (1.0f - beta1) * g;
            v = beta2 * v + (1.0f - beta2) * g * g;
            w -= lr * (m * inv_bc1) / (sqrtf(v * inv_bc2) + eps);
            e = decay * e + (1.0f - decay) * w;
        }
        return inv_debias > 0.0f ? e * inv_debias : w;
    }
};

// Four values per thread and iteration (16-byte loads and stores of every
// array; the arrays are separate allocations, so 16-byte aligned), then a
// scalar tail.  Gradient, moments, masters and average are read once and
// written once: 38 bytes per value.
__global__ void k_adam_hash(HashAdamArgs a) {
    const bool update = a.update && a.state[S_NAVAIL] >= a.min_n && a.state[S_NAVAIL] > 0;
    const float tn = (float)(a.state[S_ADAM_T] + (update ? 1u : 0u));
    HashAdamStep st{a.lr, a.beta1, a.beta2, a.eps, a.decay, a.grad_scale,
                    1.0f / (1.0f - powf(a.beta1, tn)), 1.0f / (1.0f - powf(a.beta2, tn)),
                    tn > 0.0f ? 1.0f / (1.0f - powf(a.decay, tn)) : 0.0f, update};
    const size_t n4 = a.count / 4, stride = (size_t)gridDim.x * blockDim.x;
    const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    float4* w4 = reinterpret_cast<float4*>(a.w);
    float4* m4 = reinterpret_cast<float4*>(a.m);
    float4* v4 = reinterpret_cast<float4*>(a.v);
    float4* e4 = reinterpret_cast<float4*>(a.ema);
    float4* g4 = reinterpret_cast<float4*>(a.grad);
    uint2* i4 = reinterpret_cast<uint2*>(a.infer);
    for (size_t i = t0; i < n4; i += stride) {
        float4 w = w4[i], e = e4[i];
        const float4 g = g4[i];
        float4 m = make_float4(0.f, 0.f, 0.f, 0.f), v = m;
        if (update) { m = m4[i]; v = v4[i]; }
        const float r0 = st(w.x, m.x, v.x, e.x, g.x), r1 = st(w.y, m.y, v.y, e.y, g.y);
        const float r2 = st(w.z, m.z, v.z, e.z, g.z), r3 = st(w.w, m.w, v.w, e.w, g.w);
        if (update) { m4[i] = m; v4[i] = v; w4[i] = w; e4[i] = e; }
        g4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __half2 h01 = __floats2half2_rn(r0, r1), h23 = __floats2half2_rn(r2, r3);
        i4[i] = make_uint2(*reinterpret_cast<uint32_t*>(&h01), *reinterpret_cast<uint32_t*>(&h23));
    }
    for (size_t i = 4 * n4 + t0; i < a.count; i += stride) {
        float w = a.w[i], m = update ? a.m[i] : 0.0f, v = update ? a.v[i] : 0.0f, e = a.ema[i];
        const float r = st(w, m, v, e, a.grad[i]);
        if (update) { a.m[i] = m; a.v[i] = v; a.w[i] = w; a.ema[i] = e; }
        a.grad[i] = 0.0f;
        a.infer[i] = __float2half_rn(r);
    }
}

// Initial table values: uniform in (-1e-4, 1e-4) (Mueller et al. 2022),
// from a counter-based hash of (seed, index).
__global__ void k_hash_init(float* w, size_t count, uint64_t seed) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const float u = (float)(z >> 40) * (1.0f / 16777216.0f);
        w[i] = (2.0f * u - 1.0f) * 1e-4f;
    }
}

// After a step of a model with hash-grid tables (whose table gradient reads
// the step's seed after k_wgrad): the same end of step as k_wgrad's.
__global__ void k_tick(uint32_t* state, const float* loss_sum, float inv_count, uint32_t min_n) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    tick_state(state, loss_sum, inv_count, min_n);
}

// ------------------------------------------------------------------ cache gate
// The gate judges the cache with the path tracer's own unbiased estimates: a
// training record whose suffix ran to its end (no bootstrapped tail) carries
// L_suffix / factor, an unbiased one-sample estimate of what the cache should
// answer at its head (the target of RenderKernel.cu:92-166 without a tail
// term).  Per cell of a kGateRes^3 grid over the scene bounds the gate keeps
// running sums (decayed by kGateDecay once per frame) of the sample weight n,
// of d = lum(cache at the head) - lum(target) and of lum(target).  The cell's
// running relative error is |mean d| / sqrt(mean target^2 + 0.01) (the
// offset of the loss and of relMSE); the mean of d carries the path
// tracer's noise too (its expected square is the squared bias plus the
// variance of d over n), so a cell needs both a small bias and enough
// samples to open.  A cell is open when it has kGateMinWeight of evidence
// and its error is below the threshold: cells without evidence stay closed,
// and a cell whose error grows (the lighting changed, the cache drifted)
// closes again.
constexpr float kGateDecay = 0.8f;
constexpr float kGateMinWeight = 8.0f;

struct GateGeo {
    float lo[3], inv[3];
};

__global__ void k_gate_accumulate(const TfgRegistroEntrenamiento* __restrict__ regs, const TfgColor* __restrict__ pred,
                                  const uint32_t* n_dev, uint32_t cap, uint32_t min_n, GateGeo g, float4* cells,
                                  uint32_t* state) {
    const uint32_t n = min(*n_dev, cap);
    if (n < min_n) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) state[S_GATE] = 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const TfgRegistroEntrenamiento& r = regs[i];
        if (!r.valido) continue;
        const TfgColor ts = r.throughput_sufijo;
        if (ts.r != 0.0f || ts.g != 0.0f || ts.b != 0.0f) continue;   // bootstrapped: not an unbiased estimate
        const TfgColor L = r.luz_acumulada_sufijo, f = r.factor_normalizacion;
        float t[3] = {L.r / fmaxf(f.r, 1e-8f), L.g / fmaxf(f.g, 1e-8f), L.b / fmaxf(f.b, 1e-8f)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            t[k] = fminf(t[k], 100000.0f);
            if (isnan(t[k]) || isinf(t[k])) t[k] = 0.0f;
        }
        const TfgColor q = pred[i];
        const float lt = 0.299f * t[0] + 0.587f * t[1] + 0.114f * t[2];
        const float d = (0.299f * q.r + 0.587f * q.g + 0.114f * q.b) - lt;
        const uint32_t c = gate_cell(g.lo, g.inv, (float)r.head.posicion.x, (float)r.head.posicion.y,
                                     (float)r.head.posicion.z);
        float* cell = reinterpret_cast<float*>(&cells[c]);
        atomicAdd(cell + 0, 1.0f);
        atomicAdd(cell + 1, d);
        atomicAdd(cell + 2, lt);
    }
}

__global__ void k_gate_finish(float4* __restrict__ cells, uint32_t* __restrict__ bits, uint32_t* state, float thr2,
                              const uint32_t* n_dev, uint32_t cap, uint32_t min_n) {
    if (min(*n_dev, cap) < min_n) return;   // no records this frame: sums and bits stay
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;   // the grid covers kGateCells exactly
    const float4 v = cells[c];
    bool open = false;
    if (v.x >= kGateMinWeight) {
        const float inv_n = 1.0f / v.x;
        const float err = v.y * inv_n, mean = v.z * inv_n;
        open = err * err < thr2 * (mean * mean + 0.01f);
    }
    const uint32_t word = __ballot_sync(0xFFFFFFFFu, open);
    if ((threadIdx.x & 31u) == 0u) {
        bits[c >> 5] = word;
        if (word) atomicAdd(&state[S_GATE], (uint32_t)__popc(word));
    }
    cells[c] = make_float4(v.x * kGateDecay, v.y * kGateDecay, v.z * kGateDecay, v.w * kGateDecay);
}

__global__ void k_set_word(uint32_t* state, int index, uint32_t value) {
    if (threadIdx.x == 0 && blockIdx.x == 0) state[index] = value;
}

}  // namespace mlp

// ====================================================================== host object
struct ColorMlp {
    int dev = 0;
    uint32_t batch = 16384;
    float lr = 1e-2f, beta1 = 0.9f, beta2 = 0.99f, eps = 1e-15f, decay = 0.99f;
    mlp::Bounds bounds{{-1, -1, -1}, {1, 1, 1}};
    float* w = nullptr; float* m = nullptr; float* v = nullptr; float* ema = nullptr; float* grad = nullptr;
    float* wpart = nullptr;      // weight-gradient partial sums, one slice per gradient CTA (act_tiles slices)
    uint32_t wgroups = 0;        // slices written by the last weight-gradient launch
    uint8_t* fwd = nullptr; uint8_t* bwd = nullptr; uint8_t* inf = nullptr;
    int nl = 6;                  // layers (hidden layers + 1)
    int hid = 64;                // hidden width (64 or 128)
    uint8_t* hT[mlp::kMaxLayers] = {nullptr};
    uint8_t* zT[mlp::kMaxLayers] = {nullptr};
    float* loss = nullptr;
    uint32_t* dstate = nullptr;  // mlp::S_* words
    float gate = 0.0f;           // gate threshold on a cell's relative bias (<= 0: no gate)
    float4* gate_cells = nullptr;   // running sums per gate cell (allocated with the first threshold > 0)
    uint32_t* gate_bits = nullptr;  // open cells, one bit each
    int prec = mlp::kPrecF16;    // inference operand precision
    uint8_t* inf_bf = nullptr;   // BF16 inference image (written with the FP16 one)
    uint8_t* inf_f8 = nullptr;   // FP8 inference image (re-packed when the weights changed)
    float* f8 = nullptr;         // FP8 scale words (mlp::kF8*)
    bool f8_calibrated = false;
    uint32_t act_tiles = 0;
    int sms = 148;
    TfgMlpTuning tune{};         // batch tiling of the kernels (zero fields: defaults)
    uint32_t tune_generation = 0;
    // composite encoding: hash-grid tables (hlevels 0: frequency encoding)
    int hlevels = 0;
    uint32_t hT_entries = 0;     // entries per level
    uint32_t hdense = 0;
    float hres[mlp::kHashMaxLevels] = {};
    size_t hcount = 0;           // floats per table array (levels x entries x 2)
    float* hw = nullptr; float* hm = nullptr; float* hv = nullptr; float* hema = nullptr; float* hgrad = nullptr;
    __half* hinf = nullptr;      // FP16 image of the debiased average (inference)
};

namespace {

// The encoding view the kernels take: training reads the FP32 tables,
// inference the FP16 image of their average.
mlp::HashGrid hash_view(const ColorMlp* n, bool train) {
    mlp::HashGrid g{};
    g.levels = n->hlevels;
    if (!n->hlevels) return g;
    g.master = train ? reinterpret_cast<const float2*>(n->hw) : nullptr;
    g.infer = reinterpret_cast<const __half2*>(n->hinf);
    g.T = n->hT_entries;
    g.dense = n->hdense;
    for (int l = 0; l < mlp::kHashMaxLevels; ++l) g.res[l] = n->hres[l];
    return g;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail((int)e, std::string(what) + ": " + cudaGetErrorString(e));
}

// Calls f(std::integral_constant<int, NL>) for the model's layer count.
template <typename F>
int with_layers(int nl, F&& f) {
    switch (nl) {
        case 4: return f(std::integral_constant<int, 4>{});
        case 6: return f(std::integral_constant<int, 6>{});
        case 8: return f(std::integral_constant<int, 8>{});
        default: return fail(TFG_E_INVALID, "mlp: unsupported number of layers");
    }
}

// Calls f(integral_constant<int, NL>, integral_constant<bool, HASH>) for the
// model's layer count and encoding.
template <typename F>
int with_model(const ColorMlp* n, F&& f) {
    return with_layers(n->nl, [&](auto c) {
        if (n->hlevels) return f(c, std::integral_constant<bool, true>{});
        return f(c, std::integral_constant<bool, false>{});
    });
}

// Calls f(integral_constant<int, NL>, integral_constant<int, HID>) for the
// model's layer count and width (width 128 with 3, 5 or 7 hidden layers).
template <typename F>
int with_width(const ColorMlp* n, F&& f) {
    return with_layers(n->nl, [&](auto c) {
        constexpr int NL = decltype(c)::value;
        if constexpr (NL == 4 || NL == 6 || NL == 8) {
            if (n->hid == 128) return f(c, std::integral_constant<int, 128>{});
        }
        return f(c, std::integral_constant<int, 64>{});
    });
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int repack(ColorMlp* n, cudaStream_t s, bool update, uint32_t min_n, bool ticked) {
    mlp::AdamArgs a;
    a.w = n->w; a.m = n->m; a.v = n->v; a.ema = n->ema; a.grad = n->grad;
    a.part = update ? n->wpart : nullptr;
    a.groups = update ? n->wgroups : 0u;
    a.fwd = n->fwd; a.bwd = n->bwd; a.inf = n->inf; a.inf_bf = n->inf_bf;
    a.lr = n->lr; a.beta1 = n->beta1; a.beta2 = n->beta2; a.eps = n->eps; a.decay = n->decay;
    a.grad_scale = 1.0f / (3.0f * (float)n->batch);
    a.state = n->dstate;
    a.min_n = min_n;
    a.update = update ? 1 : 0;
    a.live0 = n->hlevels ? mlp::kHashLive : mlp::kFreqLive;
    a.ticked = ticked ? 1 : 0;
    with_width(n, [&](auto c, auto w) {
        constexpr int NL = decltype(c)::value, HID = decltype(w)::value;
        mlp::k_adam<NL, HID><<<(mlp::params_h<HID>(NL) + 255) / 256, 256, 0, s>>>(a);
        return 0;
    });
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp adam");
    if (n->hlevels) {
        mlp::HashAdamArgs h;
        h.w = n->hw; h.m = n->hm; h.v = n->hv; h.ema = n->hema; h.grad = n->hgrad; h.infer = n->hinf;
        h.count = n->hcount;
        h.lr = n->lr; h.beta1 = n->beta1; h.beta2 = n->beta2; h.eps = n->eps; h.decay = n->decay;
        h.grad_scale = a.grad_scale;
        h.state = n->dstate; h.min_n = min_n; h.update = a.update;
        mlp::k_adam_hash<<<(unsigned)std::min<size_t>((n->hcount + 255) / 256, (size_t)n->sms * 16), 256, 0, s>>>(h);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "mlp adam (tables)");
    }
    return ok();
}

int ensure_acts(ColorMlp* n, uint32_t tiles) {
    if (n->act_tiles >= tiles) return ok();
    for (int l = 0; l < mlp::kMaxLayers; ++l) {
        if (n->hT[l]) cudaFree(n->hT[l]);
        if (n->zT[l]) cudaFree(n->zT[l]);
        n->hT[l] = n->zT[l] = nullptr;
    }
    if (n->wpart) cudaFree(n->wpart);
    n->wpart = nullptr;
    for (int l = 0; l < n->nl; ++l) {
        const int fh = l == 0 ? 96 : n->hid, fz = l == n->nl - 1 ? 16 : n->hid;   // features of the tiles
        cudaError_t e = cudaMalloc((void**)&n->hT[l], (size_t)tiles * 2 * fh * 128);
        if (e == cudaSuccess) e = cudaMalloc((void**)&n->zT[l], (size_t)tiles * 2 * fz * 128);
        if (e != cudaSuccess) { n->act_tiles = 0; return cuda_fail(e, "mlp activations"); }
    }
    // one slice per gradient CTA: at most one CTA per tile
    cudaError_t e = cudaMalloc((void**)&n->wpart, (size_t)tiles * mlp::params_rt(n->nl, n->hid) * sizeof(float));
    if (e != cudaSuccess) { n->act_tiles = 0; return cuda_fail(e, "mlp gradient slices"); }
    n->act_tiles = tiles;
    return ok();
}

int check_error_flag() {
    int flag = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&flag, mlp::g_mlp_error, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "mlp status");
    if (flag) {
        int zero = 0;
        cudaMemcpyToSymbol(mlp::g_mlp_error, &zero, sizeof(int));
        return fail(TFG_E_TIMEOUT, "mlp kernel: a bounded tensor-core wait gave up");
    }
    return ok();
}

// Sample tiles per weight-gradient CTA: the tuned value, else enough CTAs
// per layer (16) to spread the reduction with at least 2 tiles each.
uint32_t wgrad_tiles_per_cta(const ColorMlp* n, uint32_t tiles) {
    if (n->tune.wgrad_tiles_per_cta > 0) return std::min<uint32_t>((uint32_t)n->tune.wgrad_tiles_per_cta, tiles);
    return std::max<uint32_t>(2u, (tiles + 15u) / 16u);
}

// Inference CTAs for `tiles` tiles of 128 queries: 4 tiles in flight per CTA,
// at most one CTA per SM or the tuned count.
uint32_t infer_grid(const ColorMlp* n, uint32_t tiles) {
    uint32_t cap = (uint32_t)n->sms;
    if (n->tune.infer_ctas > 0) cap = std::min<uint32_t>(cap, (uint32_t)n->tune.infer_ctas);
    return std::max<uint32_t>(1u, std::min<uint32_t>((tiles + mlp::kSlots - 1) / mlp::kSlots, cap));
}

int enqueue_wgrad(ColorMlp* n, uint32_t tiles_per_cta, uint32_t min_n, cudaStream_t s, bool tick = false) {
    const uint32_t tiles = n->batch / mlp::kTile;
    mlp::WgradArgs wa;
    for (int l = 0; l < mlp::kMaxLayers; ++l) { wa.zT[l] = n->zT[l]; wa.hT[l] = n->hT[l]; }
    wa.part = n->wpart; wa.state = n->dstate; wa.min_n = min_n;
    wa.ntiles = tiles;
    wa.tiles_per_cta = std::max<uint32_t>(1u, tiles_per_cta);
    wa.tick = tick ? 1 : 0;
    wa.loss_sum = n->loss;
    wa.inv_count = 1.0f / (3.0f * (float)n->batch);
    const uint32_t groups = (tiles + wa.tiles_per_cta - 1) / wa.tiles_per_cta;
    with_width(n, [&](auto c, auto w) {
        constexpr int NL = decltype(c)::value, HID = decltype(w)::value;
        mlp::k_wgrad<NL, HID><<<dim3(groups, NL), 128, mlp::kWgSmemH<HID> + 1024, s>>>(wa);
        return 0;
    });
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp step: weight gradients");
    n->wgroups = groups;
    return ok();
}

// The summed gradient in n->grad (steps that do not update).
int enqueue_wgrad_sum(ColorMlp* n, uint32_t min_n, cudaStream_t s) {
    with_width(n, [&](auto c, auto w) {
        constexpr int NL = decltype(c)::value, HID = decltype(w)::value;
        mlp::k_wgrad_sum<NL, HID><<<(mlp::params_h<HID>(NL) + 255) / 256, 256, 0, s>>>(n->wpart, n->wgroups, n->grad,
                                                                                          n->dstate, min_n);
        return 0;
    });
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp step: gradient sum");
    return ok();
}

// Forward/backward, weight gradients (and, with `update`, Adam + tick) of one
// step whose record count and seed are already in the device state.
// One training step.  `navail`: records available, given by the host (0:
// already in S_NAVAIL, as a frame leaves it).
int enqueue_step(ColorMlp* n, const TfgDatosMLP* buf, uint32_t min_n, bool update, cudaStream_t s,
                 uint32_t navail = 0) {
    const uint32_t tiles = n->batch / mlp::kTile;
    cudaError_t e = cudaMemsetAsync(n->loss, 0, sizeof(float), s);
    if (e != cudaSuccess) return cuda_fail(e, "mlp step");
    mlp::TrainArgs ta;
    ta.buf = buf; ta.state = n->dstate; ta.min_n = min_n; ta.batch = n->batch;
    ta.bounds = n->bounds; ta.fwd = n->fwd; ta.bwd = n->bwd; ta.loss = n->loss;
    ta.hg = hash_view(n, true);
    ta.navail = navail;
    for (int l = 0; l < mlp::kMaxLayers; ++l) { ta.hT[l] = n->hT[l]; ta.zT[l] = n->zT[l]; }
    with_width(n, [&](auto c, auto w) {
        constexpr int NL = decltype(c)::value, HID = decltype(w)::value;
        const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)n->sms);
        if constexpr (HID == 128) mlp::k_train128<NL><<<grid, 128, mlp::kT128Smem + 1024, s>>>(ta);
        else mlp::k_train<NL><<<grid, mlp::kTrainThreads, mlp::kTrainSmem + 1024, s>>>(ta);
        return 0;
    });
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp step: forward/backward");
    // Without hash tables the weight-gradient kernel ends the step; the table
    // gradient re-draws the step's samples from its seed, so with tables
    // k_tick ends it after the table update.
    const bool tick_early = update && n->hlevels == 0;
    if (int rc = enqueue_wgrad(n, wgrad_tiles_per_cta(n, tiles), min_n, s, tick_early)) return rc;
    if (n->hlevels) {
        mlp::HashGradArgs ha;
        ha.buf = buf; ha.state = n->dstate; ha.min_n = min_n; ha.batch = n->batch; ha.bounds = n->bounds;
        ha.zT0 = n->zT[0]; ha.w0 = n->w; ha.grad = reinterpret_cast<float2*>(n->hgrad); ha.hg = hash_view(n, true);
        ha.hid = n->hid;
        mlp::k_hash_grad<<<(n->batch + mlp::kHashGradSamples - 1) / mlp::kHashGradSamples, mlp::kHashGradThreads, 0, s>>>(ha);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "mlp step: table gradient");
    }
    if (!update) return enqueue_wgrad_sum(n, min_n, s);
    if (int rc = repack(n, s, true, min_n, tick_early)) return rc;
    if (n->hlevels) {
        mlp::k_tick<<<1, 32, 0, s>>>(n->dstate, n->loss, 1.0f / (3.0f * (float)n->batch), min_n);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "mlp step: tick");
    }
    return ok();
}

int set_word(ColorMlp* n, int index, uint32_t value, cudaStream_t s) {
    mlp::k_set_word<<<1, 32, 0, s>>>(n->dstate, index, value);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp state");
    return ok();
}

int infer_impl(ColorMlp* n, const TfgDatosMLP* in, TfgColor* out, TfgColor* img, const TfgColor* thr, uint32_t count,
               const uint32_t* n_dev, cudaStream_t s) {
    if (count == 0) return ok();
    if ((reinterpret_cast<uintptr_t>(in) & 15u) != 0)
        return fail(TFG_E_INVALID, "mlp inference: input buffer must be 16-byte aligned");
    if (n->prec == mlp::kPrecF8 && !n->f8_calibrated)
        return fail(TFG_E_INVALID, "mlp inference: FP8 needs tfgMlpCalibrate first");
    const uint32_t tiles = (count + mlp::kTile - 1) / mlp::kTile;
    if (n->hid == 128) {
        uint32_t cap = (uint32_t)n->sms;
        if (n->tune.infer_ctas > 0) cap = std::min<uint32_t>(cap, (uint32_t)n->tune.infer_ctas);
        const uint32_t grid128 =
            std::max<uint32_t>(1u, std::min<uint32_t>((tiles + mlp::kSlots128 - 1) / mlp::kSlots128, cap));
        const uint8_t* wimg = n->prec == mlp::kPrecBF16 ? n->inf_bf : n->inf;
        with_model(n, [&](auto c, auto h) {
            constexpr int NL = decltype(c)::value;
            constexpr bool HASH = decltype(h)::value;
            if constexpr (NL == 4 || NL == 6) {
                const size_t sm = mlp::kInfer128Smem + 1024;
                if (n->prec == mlp::kPrecF16) {
                    mlp::k_infer128<mlp::kPrecF16, false, NL, HASH><<<grid128, mlp::kInfer128Threads, sm, s>>>(
                        in, count, n_dev, n->bounds, hash_view(n, false), wimg, out, img, thr, nullptr, nullptr, 0);
                } else if (n->prec == mlp::kPrecBF16) {
                    mlp::k_infer128<mlp::kPrecBF16, false, NL, HASH><<<grid128, mlp::kInfer128Threads, sm, s>>>(
                        in, count, n_dev, n->bounds, hash_view(n, false), wimg, out, img, thr, nullptr, nullptr, 0);
                } else {
                    mlp::k_pack_f8<NL, 128><<<NL, 1024, 0, s>>>(n->w, n->ema, n->dstate, n->decay, n->inf_f8, n->f8);
                    mlp::k_infer128<mlp::kPrecF8, true, NL, HASH><<<grid128, mlp::kInfer128Threads, sm, s>>>(
                        in, count, n_dev, n->bounds, hash_view(n, false), n->inf_f8, out, img, thr, n->f8,
                        n->f8 + mlp::kF8Amax, 0);
                    mlp::k_f8_update<<<1, 32, 0, s>>>(n->f8, n->dstate, 1);
                }
            } else if constexpr (NL == 8) {
                if (n->prec == mlp::kPrecF8) {
                    // the E4M3 image of 7 hidden layers (116,736 B) stays resident
                    const size_t sm = mlp::kInfer128Smem + 1024;
                    mlp::k_pack_f8<NL, 128><<<NL, 1024, 0, s>>>(n->w, n->ema, n->dstate, n->decay, n->inf_f8, n->f8);
                    mlp::k_infer128<mlp::kPrecF8, true, NL, HASH><<<grid128, mlp::kInfer128Threads, sm, s>>>(
                        in, count, n_dev, n->bounds, hash_view(n, false), n->inf_f8, out, img, thr, n->f8,
                        n->f8 + mlp::kF8Amax, 0);
                    mlp::k_f8_update<<<1, 32, 0, s>>>(n->f8, n->dstate, 1);
                    return 0;
                }
                // FP16 / BF16 weights stream: one tile per CTA at a time, two CTAs per SM
                const size_t sm = mlp::kT128Smem + 1024;
                const uint32_t grid_s = std::max<uint32_t>(1u, std::min<uint32_t>(tiles, 2u * cap));
                if (n->prec == mlp::kPrecF16)
                    mlp::k_infer128s<mlp::kPrecF16, false, NL, HASH><<<grid_s, 128, sm, s>>>(
                        in, count, n_dev, n->bounds, hash_view(n, false), wimg, out, img, thr, nullptr);
                else
                    mlp::k_infer128s<mlp::kPrecBF16, false, NL, HASH><<<grid_s, 128, sm, s>>>(
                        in, count, n_dev, n->bounds, hash_view(n, false), wimg, out, img, thr, nullptr);
            }
            return 0;
        });
        cudaError_t e1 = cudaGetLastError();
        if (e1 != cudaSuccess) return cuda_fail(e1, "mlp inference");
        return ok();
    }
    const uint32_t grid = infer_grid(n, tiles);
    const size_t smem = mlp::kInferSmem + 1024;
    cudaError_t e = cudaSuccess;
    const int rc = with_model(n, [&](auto c, auto h) {
        constexpr int NL = decltype(c)::value;
        constexpr bool HASH = decltype(h)::value;
        if (n->prec == mlp::kPrecF16) {
            mlp::k_infer<mlp::kPrecF16, false, NL, HASH><<<grid, mlp::kInferThreads, smem, s>>>(
                in, count, n_dev, n->bounds, hash_view(n, false), n->inf, out, img, thr, nullptr, nullptr, 0);
        } else if (n->prec == mlp::kPrecBF16) {
            mlp::k_infer<mlp::kPrecBF16, false, NL, HASH><<<grid, mlp::kInferThreads, smem, s>>>(
                in, count, n_dev, n->bounds, hash_view(n, false), n->inf_bf, out, img, thr, nullptr, nullptr, 0);
        } else {
            mlp::k_pack_f8<NL><<<NL, 1024, 0, s>>>(n->w, n->ema, n->dstate, n->decay, n->inf_f8, n->f8);
            cudaError_t e2 = cudaGetLastError();
            if (e2 != cudaSuccess) return cuda_fail(e2, "mlp inference: FP8 weight image");
            mlp::k_infer<mlp::kPrecF8, true, NL, HASH><<<grid, mlp::kInferThreads, smem, s>>>(
                in, count, n_dev, n->bounds, hash_view(n, false), n->inf_f8, out, img, thr, n->f8, n->f8 + mlp::kF8Amax,
                0);
            e2 = cudaGetLastError();
            if (e2 != cudaSuccess) return cuda_fail(e2, "mlp inference");
            mlp::k_f8_update<<<1, 32, 0, s>>>(n->f8, n->dstate, 1);
        }
        return 0;
    });
    if (rc) return rc;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp inference");
    return ok();
}

// Per-layer input amax over `count` samples through the FP16 path (every
// tile), turned into the FP8 input scales.
int calibrate_impl(ColorMlp* n, const TfgDatosMLP* in, uint32_t count, cudaStream_t s) {
    if (count == 0) return fail(TFG_E_INVALID, "tfgMlpCalibrate: no samples");
    if ((reinterpret_cast<uintptr_t>(in) & 15u) != 0)
        return fail(TFG_E_INVALID, "tfgMlpCalibrate: input buffer must be 16-byte aligned");
    const uint32_t tiles = (count + mlp::kTile - 1) / mlp::kTile;
    const uint32_t grid = std::min<uint32_t>((tiles + mlp::kSlots - 1) / mlp::kSlots, (uint32_t)n->sms);
    cudaError_t e = cudaMemsetAsync(n->f8 + mlp::kF8Amax, 0, mlp::kMaxLayers * sizeof(float), s);
    if (e != cudaSuccess) return cuda_fail(e, "tfgMlpCalibrate");
    with_model(n, [&](auto c, auto h) {
        constexpr int NL = decltype(c)::value;
        constexpr bool HASH = decltype(h)::value;
        if (n->hid == 128) {
            if constexpr (NL == 4 || NL == 6) {
                const uint32_t g128 = std::min<uint32_t>((tiles + mlp::kSlots128 - 1) / mlp::kSlots128, (uint32_t)n->sms);
                mlp::k_infer128<mlp::kPrecF16, true, NL, HASH><<<g128, mlp::kInfer128Threads, mlp::kInfer128Smem + 1024, s>>>(
                    in, count, nullptr, n->bounds, hash_view(n, false), n->inf, nullptr, nullptr, nullptr, nullptr,
                    n->f8 + mlp::kF8Amax, 1);
            } else if constexpr (NL == 8) {   // the FP16 pass streams its weights
                const uint32_t gs = std::min<uint32_t>(tiles, 2u * (uint32_t)n->sms);
                mlp::k_infer128s<mlp::kPrecF16, true, NL, HASH><<<gs, 128, mlp::kT128Smem + 1024, s>>>(
                    in, count, nullptr, n->bounds, hash_view(n, false), n->inf, nullptr, nullptr, nullptr,
                    n->f8 + mlp::kF8Amax);
            }
            return 0;
        }
        mlp::k_infer<mlp::kPrecF16, true, NL, HASH><<<grid, mlp::kInferThreads, mlp::kInferSmem + 1024, s>>>(
            in, count, nullptr, n->bounds, hash_view(n, false), n->inf, nullptr, nullptr, nullptr, nullptr,
            n->f8 + mlp::kF8Amax, 1);
        return 0;
    });
    e = cudaGetLastError();
    if (e == cudaSuccess) { mlp::k_f8_update<<<1, 32, 0, s>>>(n->f8, n->dstate, 0); e = cudaGetLastError(); }
    if (e != cudaSuccess) return cuda_fail(e, "tfgMlpCalibrate");
    n->f8_calibrated = true;
    return ok();
}

// Times `launch` (one warm-up, then `repeats` launches between two events on
// `s`); the mean in *ms.
template <typename F>
int time_launches(F&& launch, int repeats, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, float* ms) {
    if (int rc = launch()) return rc;
    cudaEventRecord(e0, s);
    for (int r = 0; r < repeats; ++r)
        if (int rc = launch()) return rc;
    cudaEventRecord(e1, s);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    if (e != cudaSuccess) return cuda_fail(e, "tfgMlpAutotune: timing");
    *ms /= (float)repeats;
    return check_error_flag();
}

// The model's autotuner: candidates in turn, the current setting first; a
// candidate replaces the best only when at least 1% faster.  The gradient
// buffer, FP8 scale words and device state words are saved before and put
// back after, so the model continues exactly as before.
int autotune_impl(ColorMlp* n, const TfgDatosMLP* in, uint32_t count, TfgColor* out, int repeats,
                  TfgMlpTuning* result, float* ms_out, cudaStream_t s) {
    if (count && (!in || !out)) return fail(TFG_E_INVALID, "tfgMlpAutotune: null inference buffer");
    if (count && (reinterpret_cast<uintptr_t>(in) & 15u) != 0)
        return fail(TFG_E_INVALID, "tfgMlpAutotune: input buffer must be 16-byte aligned");
    if (count && n->prec == mlp::kPrecF8 && !n->f8_calibrated)
        return fail(TFG_E_INVALID, "tfgMlpAutotune: FP8 needs tfgMlpCalibrate first");
    repeats = repeats > 0 ? std::min(repeats, 1000) : 5;
    const uint32_t tiles = n->batch / mlp::kTile;
    if (int rc = ensure_acts(n, tiles)) return rc;
    const size_t gbytes = (size_t)mlp::params_rt(n->nl, n->hid) * sizeof(float);
    const size_t fbytes = mlp::kF8Words * sizeof(float), sbytes = mlp::S_WORDS * sizeof(uint32_t);
    uint8_t* saved = nullptr;
    cudaError_t e = cudaMalloc((void**)&saved, gbytes + fbytes + sbytes);
    if (e != cudaSuccess) return cuda_fail(e, "tfgMlpAutotune");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(saved, n->grad, gbytes, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(saved + gbytes, n->f8, fbytes, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(saved + gbytes + fbytes, n->dstate, sbytes, cudaMemcpyDeviceToDevice, s);
    int rc = e == cudaSuccess ? 0 : cuda_fail(e, "tfgMlpAutotune: save state");
    const TfgMlpTuning before = n->tune;
    TfgMlpTuning best = n->tune;
    float best_wg = 0.0f, best_inf = 0.0f;
    // Weight gradients of one batch; the record count is set so the kernel runs.
    if (!rc) rc = set_word(n, mlp::S_NAVAIL, n->batch, s);
    if (!rc) {
        std::vector<uint32_t> cands{wgrad_tiles_per_cta(n, tiles)};
        for (uint32_t t = 1; t <= 64 && t <= tiles; t *= 2)
            if (t != cands[0]) cands.push_back(t);
        for (size_t i = 0; i < cands.size() && !rc; ++i) {
            float ms = 0.0f;
            // the gradient CTAs and the sum of their slices (which the Adam step does in a frame)
            rc = time_launches([&] {
                const int r = enqueue_wgrad(n, cands[i], 0, s);
                return r ? r : enqueue_wgrad_sum(n, 0, s);
            }, repeats, s, e0, e1, &ms);
            if (!rc && (i == 0 || ms < 0.99f * best_wg)) { best_wg = ms; best.wgrad_tiles_per_cta = (int32_t)cands[i]; }
        }
    }
    // Inference of the caller's batch.
    if (!rc && count) {
        const int sms = n->sms;
        std::vector<int> cands{n->tune.infer_ctas > 0 ? std::min(n->tune.infer_ctas, sms) : sms};
        for (int c : {sms, 3 * sms / 4, sms / 2})
            if (c > 0 && c != cands[0]) cands.push_back(c);
        for (size_t i = 0; i < cands.size() && !rc; ++i) {
            n->tune.infer_ctas = cands[i];
            float ms = 0.0f;
            rc = time_launches([&] { return infer_impl(n, in, out, nullptr, nullptr, count, nullptr, s); }, repeats, s,
                               e0, e1, &ms);
            if (!rc && (i == 0 || ms < 0.99f * best_inf)) { best_inf = ms; best.infer_ctas = cands[i]; }
        }
    }
    // Put the model back as it was.
    cudaError_t r = cudaMemcpyAsync(n->grad, saved, gbytes, cudaMemcpyDeviceToDevice, s);
    if (r == cudaSuccess) r = cudaMemcpyAsync(n->f8, saved + gbytes, fbytes, cudaMemcpyDeviceToDevice, s);
    if (r == cudaSuccess) r = cudaMemcpyAsync(n->dstate, saved + gbytes + fbytes, sbytes, cudaMemcpyDeviceToDevice, s);
    if (r == cudaSuccess) r = cudaStreamSynchronize(s);
    cudaFree(saved);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc) { n->tune = before; return rc; }
    if (r != cudaSuccess) { n->tune = before; return cuda_fail(r, "tfgMlpAutotune: restore state"); }
    if (best.infer_ctas == n->sms) best.infer_ctas = 0;
    n->tune = best;
    ++n->tune_generation;
    if (result) *result = best;
    if (ms_out) { ms_out[0] = best_wg; ms_out[1] = best_inf; }
    return ok();
}

}  // namespace

// ------------------------------------------------------------------ internal API (frame driver)
int mlp_prepare(ColorMlp* n) { return ensure_acts(n, n->batch / mlp::kTile); }
uint32_t* mlp_state(ColorMlp* n) { return n->dstate; }
uint32_t* mlp_navail(ColorMlp* n) { return n->dstate + mlp::S_NAVAIL; }
int mlp_enqueue_infer(ColorMlp* n, const TfgDatosMLP* in, TfgColor* out, TfgColor* img, const TfgColor* thr,
                      uint32_t max_count, const uint32_t* n_dev, cudaStream_t s) {
    return infer_impl(n, in, out, img, thr, max_count, n_dev, s);
}
int mlp_enqueue_train(ColorMlp* n, const TfgDatosMLP* buf, uint32_t min_n, cudaStream_t s) {
    return enqueue_step(n, buf, min_n, true, s);
}
int mlp_set_gate_threshold(ColorMlp* n, float g) {
    if (!(g >= 0.0f)) return fail(TFG_E_INVALID, "nrc frame: gate_threshold must be >= 0");
    if (g > 0.0f && !n->gate_cells) {
        cudaError_t e = cudaMalloc((void**)&n->gate_cells, (size_t)kGateCells * sizeof(float4));
        if (e == cudaSuccess) e = cudaMalloc((void**)&n->gate_bits, (size_t)kGateCells / 8);
        if (e == cudaSuccess) e = cudaMemset(n->gate_cells, 0, (size_t)kGateCells * sizeof(float4));
        if (e == cudaSuccess) e = cudaMemset(n->gate_bits, 0, (size_t)kGateCells / 8);
        if (e != cudaSuccess) {
            if (n->gate_cells) cudaFree(n->gate_cells);
            if (n->gate_bits) cudaFree(n->gate_bits);
            n->gate_cells = nullptr; n->gate_bits = nullptr;
            return cuda_fail(e, "nrc frame: gate grid");
        }
    }
    n->gate = g;
    return ok();
}

void mlp_gate_view(ColorMlp* n, CachePolicy& p) {
    p.gate_bits = n->gate > 0.0f ? n->gate_bits : nullptr;
    for (int k = 0; k < 3; ++k) {
        p.gate_lo[k] = n->bounds.lo[k];
        const float ext = n->bounds.hi[k] - n->bounds.lo[k];
        p.gate_inv[k] = ext > 0.0f ? (float)kGateRes / ext : 0.0f;
    }
}

int mlp_enqueue_gate_update(ColorMlp* n, const TfgRegistroEntrenamiento* regs, const TfgColor* tail_pred,
                            const uint32_t* n_dev, uint32_t cap, uint32_t min_n, cudaStream_t s) {
    if (!(n->gate > 0.0f) || !n->gate_cells) return ok();
    CachePolicy p;
    mlp_gate_view(n, p);
    mlp::GateGeo g;
    for (int k = 0; k < 3; ++k) { g.lo[k] = p.gate_lo[k]; g.inv[k] = p.gate_inv[k]; }
    const unsigned blocks = (unsigned)std::max(1u, std::min((cap + 255u) / 256u, 148u * 4u));
    mlp::k_gate_accumulate<<<blocks, 256, 0, s>>>(regs, tail_pred, n_dev, cap, min_n, g, n->gate_cells, n->dstate);
    static_assert(kGateCells % 256 == 0, "gate grid: whole blocks");
    mlp::k_gate_finish<<<kGateCells / 256, 256, 0, s>>>(n->gate_cells, n->gate_bits, n->dstate, n->gate * n->gate,
                                                          n_dev, cap, min_n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "nrc frame: gate update");
    return ok();
}
int mlp_precision(const ColorMlp* n) { return n->prec; }
uint32_t mlp_tuning_generation(const ColorMlp* n) { return n->tune_generation; }

}  // namespace tfg

using tfg::ColorMlp;
namespace M = tfg::mlp;

namespace {
template <int NL>
void set_kernel_attrs() {
    const int ism = M::kInferSmem + 1024;
    cudaFuncSetAttribute(M::k_infer<M::kPrecF16, false, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ism);
    cudaFuncSetAttribute(M::k_infer<M::kPrecF16, true, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ism);
    cudaFuncSetAttribute(M::k_infer<M::kPrecBF16, false, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ism);
    cudaFuncSetAttribute(M::k_infer<M::kPrecF8, true, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ism);
    cudaFuncSetAttribute(M::k_infer<M::kPrecF16, false, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ism);
    cudaFuncSetAttribute(M::k_infer<M::kPrecF16, true, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ism);
    cudaFuncSetAttribute(M::k_infer<M::kPrecBF16, false, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ism);
    cudaFuncSetAttribute(M::k_infer<M::kPrecF8, true, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ism);
    cudaFuncSetAttribute(M::k_train<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, M::kTrainSmem + 1024);
    cudaFuncSetAttribute(M::k_wgrad<NL, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, M::kWgSmem + 1024);
    if constexpr (NL == 4 || NL == 6) {
        const int i128 = M::kInfer128Smem + 1024;
        cudaFuncSetAttribute(M::k_infer128<M::kPrecF16, false, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecBF16, false, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecF16, true, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecF8, true, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecF16, false, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecBF16, false, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecF16, true, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecF8, true, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_train128<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, M::kT128Smem + 1024);
        cudaFuncSetAttribute(M::k_wgrad<NL, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, M::kWgSmemH<128> + 1024);
    }
    if constexpr (NL == 8) {   // width 128 with 7 hidden layers: streamed weights
        const int s128 = M::kT128Smem + 1024;
        const int i128 = M::kInfer128Smem + 1024;
        cudaFuncSetAttribute(M::k_infer128s<M::kPrecF16, false, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128);
        cudaFuncSetAttribute(M::k_infer128s<M::kPrecBF16, false, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128);
        cudaFuncSetAttribute(M::k_infer128s<M::kPrecF16, true, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128);
        cudaFuncSetAttribute(M::k_infer128s<M::kPrecF16, false, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128);
        cudaFuncSetAttribute(M::k_infer128s<M::kPrecBF16, false, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128);
        cudaFuncSetAttribute(M::k_infer128s<M::kPrecF16, true, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecF8, true, NL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_infer128<M::kPrecF8, true, NL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, i128);
        cudaFuncSetAttribute(M::k_train128<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, s128);
        cudaFuncSetAttribute(M::k_wgrad<NL, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, M::kWgSmemH<128> + 1024);
    }
}
}  // namespace

extern "C" int tfgMlpCreate(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed, TfgColorMLP** out) {
    return tfgMlpCreateEx(n_in, n_out, batch, seed, 5, out);
}

extern "C" void tfgHashGridConfigReference(TfgHashGridConfig* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->n_levels = 16;              // mlp.cpp:33-39
    c->log2_hashmap_size = 19;
    c->base_resolution = 16.0f;
    c->per_level_scale = 1.5f;
}

namespace tfg {
namespace {

// Tables of the composite encoding: sizes, level resolutions, FP32 arrays and
// the FP16 inference image (written by the first re-pack).
int create_tables(ColorMlp* n, const TfgHashGridConfig& c, uint64_t seed) {
    if (c.n_levels < 1 || c.n_levels > M::kHashMaxLevels)
        return fail(TFG_E_INVALID, "tfgMlpCreateHashGrid: n_levels must be in [1, 16]");
    if (c.log2_hashmap_size < 10 || c.log2_hashmap_size > 24)
        return fail(TFG_E_INVALID, "tfgMlpCreateHashGrid: log2_hashmap_size must be in [10, 24]");
    if (!(c.base_resolution >= 2.0f) || !(c.per_level_scale >= 1.0f))
        return fail(TFG_E_INVALID, "tfgMlpCreateHashGrid: base_resolution >= 2 and per_level_scale >= 1");
    const uint32_t T = 1u << c.log2_hashmap_size;
    n->hlevels = c.n_levels;
    n->hT_entries = T;
    n->hdense = 0;
    for (int l = 0; l < c.n_levels; ++l) {
        const double N = std::floor((double)c.base_resolution * std::pow((double)c.per_level_scale, (double)l));
        if (N < 1.0 || N > (double)(1u << 20))
            return fail(TFG_E_INVALID, "tfgMlpCreateHashGrid: a level resolution leaves [1, 2^20]");
        n->hres[l] = (float)N;
        const uint64_t st = (uint64_t)N + 1u;
        if (st * st * st <= (uint64_t)T) n->hdense |= 1u << l;
    }
    n->hcount = (size_t)c.n_levels * T * 2u;
    const size_t hb = n->hcount * sizeof(float);
    cudaError_t e = cudaMalloc((void**)&n->hw, hb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->hm, hb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->hv, hb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->hema, hb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->hgrad, hb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->hinf, n->hcount * sizeof(__half));
    if (e == cudaSuccess) e = cudaMemset(n->hm, 0, hb);
    if (e == cudaSuccess) e = cudaMemset(n->hv, 0, hb);
    if (e == cudaSuccess) e = cudaMemset(n->hema, 0, hb);
    if (e == cudaSuccess) e = cudaMemset(n->hgrad, 0, hb);
    if (e != cudaSuccess) return cuda_fail(e, "tfgMlpCreateHashGrid");
    M::k_hash_init<<<(unsigned)std::min<size_t>((n->hcount + 255) / 256, (size_t)n->sms * 16), 256>>>(
        n->hw, n->hcount, seed ^ 0x7AB1E5ull);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "tfgMlpCreateHashGrid");
    return ok();
}

int create_model(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed, int32_t hidden_layers, int32_t width,
                 const TfgHashGridConfig* hc, TfgColorMLP** out) {
    if (!out) return tfg::fail(TFG_E_INVALID, "tfgMlpCreate: out is null");
    *out = nullptr;
    if (hidden_layers != 3 && hidden_layers != 5 && hidden_layers != 7)
        return tfg::fail(TFG_E_INVALID, "tfgMlpCreate: hidden_layers must be 3, 5 or 7");
    if (width != 64 && width != 128) return tfg::fail(TFG_E_INVALID, "tfgMlpCreate: width must be 64 or 128");
    const int nl = hidden_layers + 1;
    if (n_in != 15 || n_out != 3) return tfg::fail(TFG_E_INVALID, "tfgMlpCreate: the cache takes 15 inputs and 3 outputs");
    if (batch == 0 || batch % M::kTile != 0 || batch > (1u << 24))
        return tfg::fail(TFG_E_INVALID, "tfgMlpCreate: batch must be a positive multiple of 128");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpCreate");
    if (int rc = tfg::require_sm100(dev)) return rc;
    ColorMlp* n = new ColorMlp();
    n->dev = dev;
    n->batch = batch;
    n->nl = nl;
    n->hid = width;
    cudaDeviceGetAttribute(&n->sms, cudaDevAttrMultiProcessorCount, dev);
    const int nparams = M::params_rt(nl, width);
    const size_t pb = nparams * sizeof(float);
    const size_t fwd_bytes = M::fwd_bytes_rt(nl, width), bwd_bytes = M::bwd_bytes_rt(nl, width),
                 f8_bytes = width == 128 ? M::f8_bytes_h<128>(nl) : M::f8_bytes_of(nl);
    e = cudaMalloc((void**)&n->w, pb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->m, pb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->v, pb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->ema, pb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->grad, pb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->fwd, fwd_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->bwd, bwd_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->inf, fwd_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->inf_bf, fwd_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->inf_f8, f8_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->f8, M::kF8Words * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void**)&n->dstate, M::S_WORDS * sizeof(uint32_t));
    if (e != cudaSuccess) { tfgMlpDestroy(reinterpret_cast<TfgColorMLP*>(n)); return tfg::cuda_fail(e, "tfgMlpCreate"); }
    cudaMemset(n->fwd, 0, fwd_bytes);
    cudaMemset(n->bwd, 0, bwd_bytes);
    cudaMemset(n->inf, 0, fwd_bytes);
    cudaMemset(n->inf_bf, 0, fwd_bytes);
    cudaMemset(n->inf_f8, 0, f8_bytes);
    cudaMemset(n->f8, 0, M::kF8Words * sizeof(float));
    cudaMemset(n->dstate, 0, M::S_WORDS * sizeof(uint32_t));
    if (hc) {
        if (int rc = create_tables(n, *hc, seed)) { tfgMlpDestroy(reinterpret_cast<TfgColorMLP*>(n)); return rc; }
    }
    const int live0 = hc ? M::kHashLive : M::kFreqLive;
    // Uniform (-s, s) initialisation with s = sqrt(6 / (fan_in + fan_out)) per layer.
    std::vector<float> h(nparams, 0.0f);
    uint64_t st = seed ? seed : 0x5EEDull;
    for (int l = 0; l < nl; ++l) {
        const int fan_in = l == 0 ? live0 : width, fan_out = l == nl - 1 ? 3 : width;
        const float sc = std::sqrt(6.0f / (float)(fan_in + fan_out));
        for (int r = 0; r < M::rows_rt(nl, l, width); ++r)
            for (int c = 0; c < M::cols_rt(l, width); ++c) {
                const bool live = !(l == nl - 1 && r >= 3) && !(l == 0 && c >= live0);
                const double u = (double)(tfg::splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
                h[M::poff_rt(nl, l, width) + r * M::cols_rt(l, width) + c] = live ? (float)((2.0 * u - 1.0) * sc) : 0.0f;
            }
    }
    // The weight average starts at zero and is debiased by 1 - decay^t for
    // inference; before the first step inference uses the weights themselves.
    e = cudaMemcpy(n->w, h.data(), pb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(n->ema, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(n->m, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(n->v, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(n->grad, 0, pb);
    if (e != cudaSuccess) { tfgMlpDestroy(reinterpret_cast<TfgColorMLP*>(n)); return tfg::cuda_fail(e, "tfgMlpCreate"); }
    if (int rc = tfg::repack(n, 0, false, 1, false)) { tfgMlpDestroy(reinterpret_cast<TfgColorMLP*>(n)); return rc; }
    static bool attrs = false;
    if (!attrs) {
        set_kernel_attrs<4>();
        set_kernel_attrs<6>();
        set_kernel_attrs<8>();
        attrs = true;
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { tfgMlpDestroy(reinterpret_cast<TfgColorMLP*>(n)); return tfg::cuda_fail(e, "tfgMlpCreate"); }
    *out = reinterpret_cast<TfgColorMLP*>(n);
    return tfg::ok();
}

}  // namespace
}  // namespace tfg

extern "C" int tfgMlpCreateEx(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed, int32_t hidden_layers,
                              TfgColorMLP** out) {
    return tfg::create_model(n_in, n_out, batch, seed, hidden_layers, 64, nullptr, out);
}

extern "C" int tfgMlpCreateHashGrid(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed,
                                    int32_t hidden_layers, const TfgHashGridConfig* config, TfgColorMLP** out) {
    if (!config) return tfg::fail(TFG_E_INVALID, "tfgMlpCreateHashGrid: config is null");
    return tfg::create_model(n_in, n_out, batch, seed, hidden_layers, 64, config, out);
}

extern "C" int tfgMlpCreateWide(uint32_t n_in, uint32_t n_out, uint32_t batch, uint64_t seed, int32_t hidden_layers,
                                int32_t width, const TfgHashGridConfig* config, TfgColorMLP** out) {
    return tfg::create_model(n_in, n_out, batch, seed, hidden_layers, width, config, out);
}

namespace tfg {
namespace mlp {
__global__ void k_one_blob(const float* __restrict__ in, float* __restrict__ out, int32_t n) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float o[kBlobBins];
    one_blob(in[i], o);
#pragma unroll
    for (int b = 0; b < kBlobBins; ++b) out[kBlobBins * i + b] = o[b];
}
}  // namespace mlp
}  // namespace tfg

namespace tfg {
namespace mlp {
// Layer-0 input of the cache kernels, unpacked to floats: 96 features per
// query, each exactly the FP16 / BF16 operand the first GEMM reads.
template <int PREC>
__device__ __forceinline__ void unpack_words(const uint32_t (&w)[48], float* __restrict__ o) {
#pragma unroll
    for (int k = 0; k < 48; ++k) {
        float2 v;
        if constexpr (PREC == kPrecBF16) v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[k]));
        else v = __half22float2(*reinterpret_cast<const __half2*>(&w[k]));
        o[2 * k] = v.x;
        o[2 * k + 1] = v.y;
    }
}

template <int PREC, bool HASH>
__global__ void k_encode_infer(const TfgDatosMLP* __restrict__ in, uint32_t n, Bounds b, HashGrid g,
                               float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t w[48];
    encode_words<PREC, HASH>(in[i], b, g, w);
    unpack_words<PREC>(w, out + 96 * (size_t)i);
}

__global__ void k_encode_train(const TfgDatosMLP* __restrict__ in, uint32_t n, Bounds b, HashGrid g,
                               float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t w[48];
    encode(in[i], b, g, w);
    unpack_words<kPrecF16>(w, out + 96 * (size_t)i);
}
}  // namespace mlp
}  // namespace tfg

extern "C" int tfgMlpEncodeFeatures(TfgColorMLP* h, const TfgDatosMLP* in, uint32_t n, int32_t pass, float* out,
                                    void* stream) {
    ColorMlp* m = reinterpret_cast<ColorMlp*>(h);
    if (!m) return tfg::fail(TFG_E_INVALID, "tfgMlpEncodeFeatures: model is null");
    if (pass != TFG_ENCODE_TRAINING && pass != TFG_ENCODE_INFERENCE)
        return tfg::fail(TFG_E_INVALID, "tfgMlpEncodeFeatures: pass must be TFG_ENCODE_TRAINING or TFG_ENCODE_INFERENCE");
    if (pass == TFG_ENCODE_INFERENCE && m->prec == tfg::mlp::kPrecF8)
        return tfg::fail(TFG_E_INVALID, "tfgMlpEncodeFeatures: FP8 inference scales its features per call; "
                                        "select FP16 or BF16 first");
    if (n == 0) return tfg::ok();
    if (!in || !out) return tfg::fail(TFG_E_INVALID, "tfgMlpEncodeFeatures: null pointer");
    if (int rc = tfg::require_sm100(m->dev)) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned blocks = (n + 127) / 128;
    namespace M = tfg::mlp;
    const M::HashGrid g = tfg::hash_view(m, pass == TFG_ENCODE_TRAINING);
    if (pass == TFG_ENCODE_TRAINING) {
        M::k_encode_train<<<blocks, 128, 0, s>>>(in, n, m->bounds, g, out);
    } else if (m->prec == M::kPrecBF16) {
        if (m->hlevels) M::k_encode_infer<M::kPrecBF16, true><<<blocks, 128, 0, s>>>(in, n, m->bounds, g, out);
        else M::k_encode_infer<M::kPrecBF16, false><<<blocks, 128, 0, s>>>(in, n, m->bounds, g, out);
    } else {
        if (m->hlevels) M::k_encode_infer<M::kPrecF16, true><<<blocks, 128, 0, s>>>(in, n, m->bounds, g, out);
        else M::k_encode_infer<M::kPrecF16, false><<<blocks, 128, 0, s>>>(in, n, m->bounds, g, out);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return tfg::fail((int)e, std::string("tfgMlpEncodeFeatures: ") + cudaGetErrorString(e));
    return tfg::ok();
}

extern "C" int tfgOneBlobBins(const float* values, float* bins, int32_t n, void* stream) {
    if (n < 0) return tfg::fail(TFG_E_INVALID, "tfgOneBlobBins: negative n");
    if (n == 0) return tfg::ok();
    if (!values || !bins) return tfg::fail(TFG_E_INVALID, "tfgOneBlobBins: null pointer");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return tfg::fail((int)e, cudaGetErrorString(e));
    if (int rc = tfg::require_sm100(dev)) return rc;
    tfg::mlp::k_one_blob<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(values, bins, n);
    e = cudaGetLastError();
    if (e != cudaSuccess) return tfg::fail((int)e, std::string("tfgOneBlobBins: ") + cudaGetErrorString(e));
    return tfg::ok();
}

extern "C" int64_t tfgMlpHashParamCount(const TfgColorMLP* h) {
    const ColorMlp* n = reinterpret_cast<const ColorMlp*>(h);
    return n ? (int64_t)n->hcount : 0;
}

extern "C" int tfgMlpGetHashParams(TfgColorMLP* h, int which, float* host, int64_t count) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !host || !n->hlevels || count != (int64_t)n->hcount)
        return tfg::fail(TFG_E_INVALID, "tfgMlpGetHashParams: bad argument");
    const float* src = which == 0 ? n->hw : which == 1 ? n->hema : which == 2 ? n->hm : which == 3 ? n->hv : nullptr;
    if (!src) return tfg::fail(TFG_E_INVALID, "tfgMlpGetHashParams: unknown array");
    cudaError_t e = cudaMemcpy(host, src, n->hcount * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpGetHashParams");
    return tfg::ok();
}

extern "C" int tfgMlpSetHashParams(TfgColorMLP* h, const float* host, int64_t count) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !host || !n->hlevels || count != (int64_t)n->hcount)
        return tfg::fail(TFG_E_INVALID, "tfgMlpSetHashParams: bad argument");
    cudaError_t e = cudaMemcpy(n->hw, host, n->hcount * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpSetHashParams");
    // restart the optimiser of the whole model (tfgMlpSetParams clears the tables' state too)
    std::vector<float> w((size_t)M::params_rt(n->nl, n->hid));
    e = cudaMemcpy(w.data(), n->w, w.size() * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpSetHashParams");
    return tfgMlpSetParams(h, w.data(), (uint32_t)w.size());
}

extern "C" void tfgMlpDestroy(TfgColorMLP* h) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n) return;
    for (void* p : {(void*)n->w, (void*)n->m, (void*)n->v, (void*)n->ema, (void*)n->grad, (void*)n->fwd, (void*)n->bwd,
                    (void*)n->inf, (void*)n->inf_bf, (void*)n->inf_f8, (void*)n->f8, (void*)n->loss, (void*)n->dstate,
                    (void*)n->hw, (void*)n->hm, (void*)n->hv, (void*)n->hema, (void*)n->hgrad, (void*)n->hinf,
                    (void*)n->gate_cells, (void*)n->gate_bits, (void*)n->wpart})
        if (p) cudaFree(p);
    for (int l = 0; l < M::kMaxLayers; ++l) {
        if (n->hT[l]) cudaFree(n->hT[l]);
        if (n->zT[l]) cudaFree(n->zT[l]);
    }
    delete n;
}

extern "C" int tfgMlpSetBounds(TfgColorMLP* h, const TfgSceneBounds* b) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !b) return tfg::fail(TFG_E_INVALID, "tfgMlpSetBounds: null argument");
    n->bounds = M::Bounds{{(float)b->min.x, (float)b->min.y, (float)b->min.z}, {(float)b->max.x, (float)b->max.y, (float)b->max.z}};
    return tfg::ok();
}

extern "C" int tfgMlpSetHyperparams(TfgColorMLP* h, float lr, float beta1, float beta2, float eps, float ema_decay) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !(lr > 0.0f) || !(beta1 >= 0.0f && beta1 < 1.0f) || !(beta2 >= 0.0f && beta2 < 1.0f) || !(eps >= 0.0f) ||
        !(ema_decay >= 0.0f && ema_decay < 1.0f))
        return tfg::fail(TFG_E_INVALID, "tfgMlpSetHyperparams: value out of range");
    n->lr = lr; n->beta1 = beta1; n->beta2 = beta2; n->eps = eps; n->decay = ema_decay;
    return tfg::ok();
}

extern "C" int tfgMlpInference(TfgColorMLP* h, const TfgDatosMLP* in, TfgColor* out, uint32_t count, void* stream) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || (count && (!in || !out))) return tfg::fail(TFG_E_INVALID, "tfgMlpInference: null argument");
    return tfg::infer_impl(n, in, out, nullptr, nullptr, count, nullptr, (cudaStream_t)stream);
}

extern "C" int tfgMlpSetPrecision(TfgColorMLP* h, int32_t precision) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n) return tfg::fail(TFG_E_INVALID, "tfgMlpSetPrecision: null model");
    if (precision != TFG_MLP_FP16 && precision != TFG_MLP_BF16 && precision != TFG_MLP_FP8)
        return tfg::fail(TFG_E_INVALID, "tfgMlpSetPrecision: unknown precision");
    n->prec = precision;
    return tfg::ok();
}

extern "C" int tfgMlpTuningSet(TfgColorMLP* h, const TfgMlpTuning* t) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !t) return tfg::fail(TFG_E_INVALID, "tfgMlpTuningSet: null argument");
    if (t->wgrad_tiles_per_cta < 0 || t->wgrad_tiles_per_cta > 4096)
        return tfg::fail(TFG_E_INVALID, "tfgMlpTuningSet: wgrad_tiles_per_cta must be in [0, 4096]");
    if (t->infer_ctas < 0 || t->infer_ctas > 4096)
        return tfg::fail(TFG_E_INVALID, "tfgMlpTuningSet: infer_ctas must be in [0, 4096]");
    n->tune = *t;
    ++n->tune_generation;
    return tfg::ok();
}

extern "C" int tfgMlpTuningGet(TfgColorMLP* h, TfgMlpTuning* out) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !out) return tfg::fail(TFG_E_INVALID, "tfgMlpTuningGet: null argument");
    *out = n->tune;
    return tfg::ok();
}

extern "C" int tfgMlpAutotune(TfgColorMLP* h, const TfgDatosMLP* in, uint32_t count, TfgColor* out, int32_t repeats,
                              TfgMlpTuning* result, float* ms_out, void* stream) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n) return tfg::fail(TFG_E_INVALID, "tfgMlpAutotune: null model");
    return tfg::autotune_impl(n, in, count, out, repeats, result, ms_out, (cudaStream_t)stream);
}

extern "C" int tfgMlpCalibrate(TfgColorMLP* h, const TfgDatosMLP* in, uint32_t count, void* stream) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !in) return tfg::fail(TFG_E_INVALID, "tfgMlpCalibrate: null argument");
    return tfg::calibrate_impl(n, in, count, (cudaStream_t)stream);
}

extern "C" int tfgMlpInferenceComposite(TfgColorMLP* h, const TfgDatosMLP* in, const TfgColor* throughput,
                                        TfgColor* img, uint32_t count, void* stream) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || (count && (!in || !throughput || !img)))
        return tfg::fail(TFG_E_INVALID, "tfgMlpInferenceComposite: null argument");
    return tfg::infer_impl(n, in, nullptr, img, throughput, count, nullptr, (cudaStream_t)stream);
}

extern "C" int tfgMlpTrainStep(TfgColorMLP* h, const TfgDatosMLP* buffer, uint32_t n_available, float* loss_out,
                               void* stream) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !buffer) return tfg::fail(TFG_E_INVALID, "tfgMlpTrainStep: null argument");
    if (loss_out) *loss_out = 0.0f;
    if (n_available < 100) return tfg::ok();   // mlp.cpp:96: too few samples, no step
    cudaStream_t s = (cudaStream_t)stream;
    if (int rc = tfg::mlp_prepare(n)) return rc;
    if (int rc = tfg::enqueue_step(n, buffer, 100, true, s, n_available)) return rc;
    if (loss_out) {
        float l = 0.0f;
        cudaError_t e = cudaMemcpyAsync(&l, n->loss, sizeof(float), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpTrainStep: loss");
        *loss_out = l / (3.0f * (float)n->batch);
        if (int rc = tfg::check_error_flag()) return rc;
    }
    return tfg::ok();
}

extern "C" int tfgMlpGetParams(TfgColorMLP* h, int which, float* host, uint32_t count) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !host || count != (uint32_t)M::params_rt(n->nl, n->hid))
        return tfg::fail(TFG_E_INVALID, "tfgMlpGetParams: bad argument");
    const float* src = which == 0 ? n->w : which == 1 ? n->ema : which == 2 ? n->m : which == 3 ? n->v : nullptr;
    if (!src) return tfg::fail(TFG_E_INVALID, "tfgMlpGetParams: unknown array");
    cudaError_t e = cudaMemcpy(host, src, count * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpGetParams");
    return tfg::ok();
}

extern "C" int tfgMlpSetParams(TfgColorMLP* h, const float* host, uint32_t count) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !host || count != (uint32_t)M::params_rt(n->nl, n->hid))
        return tfg::fail(TFG_E_INVALID, "tfgMlpSetParams: bad argument");
    const size_t pb = count * sizeof(float);
    cudaError_t e = cudaMemcpy(n->w, host, pb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(n->ema, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(n->m, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(n->v, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(n->grad, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(n->dstate + M::S_ADAM_T, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(n->dstate + M::S_F8_VER, 0, sizeof(uint32_t));
    if (n->hlevels) {
        const size_t hb = n->hcount * sizeof(float);
        if (e == cudaSuccess) e = cudaMemset(n->hema, 0, hb);
        if (e == cudaSuccess) e = cudaMemset(n->hm, 0, hb);
        if (e == cudaSuccess) e = cudaMemset(n->hv, 0, hb);
        if (e == cudaSuccess) e = cudaMemset(n->hgrad, 0, hb);
    }
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpSetParams");
    if (int rc = tfg::repack(n, 0, false, 1, false)) return rc;
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpSetParams");
    return tfg::ok();
}

extern "C" int tfgMlpComputeGradient(TfgColorMLP* h, const TfgDatosMLP* buffer, uint32_t n_available, uint32_t seed,
                                     float* host_grad, uint32_t count, float* loss_out) {
    return tfgMlpComputeGradientEx(h, buffer, n_available, seed, host_grad, count, nullptr, 0, loss_out);
}

extern "C" int tfgMlpComputeGradientEx(TfgColorMLP* h, const TfgDatosMLP* buffer, uint32_t n_available, uint32_t seed,
                                       float* host_grad, uint32_t count, float* host_table_grad, int64_t table_count,
                                       float* loss_out) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !buffer || !host_grad || count != (uint32_t)M::params_rt(n->nl, n->hid) || n_available == 0)
        return tfg::fail(TFG_E_INVALID, "tfgMlpComputeGradient: bad argument");
    if (host_table_grad && table_count != (int64_t)n->hcount)
        return tfg::fail(TFG_E_INVALID, "tfgMlpComputeGradientEx: table_count differs from tfgMlpHashParamCount");
    if (int rc = tfg::mlp_prepare(n)) return rc;
    uint32_t saved[M::S_WORDS];
    cudaError_t e = cudaMemcpy(saved, n->dstate, sizeof(saved), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(n->grad, 0, count * sizeof(float));
    if (e == cudaSuccess && n->hlevels) e = cudaMemset(n->hgrad, 0, n->hcount * sizeof(float));
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpComputeGradient");
    if (int rc = tfg::set_word(n, M::S_NAVAIL, n_available, 0)) return rc;
    if (int rc = tfg::set_word(n, M::S_STEP, seed, 0)) return rc;
    if (int rc = tfg::enqueue_step(n, buffer, 1, false, 0)) return rc;
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpComputeGradient");
    if (int rc = tfg::check_error_flag()) return rc;
    std::vector<float> g(count);
    float l = 0.0f;
    e = cudaMemcpy(g.data(), n->grad, count * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&l, n->loss, sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(n->grad, 0, count * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(n->dstate, saved, sizeof(saved), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpComputeGradient");
    const float sc = 1.0f / (3.0f * (float)n->batch);
    for (uint32_t i = 0; i < count; ++i) host_grad[i] = g[i] * sc;
    if (n->hlevels) {
        if (host_table_grad) {
            e = cudaMemcpy(host_table_grad, n->hgrad, n->hcount * sizeof(float), cudaMemcpyDeviceToHost);
            for (size_t i = 0; e == cudaSuccess && i < n->hcount; ++i) host_table_grad[i] *= sc;
        }
        if (e == cudaSuccess) e = cudaMemset(n->hgrad, 0, n->hcount * sizeof(float));
        if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpComputeGradientEx");
    }
    if (loss_out) *loss_out = l * sc;
    return tfg::ok();
}

extern "C" int32_t tfgMlpParamCount(const TfgColorMLP* h) {
    const ColorMlp* n = reinterpret_cast<const ColorMlp*>(h);
    return n ? M::params_rt(n->nl, n->hid) : 0;
}

// ------------------------------------------------------------------ checkpoints
// The reference saves tiny-cuda-nn's serialised trainer (weights and
// optimiser state, mlp.cpp:173-194) and reloads it for reconstruction
// (mlp.cpp:196-276).  Here a checkpoint is one little-endian binary file:
// 8-byte magic "TFGNRC01", u32 version 1, i32 hidden layers, u32 parameter
// count, f32 bounds[6], f32 lr / beta1 / beta2 / eps / decay, u32 state[8]
// (step, Adam t, ...), then the FP32 weights, weight average, Adam m and v.
namespace {
constexpr char kCkptMagic[8] = {'T', 'F', 'G', 'N', 'R', 'C', '0', '1'};
}

extern "C" int tfgMlpSave(TfgColorMLP* h, const char* path) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !path) return tfg::fail(TFG_E_INVALID, "tfgMlpSave: null argument");
    const uint32_t np = (uint32_t)M::params_rt(n->nl, n->hid);
    std::vector<float> arrays[4];
    uint32_t st[M::S_WORDS];
    const float* src[4] = {n->w, n->ema, n->m, n->v};
    cudaError_t e = cudaDeviceSynchronize();
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
        arrays[k].resize(np);
        e = cudaMemcpy(arrays[k].data(), src[k], np * sizeof(float), cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess) e = cudaMemcpy(st, n->dstate, sizeof(st), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpSave");
    FILE* f = std::fopen(path, "wb");
    if (!f) return tfg::fail(TFG_E_INVALID, std::string("tfgMlpSave: cannot open ") + path);
    // version 1: frequency encoding; version 2 adds the composite encoding's
    // table description and its four table arrays
    const uint32_t version = n->hlevels ? 2 : 1;
    const int32_t hidden = n->nl - 1;
    const float hyper[5] = {n->lr, n->beta1, n->beta2, n->eps, n->decay};
    bool good = std::fwrite(kCkptMagic, 1, 8, f) == 8 && std::fwrite(&version, 4, 1, f) == 1 &&
                std::fwrite(&hidden, 4, 1, f) == 1 && std::fwrite(&np, 4, 1, f) == 1 &&
                std::fwrite(n->bounds.lo, 4, 3, f) == 3 && std::fwrite(n->bounds.hi, 4, 3, f) == 3 &&
                std::fwrite(hyper, 4, 5, f) == 5 && std::fwrite(st, 4, M::S_WORDS, f) == (size_t)M::S_WORDS;
    for (int k = 0; k < 4 && good; ++k) good = std::fwrite(arrays[k].data(), 4, np, f) == np;
    if (good && n->hlevels) {
        const int32_t lv = n->hlevels;
        const uint64_t cnt = n->hcount;
        good = std::fwrite(&lv, 4, 1, f) == 1 && std::fwrite(&n->hT_entries, 4, 1, f) == 1 &&
               std::fwrite(n->hres, 4, M::kHashMaxLevels, f) == (size_t)M::kHashMaxLevels && std::fwrite(&cnt, 8, 1, f) == 1;
        const float* tsrc[4] = {n->hw, n->hema, n->hm, n->hv};
        std::vector<float> buf(n->hcount);
        for (int k = 0; k < 4 && good; ++k) {
            good = cudaMemcpy(buf.data(), tsrc[k], n->hcount * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess &&
                   std::fwrite(buf.data(), 4, n->hcount, f) == n->hcount;
        }
    }
    if (std::fclose(f) != 0 || !good) return tfg::fail(TFG_E_INVALID, std::string("tfgMlpSave: write failed: ") + path);
    return tfg::ok();
}

extern "C" int tfgMlpLoad(TfgColorMLP* h, const char* path) {
    ColorMlp* n = reinterpret_cast<ColorMlp*>(h);
    if (!n || !path) return tfg::fail(TFG_E_INVALID, "tfgMlpLoad: null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return tfg::fail(TFG_E_INVALID, std::string("tfgMlpLoad: cannot open ") + path);
    char magic[8];
    uint32_t version = 0, np = 0;
    int32_t hidden = 0;
    float lo[3], hi[3], hyper[5];
    uint32_t st[M::S_WORDS];
    const uint32_t want_version = n->hlevels ? 2 : 1;
    bool good = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kCkptMagic, 8) == 0 &&
                std::fread(&version, 4, 1, f) == 1 && version == want_version && std::fread(&hidden, 4, 1, f) == 1 &&
                std::fread(&np, 4, 1, f) == 1 && std::fread(lo, 4, 3, f) == 3 && std::fread(hi, 4, 3, f) == 3 &&
                std::fread(hyper, 4, 5, f) == 5 && std::fread(st, 4, M::S_WORDS, f) == (size_t)M::S_WORDS;
    if (!good) {
        std::fclose(f);
        return tfg::fail(TFG_E_INVALID, std::string("tfgMlpLoad: not a cache checkpoint: ") + path);
    }
    if (hidden != n->nl - 1 || np != (uint32_t)M::params_rt(n->nl, n->hid)) {
        std::fclose(f);
        return tfg::fail(TFG_E_INVALID, "tfgMlpLoad: the checkpoint's network depth differs from this model's");
    }
    std::vector<float> arrays[4];
    for (int k = 0; k < 4 && good; ++k) {
        arrays[k].resize(np);
        good = std::fread(arrays[k].data(), 4, np, f) == np;
    }
    std::vector<float> tables[4];
    if (good && n->hlevels) {
        int32_t lv = 0;
        uint32_t T = 0;
        float res[M::kHashMaxLevels];
        uint64_t cnt = 0;
        good = std::fread(&lv, 4, 1, f) == 1 && std::fread(&T, 4, 1, f) == 1 &&
               std::fread(res, 4, M::kHashMaxLevels, f) == (size_t)M::kHashMaxLevels && std::fread(&cnt, 8, 1, f) == 1;
        if (good && (lv != n->hlevels || T != n->hT_entries || cnt != n->hcount ||
                     std::memcmp(res, n->hres, sizeof(res)) != 0)) {
            std::fclose(f);
            return tfg::fail(TFG_E_INVALID, "tfgMlpLoad: the checkpoint's hash-grid tables differ from this model's");
        }
        for (int k = 0; k < 4 && good; ++k) {
            tables[k].resize(n->hcount);
            good = std::fread(tables[k].data(), 4, n->hcount, f) == n->hcount;
        }
    }
    std::fclose(f);
    if (!good) return tfg::fail(TFG_E_INVALID, std::string("tfgMlpLoad: truncated checkpoint: ") + path);
    float* dst[4] = {n->w, n->ema, n->m, n->v};
    cudaError_t e = cudaDeviceSynchronize();
    for (int k = 0; k < 4 && e == cudaSuccess; ++k)
        e = cudaMemcpy(dst[k], arrays[k].data(), np * sizeof(float), cudaMemcpyHostToDevice);
    st[M::S_F8_VER] = 0;   // the FP8 image is re-packed on its next use
    if (e == cudaSuccess) e = cudaMemcpy(n->dstate, st, sizeof(st), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(n->grad, 0, np * sizeof(float));
    if (n->hlevels) {
        float* tdst[4] = {n->hw, n->hema, n->hm, n->hv};
        for (int k = 0; k < 4 && e == cudaSuccess; ++k)
            e = cudaMemcpy(tdst[k], tables[k].data(), n->hcount * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(n->hgrad, 0, n->hcount * sizeof(float));
    }
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpLoad");
    n->bounds = M::Bounds{{lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}};
    n->lr = hyper[0]; n->beta1 = hyper[1]; n->beta2 = hyper[2]; n->eps = hyper[3]; n->decay = hyper[4];
    if (int rc = tfg::repack(n, 0, false, 1, false)) return rc;   // operand images of the loaded arrays
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpLoad");
    return tfg::ok();
}

// Diagnostic for the failure path: one thread waits on an mbarrier that
// nothing arrives on, with the given limit, through the same bounded wait the
// cache kernels use; on giving up it sets the same error flag.
__global__ void k_selftest_wait(uint64_t limit_ns) {
    __shared__ uint64_t mb;
    if (threadIdx.x != 0) return;
    tfg::umma::mbar_init(&mb, 1);
    tfg::umma::mbar_fence_init();
    if (!tfg::umma::mbar_wait(&mb, 0, limit_ns)) atomicExch(&M::g_mlp_error, 1);
}

extern "C" int tfgMlpSelfTestWait(uint32_t timeout_us) {
    if (timeout_us == 0 || timeout_us > 2000000u)
        return tfg::fail(TFG_E_INVALID, "tfgMlpSelfTestWait: timeout must be in (0, 2 s]");
    k_selftest_wait<<<1, 32>>>((uint64_t)timeout_us * 1000ull);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return tfg::cuda_fail(e, "tfgMlpSelfTestWait");
    return tfg::check_error_flag();
}

extern "C" int tfgMlpStatus(void) {
    return tfg::check_error_flag();
}
