// Final image of a render on the GPU and headless image files.
//
// The reference sums frames on the host, scales the sum by 1 / frames,
// applies its ACES-style "filmic" curve per channel and writes an 8-bit PNG
// (main.cpp:1108-1115, imagen.h:193-214, imagen_utils.h:59-62).  Here the sum
// stays in device memory (k_accumulate in nrc_kernels.cu) and one kernel
// produces both the averaged HDR image and the tone-mapped 8-bit RGB bytes,
// so only the bytes the caller wants cross PCIe.  Files are written as PPM
// (8-bit) and PFM (float) -- formats that need no image library.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/tfg_pt.h"
#include "tfg_errors.h"
#include "tfg_runtime.h"

namespace tfg {
namespace {

// imagen.h:193-204, evaluated in the written order without contraction.
__device__ __forceinline__ float aces_filmic(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    x = __fmul_rn(x, 0.6f);
    const float num = __fmul_rn(x, __fadd_rn(__fmul_rn(a, x), b));
    const float den = __fadd_rn(__fmul_rn(x, __fadd_rn(__fmul_rn(c, x), d)), e);
    const float v = __fdiv_rn(num, den);
    return fminf(fmaxf(v, 0.0f), 1.0f);
}

// imagen_utils.h:59-62: round(clamp(v, 0, 1) * 255), halves away from zero.
__device__ __forceinline__ uint8_t to_byte(float v) {
    return (uint8_t)roundf(__fmul_rn(fminf(fmaxf(v, 0.0f), 1.0f), 255.0f));
}

__global__ void k_tonemap_filmic(const float* __restrict__ sum, float inv, uint32_t n, float* __restrict__ hdr,
                                 uint8_t* __restrict__ rgb8) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float v = __fmul_rn(sum[3 * (size_t)i + k], inv);
            if (hdr) hdr[3 * (size_t)i + k] = v;
            if (rgb8) rgb8[3 * (size_t)i + k] = to_byte(aces_filmic(v));
        }
    }
}

}  // namespace
}  // namespace tfg

extern "C" int tfgToneMapFilmic(const float* accum, int32_t frames, int32_t W, int32_t H, float* hdr_out,
                                uint8_t* rgb8_out, void* stream) {
    using namespace tfg;
    if (!accum || (!hdr_out && !rgb8_out)) return fail(TFG_E_INVALID, "tfgToneMapFilmic: null argument");
    if (W <= 0 || H <= 0 || frames <= 0) return fail(TFG_E_INVALID, "tfgToneMapFilmic: bad size or frame count");
    const uint32_t n = (uint32_t)W * (uint32_t)H;
    const float inv = 1.0f / (float)frames;   // main.cpp:1108
    const uint32_t blocks = std::min<uint32_t>((n + 255) / 256, 148u * 16u);
    k_tonemap_filmic<<<blocks, 256, 0, (cudaStream_t)stream>>>(accum, inv, n, hdr_out, rgb8_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail((int)e, std::string("tfgToneMapFilmic: ") + cudaGetErrorString(e));
    return ok();
}

extern "C" int tfgWritePPM(const char* path, const uint8_t* rgb8, int32_t W, int32_t H) {
    using namespace tfg;
    if (!path || !rgb8 || W <= 0 || H <= 0) return fail(TFG_E_INVALID, "tfgWritePPM: bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(TFG_E_INVALID, std::string("tfgWritePPM: cannot open ") + path);
    std::fprintf(f, "P6\n%d %d\n255\n", W, H);
    const size_t bytes = (size_t)W * H * 3;
    const bool good = std::fwrite(rgb8, 1, bytes, f) == bytes;
    if (std::fclose(f) != 0 || !good) return fail(TFG_E_INVALID, std::string("tfgWritePPM: write failed: ") + path);
    return ok();
}

// PFM: rows bottom to top, negative scale = little-endian floats.
extern "C" int tfgWritePFM(const char* path, const float* rgb, int32_t W, int32_t H) {
    using namespace tfg;
    if (!path || !rgb || W <= 0 || H <= 0) return fail(TFG_E_INVALID, "tfgWritePFM: bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(TFG_E_INVALID, std::string("tfgWritePFM: cannot open ") + path);
    std::fprintf(f, "PF\n%d %d\n-1.0\n", W, H);
    bool good = true;
    for (int y = H - 1; y >= 0 && good; --y)
        good = std::fwrite(rgb + (size_t)y * W * 3, sizeof(float), (size_t)W * 3, f) == (size_t)W * 3;
    if (std::fclose(f) != 0 || !good) return fail(TFG_E_INVALID, std::string("tfgWritePFM: write failed: ") + path);
    return ok();
}
