// Measurement kernels for the roofline of the traversal stages.
//
// The CWBVH of the benchmark scene (95,716 nodes of 80 B plus 48 MB of
// watertight triangles) sits in the 126 MB L2, and a traversal step reads
// one 80-byte node (five 16-byte loads) at an address no neighbouring lane
// shares.  A streaming copy does not bound that access pattern; this kernel
// does: every thread reads `reads` records of 80 bytes at hashed, independent
// indices of an L2-resident table (five 16-byte loads each, all in flight
// together) and folds them into one word, so the bytes it moves per second
// are the random-gather bandwidth of L2 that traversal can at best reach.
#include <cuda_runtime.h>

#include <string>

#include "../../include/tfg_pt.h"
#include "tfg_errors.h"
#include "tfg_runtime.h"

namespace tfg {
namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    // integer finaliser of MurmurHash3: decorrelates consecutive indices
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(256) k_l2_gather(const float4* __restrict__ table, uint32_t records, uint32_t reads,
                                                   uint32_t seed, uint32_t* __restrict__ sink) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
#pragma unroll 4
    for (uint32_t k = 0; k < reads; ++k) {
        const uint32_t r = mix32(seed ^ mix32(tid * 0x9E3779B1u + k)) % records;
        const float4* p = table + 5 * (size_t)r;
        float4 v[5];
#pragma unroll
        for (int j = 0; j < 5; ++j) v[j] = __ldg(p + j);
#pragma unroll
        for (int j = 0; j < 5; ++j)
            acc ^= __float_as_uint(v[j].x) ^ __float_as_uint(v[j].y) ^ __float_as_uint(v[j].z) ^ __float_as_uint(v[j].w);
    }
    if (acc == 0x7FFFFFFFu) sink[0] = acc;   // keeps the loads; the word itself is never read
}

}  // namespace
}  // namespace tfg

extern "C" int tfgL2GatherPass(const void* table, uint32_t records, uint32_t reads_per_thread, uint32_t seed,
                               uint32_t* sink, int32_t blocks, void* stream) {
    using namespace tfg;
    if (!table || !sink || records == 0 || reads_per_thread == 0 || blocks <= 0)
        return fail(TFG_E_INVALID, "tfgL2GatherPass: bad argument");
    if ((reinterpret_cast<uintptr_t>(table) & 15u) != 0)
        return fail(TFG_E_INVALID, "tfgL2GatherPass: table must be 16-byte aligned");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    k_l2_gather<<<blocks, 256, 0, (cudaStream_t)stream>>>(static_cast<const float4*>(table), records, reads_per_thread,
                                                          seed, sink);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail((int)e, std::string("tfgL2GatherPass: ") + cudaGetErrorString(e));
    return ok();
}
