// C-ABI shim over the reference's own GPU kernels -- TEST INFRASTRUCTURE ONLY.
//
// Compiled together with the unmodified reference sources RenderKernel.cu and
// NrcKernel.cu (from the reference checkout, by oracle/build_oracle.py) into
// oracle/_ref/libtfgref.so.  Tests call it on the GPU to compare the product
// kernels with the reference's kernels on identical inputs.  Nothing in the
// product library links or calls it.
//
// The wrappers only translate plain pointers into the reference's argument
// types (dim3, ImagenGPU and TinyBVHD_GPU by value) and launch on the legacy
// default stream as the reference does (RenderKernel.cu:270).
#include <cstdint>

#include "RenderKernel.h"
#include "NrcKernel.h"
#include "escenario.h"   // pulls in traverse_cwbvh.cuh

__global__ void ref_trace_kernel(const float4* nodes, const float4* tris, const float* rays, int n, float* hits,
                                 uint32_t* steps) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + 8 * (size_t)i;
    const float3 O = make_float3(r[0], r[1], r[2]);
    const float3 D = make_float3(r[4], r[5], r[6]);
    const float3 rD = make_float3(1.0f / D.x, 1.0f / D.y, 1.0f / D.z);
    uint32_t sc = 0;
    float4 h = traverse_cwbvh(nodes, tris, O, D, rD, r[3], &sc);
    // A miss leaves t at t_max (the reference's caller rejects it by t, escenario.h:349).
    uint32_t id = __float_as_uint(h.w);
    if (!(h.x < r[3])) { id = 0xFFFFFFFFu; h.y = 0.0f; h.z = 0.0f; }
    hits[4 * (size_t)i + 0] = h.x;
    hits[4 * (size_t)i + 1] = h.y;
    hits[4 * (size_t)i + 2] = h.z;
    hits[4 * (size_t)i + 3] = __uint_as_float(id);
    if (steps) steps[i] = sc;
}

extern "C" {

int ref_trace(const float* nodes, const float* tris, const float* rays, int n, float* hits, uint32_t* steps) {
    if (n <= 0) return 0;
    ref_trace_kernel<<<(n + 127) / 128, 128>>>(reinterpret_cast<const float4*>(nodes),
                                                reinterpret_cast<const float4*>(tris), rays, n, hits, steps);
    return (int)cudaGetLastError();
}

// launchKernelRenderTiny with a 16x16 block as main.cpp:866-868.  The kernel
// has no x/y bounds guard, so inference/throughput buffers must hold
// ceil(H/16)*16*W + 16 entries.
int ref_render_tiny(const void* camara, const void* prims, int nprims, const void* luces, int nluces, int W, int H,
                    int frame, float* d_nodos, float* d_tris, unsigned num_nodos, unsigned num_tris,
                    const void* bvh_prims, int n_bvh_prims, void* img, void* regs, unsigned* counter, int cap,
                    void* infer, void* thr, int use_inf, int train) {
    dim3 block(16, 16);
    dim3 grid((W + 15) / 16, (H + 15) / 16);
    TinyBVHD_GPU bvh;
    bvh.d_nodos = reinterpret_cast<float4*>(d_nodos);
    bvh.d_tris = reinterpret_cast<float4*>(d_tris);
    bvh.num_nodos = num_nodos;
    bvh.num_tris = num_tris;
    ImagenGPU im(W, H, reinterpret_cast<Color*>(img));
    launchKernelRenderTiny(grid, block, reinterpret_cast<const Camara*>(camara),
                           reinterpret_cast<const Primitiva*>(prims), nprims,
                           reinterpret_cast<const LuzPuntual*>(luces), nluces, nullptr, 0, W, H, 1, frame, bvh,
                           reinterpret_cast<const Primitiva*>(bvh_prims), n_bvh_prims, im, nullptr,
                           reinterpret_cast<RegistroEntrenamiento*>(regs), counter, cap,
                           reinterpret_cast<DatosMLP*>(infer), reinterpret_cast<Color*>(thr), use_inf != 0,
                           train != 0);
    return (int)cudaGetLastError();
}

int ref_camera(void* cam, int W, int H) {
    launchInicializarCamara(reinterpret_cast<Camara*>(cam), W, H);
    return (int)cudaGetLastError();
}

int ref_composite(void* img, void* pred, void* thr, int W, int H) {
    dim3 block(16, 16), grid((W + 15) / 16, (H + 15) / 16);
    launchKernelComposite(grid, block, reinterpret_cast<Color*>(img), reinterpret_cast<Color*>(pred),
                          reinterpret_cast<Color*>(thr), W, H);
    return (int)cudaGetLastError();
}

int ref_targets(void* regs, void* tail, void* out, int n) {
    launchKernelCalcularTargets(dim3((n + 255) / 256), dim3(256), reinterpret_cast<RegistroEntrenamiento*>(regs),
                                reinterpret_cast<Color*>(tail), reinterpret_cast<DatosMLP*>(out), n);
    return (int)cudaGetLastError();
}

int ref_tail(const void* regs, void* out, int n) {
    launchKernelPrepararInferenciaTail(dim3((n + 255) / 256), dim3(256),
                                       reinterpret_cast<const RegistroEntrenamiento*>(regs),
                                       reinterpret_cast<DatosMLP*>(out), n);
    return (int)cudaGetLastError();
}

int ref_indices(int* idx, int max_range, int count, unsigned seed) {
    launchGenerarIndicesAleatorios((count + 255) / 256, 256, 0, idx, max_range, count, seed);
    return (int)cudaGetLastError();
}

int ref_train_rows(const void* buf, const int* idx, int batch, int n_in, int n_out, const void* bounds, float* in,
                   float* tgt) {
    launchPrepararDatosEntrenamiento((batch + 255) / 256, 256, 0, reinterpret_cast<const DatosMLP*>(buf), idx, batch,
                                     n_in, n_out, *reinterpret_cast<const SceneBounds*>(bounds), in, tgt);
    return (int)cudaGetLastError();
}

int ref_infer_rows(const void* datos, unsigned n, unsigned n_in, float* out, const void* bounds) {
    launchPrepararDatosInferencia((n + 255) / 256, 256, 0, reinterpret_cast<const DatosMLP*>(datos), n, n_in, out,
                                  *reinterpret_cast<const SceneBounds*>(bounds));
    return (int)cudaGetLastError();
}

int ref_scrub(float* net, void* out, int n) {
    launchGuardarSalidaInferencia((n + 255) / 256, 256, 0, net, reinterpret_cast<Color*>(out), n);
    return (int)cudaGetLastError();
}

int ref_sync(void) { return (int)cudaDeviceSynchronize(); }

}  // extern "C"
