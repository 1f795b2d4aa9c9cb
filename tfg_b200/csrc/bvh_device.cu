// Device upload of a CWBVH build: the drop-in for TinyBVH::construirBVH and
// its destructor (tinybvh_wrapper.cpp:22-83).  The reference uploads nodes,
// compressed triangles and the triangle primitives in input order; this also
// uploads the 48-byte watertight triangle array built from the same nodes.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/tfg_pt.h"
#include "tfg_errors.h"

extern "C" int tfgTinyBVHConstruir(const TfgPrimitiva* prims, int32_t n, TfgTinyBVH* out) {
    if (!out) return tfg::fail(TFG_E_INVALID, "tfgTinyBVHConstruir: out is null");
    std::memset(out, 0, sizeof(*out));
    if (n < 0 || (n > 0 && !prims)) return tfg::fail(TFG_E_INVALID, "tfgTinyBVHConstruir: bad primitive array");
    std::vector<float> verts;
    std::vector<TfgPrimitiva> tris;
    verts.reserve(9 * (size_t)n);
    for (int32_t i = 0; i < n; ++i) {
        if (prims[i].tipo != TFG_TRIANGULO) continue;
        const auto& t = prims[i].u.triangulo;
        const TfgVec3d* v[3] = {&t.v0, &t.v1, &t.v2};
        for (int k = 0; k < 3; ++k) {
            verts.push_back((float)v[k]->x);
            verts.push_back((float)v[k]->y);
            verts.push_back((float)v[k]->z);
        }
        tris.push_back(prims[i]);
    }
    if (tris.empty()) return tfg::ok();   // the reference leaves an empty BVH too (tinybvh_wrapper.cpp:46-49)
    TfgCWBVHHost h;
    if (int rc = tfgCWBVHBuild(verts.data(), (uint32_t)tris.size(), &h)) return rc;
    const size_t nb = (size_t)h.num_nodes * 80, tb = (size_t)h.num_tris * 64, wb = (size_t)h.num_tris * 48,
                 pb = tris.size() * sizeof(TfgPrimitiva);
    cudaError_t e = cudaMalloc((void**)&out->ref.d_nodos, nb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&out->ref.d_tris, tb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&out->d_tris_wt, wb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&out->d_primitivas, pb);
    if (e == cudaSuccess) e = cudaMemcpy(out->ref.d_nodos, h.nodes, nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(out->ref.d_tris, h.tris_ref, tb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(out->d_tris_wt, h.tris_wt, wb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(out->d_primitivas, tris.data(), pb, cudaMemcpyHostToDevice);
    out->ref.num_nodos = h.num_nodes;
    out->ref.num_tris = h.num_tris;
    out->num_primitivas = (uint32_t)tris.size();
    out->max_depth = h.max_depth;
    tfgCWBVHFree(&h);
    if (e != cudaSuccess) {
        tfgTinyBVHLiberar(out);
        return tfg::fail((int)e, std::string("tfgTinyBVHConstruir: ") + cudaGetErrorString(e));
    }
    return tfg::ok();
}

extern "C" void tfgTinyBVHLiberar(TfgTinyBVH* b) {
    if (!b) return;
    if (b->ref.d_nodos) cudaFree(b->ref.d_nodos);
    if (b->ref.d_tris) cudaFree(b->ref.d_tris);
    if (b->d_tris_wt) cudaFree(b->d_tris_wt);
    if (b->d_primitivas) cudaFree(b->d_primitivas);
    std::memset(b, 0, sizeof(*b));
}
