// Compressed-wide-BVH traversal (Ylitie, Karras, Laine 2017, Alg. 1) over the
// 80-byte node layout documented in cwbvh_build.cpp.  Semantics match the
// reference traversal (traverse_cwbvh.cuh:51-257): children are visited in
// descending octant-permuted slot order, a node's leaf triangles are tested
// as soon as the node is decoded (highest triangle bit first), a triangle is
// accepted when 0 < t < t_current, and ties keep the first one found.  So on
// the same BVH and triangle layout the closest-hit ids agree bit for bit,
// except on edge hits of rays lying exactly in an axis plane (next list).
//
// Differences are in mechanics, not results:
//  * a direction component of exactly zero takes a finite reciprocal of the
//    zero's sign in the slab tests (slab_rcp), where 1/0 = infinity turned
//    into NaN and stopped that axis from culling boxes; such a ray counts as
//    moving infinitesimally to that side, so when it lies exactly in a plane
//    through mesh edges it can find the triangle on the other side of an edge
//    it hits, or none of the two, where the reference found one;
//  * the traversal stack keeps its top kSmemStack entries in shared memory
//    (one column per thread, conflict-free) and spills deeper entries to a
//    small local array, instead of a 64-entry local-memory stack;
//  * child hit bits are built with a SWAR decode of the meta bytes and
//    plain shifts (no video instructions);
//  * an any-hit variant stops at the first accepted triangle (shadow rays);
//  * a watertight triangle test (Woop, Benthin, Wald 2013) is available over
//    the 48-byte vertex layout, in addition to the reference's transform test.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pt_common.cuh"

namespace tfg {

constexpr int kStackTotal = 64;   // same depth bound as the reference (traverse_cwbvh.cuh:4)
constexpr int kSmemStack = 12;    // entries per thread kept in shared memory
// Upper bound on node visits per ray.  A valid CWBVH never comes close (each
// node is decoded at most once per ray); the bound only keeps a corrupt
// caller-supplied BVH from looping forever.
constexpr uint32_t kMaxNodeVisits = 1u << 22;

// Per-thread traversal stack: shared-memory column + local spill.
struct TravStack {
    uint2* smem;      // base of this block's shared stack, [kSmemStack][blockDim.x]
    int stride;       // blockDim.x
    int tid;
    uint2 spill[kStackTotal - kSmemStack];

    __device__ __forceinline__ void put(uint32_t sp, uint2 v) {
        if (sp < (uint32_t)kSmemStack) smem[sp * stride + tid] = v;
        else spill[sp - kSmemStack] = v;
    }
    __device__ __forceinline__ uint2 get(uint32_t sp) const {
        return sp < (uint32_t)kSmemStack ? smem[sp * stride + tid] : spill[sp - kSmemStack];
    }
};

__device__ __forceinline__ uint32_t msb_index(uint32_t v) { return 31u - (uint32_t)__clz(v); }

// Reciprocal of a direction component for the slab tests.  An exactly zero
// component gets +-2^100 (the zero's sign) instead of +-infinity: with
// infinity, a child plane at the node origin gives 0 * infinity = NaN, the
// min / max chain then drops that axis from the box test, and a ray lying in
// an axis plane decodes every box it passes near (one camera ray of the
// 1080p bench frame: 382 nodes instead of 7).  A power of two keeps the
// scaled products exact, so such a ray is culled by the same rounded slab
// arithmetic as any other; the triangle tests use the direction itself.
__device__ __forceinline__ float slab_rcp(float d) { return d != 0.0f ? 1.0f / d : copysignf(0x1p100f, d); }
// Byte k of w as a float.
__device__ __forceinline__ float byte_f(uint32_t w, int k) { return (float)((w >> (8 * k)) & 0xFFu); }

// Per-ray constants of the watertight test: permutation and shear.
struct WtRay {
    int kx, ky, kz;
    float Sx, Sy, Sz;
};

__device__ __forceinline__ float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

__device__ __forceinline__ WtRay wt_setup(V3 D) {
    WtRay r;
    float ax = fabsf(D.x), ay = fabsf(D.y), az = fabsf(D.z);
    r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    r.kx = r.kz == 2 ? 0 : r.kz + 1;
    r.ky = r.kx == 2 ? 0 : r.kx + 1;
    if (comp(D, r.kz) < 0.0f) { int t = r.kx; r.kx = r.ky; r.ky = t; }
    float dz = comp(D, r.kz);
    r.Sx = comp(D, r.kx) / dz;
    r.Sy = comp(D, r.ky) / dz;
    r.Sz = 1.0f / dz;
    return r;
}

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013).  Edge
// functions are evaluated without contraction so that a shared edge gives
// exactly opposite values in its two triangles; a zero edge value is
// re-evaluated in FP64 as the paper prescribes.  Returns the hit when
// tmin < t < tmax; u, v are the weights of v1 and v2.
__device__ __forceinline__ bool wt_hit(const float4* __restrict__ tw, uint32_t k, V3 O, const WtRay& r, float tmin,
                                       float tmax, float& t, float& u, float& v) {
    float4 a4 = __ldg(&tw[3 * k + 0]);
    float4 b4 = __ldg(&tw[3 * k + 1]);
    float4 c4 = __ldg(&tw[3 * k + 2]);
    V3 A = v3(a4.x, a4.y, a4.z) - O;
    V3 B = v3(b4.x, b4.y, b4.z) - O;
    V3 C = v3(c4.x, c4.y, c4.z) - O;
    float Az = comp(A, r.kz), Bz = comp(B, r.kz), Cz = comp(C, r.kz);
    float Ax = fmaf(-r.Sx, Az, comp(A, r.kx));
    float Ay = fmaf(-r.Sy, Az, comp(A, r.ky));
    float Bx = fmaf(-r.Sx, Bz, comp(B, r.kx));
    float By = fmaf(-r.Sy, Bz, comp(B, r.ky));
    float Cx = fmaf(-r.Sx, Cz, comp(C, r.kx));
    float Cy = fmaf(-r.Sy, Cz, comp(C, r.ky));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float Vv = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || Vv == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        Vv = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || Vv < 0.0f || W < 0.0f) && (U > 0.0f || Vv > 0.0f || W > 0.0f)) return false;
    float det = U + Vv + W;
    if (det == 0.0f) return false;
    Az *= r.Sz; Bz *= r.Sz; Cz *= r.Sz;
    float T = U * Az + Vv * Bz + W * Cz;
    float rcp = 1.0f / det;
    float tt = T * rcp;
    if (!(tt > tmin) || !(tt < tmax)) return false;
    t = tt;
    u = Vv * rcp;
    v = W * rcp;
    return true;
}

// Reference transform test (traverse_cwbvh.cuh:189-209): plane row then the
// two barycentric rows of the world-to-triangle transform.
__device__ __forceinline__ bool ref_hit(const float4* __restrict__ tr, uint32_t addr, V3 O, V3 D, float tmin,
                                        float tmax, float& t, float& u, float& v, uint32_t& id) {
    const float4 T2 = __ldg(&tr[addr + 2]);
    const float transS = T2.x * O.x + T2.y * O.y + T2.z * O.z + T2.w;
    const float transD = T2.x * D.x + T2.y * D.y + T2.z * D.z;
    const float d = -transS / transD;
    if (d <= tmin || d >= tmax) return false;
    const float4 T0 = __ldg(&tr[addr + 0]);
    const float4 T1 = __ldg(&tr[addr + 1]);
    const V3 I = v3(O.x + d * D.x, O.y + d * D.y, O.z + d * D.z);
    const float uu = T0.x * I.x + T0.y * I.y + T0.z * I.z + T0.w;
    const float vv = T1.x * I.x + T1.y * I.y + T1.z * I.z + T1.w;
    if (uu >= 0.0f && vv >= 0.0f && uu + vv < 1.0f) {
        t = d; u = uu; v = vv;
        id = __float_as_uint(__ldg(&tr[addr + 3]).w);
        return true;
    }
    return false;
}

// Decode one node and return its child hit mask: bits 24..31 = inner children
// in octant-permuted order, bits 0..23 = leaf triangles relative to the node's
// triangle base.  Also returns the node's child base, triangle base and imask.
__device__ __forceinline__ uint32_t decode_node(const float4* __restrict__ nodes, uint32_t node, V3 O, V3 rD,
                                                uint32_t octinv, float tmax, uint32_t& child_base,
                                                uint32_t& tri_base, uint32_t& imask) {
    const float4 n0 = __ldg(&nodes[5 * node + 0]);
    const float4 n1 = __ldg(&nodes[5 * node + 1]);
    const float4 n2 = __ldg(&nodes[5 * node + 2]);
    const float4 n3 = __ldg(&nodes[5 * node + 3]);
    const float4 n4 = __ldg(&nodes[5 * node + 4]);
    const uint32_t ew = __float_as_uint(n0.w);
    child_base = __float_as_uint(n1.x);
    tri_base = __float_as_uint(n1.y);
    imask = ew >> 24;
    // 2^e per axis from the signed exponent bytes.
    const float sx = __uint_as_float((uint32_t)((int)(int8_t)(ew & 0xFF) + 127) << 23);
    const float sy = __uint_as_float((uint32_t)((int)(int8_t)((ew >> 8) & 0xFF) + 127) << 23);
    const float sz = __uint_as_float((uint32_t)((int)(int8_t)((ew >> 16) & 0xFF) + 127) << 23);
    const float idx = sx * rD.x, idy = sy * rD.y, idz = sz * rD.z;
    const float ox = (n0.x - O.x) * rD.x, oy = (n0.y - O.y) * rD.y, oz = (n0.z - O.z) * rD.z;
    const bool nx = rD.x < 0.0f, ny = rD.y < 0.0f, nz = rD.z < 0.0f;
    // Near / far quantised planes per axis (swap lo and hi for negative directions).
    const uint32_t qw[2][6] = {
        {__float_as_uint(n2.x), __float_as_uint(n2.z), __float_as_uint(n3.x), __float_as_uint(n3.z),
         __float_as_uint(n4.x), __float_as_uint(n4.z)},
        {__float_as_uint(n2.y), __float_as_uint(n2.w), __float_as_uint(n3.y), __float_as_uint(n3.w),
         __float_as_uint(n4.y), __float_as_uint(n4.w)}};
    uint32_t hitmask = 0;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const uint32_t m4 = __float_as_uint(half == 0 ? n1.z : n1.w);
        const uint32_t inner4 = (m4 & (m4 << 1)) & 0x10101010u;
        const uint32_t bidx4 = (m4 ^ ((inner4 >> 4) * octinv)) & 0x1F1F1F1Fu;
        const uint32_t cbit4 = (m4 >> 5) & 0x07070707u;
        const uint32_t lox = nx ? qw[half][3] : qw[half][0], hix = nx ? qw[half][0] : qw[half][3];
        const uint32_t loy = ny ? qw[half][4] : qw[half][1], hiy = ny ? qw[half][1] : qw[half][4];
        const uint32_t loz = nz ? qw[half][5] : qw[half][2], hiz = nz ? qw[half][2] : qw[half][5];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float tn = fmaxf(fmaxf(fmaxf(fmaf(byte_f(lox, k), idx, ox), fmaf(byte_f(loy, k), idy, oy)),
                                         fmaf(byte_f(loz, k), idz, oz)), 0.0f);
            const float tf = fminf(fminf(fminf(fmaf(byte_f(hix, k), idx, ox), fmaf(byte_f(hiy, k), idy, oy)),
                                         fmaf(byte_f(hiz, k), idz, oz)), tmax);
            if (tn <= tf) hitmask |= ((cbit4 >> (8 * k)) & 7u) << ((bidx4 >> (8 * k)) & 31u);
        }
    }
    return hitmask;
}

// Work done by one traversal: nodes decoded and triangles tested.
struct TravCounts {
    uint32_t nodes = 0, tris = 0;
};

// Per-ray traversal state, advanced one node at a time by step(): lets a
// persistent kernel give an idle lane a new ray while the other lanes of its
// warp are still traversing.  Closest hit (ANY_HIT = false) or first hit
// (ANY_HIT = true); tmax is the current upper bound (exclusive) and becomes
// the hit distance; id / hu / hv are valid when `found`.
template <int TRI_FMT, bool ANY_HIT>
struct CwbvhRay {
    V3 O, D, rD;
    uint32_t octinv;
    WtRay wr;
    float tmin, tmax, hu, hv;
    uint32_t id;
    bool found;
    uint2 ng;
    uint32_t sp, nsteps, ntris;

    __device__ __forceinline__ void init(V3 O_, V3 D_, float tmin_, float tmax_) {
        O = O_; D = D_; tmin = tmin_; tmax = tmax_;
        rD = v3(slab_rcp(D.x), slab_rcp(D.y), slab_rcp(D.z));
        octinv = 7u - ((D.x < 0.0f ? 4u : 0u) | (D.y < 0.0f ? 2u : 0u) | (D.z < 0.0f ? 1u : 0u));
        if (TRI_FMT == 1) wr = wt_setup(D);
        ng = make_uint2(0u, 0x80000000u);
        sp = 0; nsteps = 0; ntris = 0;
        found = false;
        id = 0; hu = 0.0f; hv = 0.0f;
    }

    // Decode the next inner node, test its triangles and pop the stack when
    // its group is empty.  Returns false once the traversal is complete.
    __device__ __forceinline__ bool step(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                                         TravStack& st) {
        if (nsteps >= kMaxNodeVisits) return false;
        ++nsteps;
        const uint32_t bit = msb_index(ng.y);
        const uint32_t imask_parent = ng.y & 0xFFu;
        ng.y &= ~(1u << bit);
        if (ng.y > 0x00FFFFFFu && sp < (uint32_t)kStackTotal) { st.put(sp, ng); ++sp; }
        const uint32_t slot = (bit - 24u) ^ octinv;
        const uint32_t rel = __popc(imask_parent & ~(0xFFFFFFFFu << slot));
        uint32_t cbase, tbase, imask;
        const uint32_t hm = decode_node(nodes, ng.x + rel, O, rD, octinv, tmax, cbase, tbase, imask);
        ng = make_uint2(cbase, (hm & 0xFF000000u) | imask);
        uint32_t tbits = hm & 0x00FFFFFFu;
        while (tbits) {
            ++ntris;
            const uint32_t k = msb_index(tbits);
            tbits &= ~(1u << k);
            float t, u, v;
            if (TRI_FMT == 0) {
                uint32_t tid;
                if (ref_hit(tris, tbase + 4u * k, O, D, tmin, tmax, t, u, v, tid)) {
                    tmax = t; hu = u; hv = v; id = tid; found = true;
                    if (ANY_HIT) return false;
                }
            } else {
                const uint32_t tri = (tbase >> 2) + k;
                if (wt_hit(tris, tri, O, wr, tmin, tmax, t, u, v)) {
                    tmax = t; hu = u; hv = v; id = __float_as_uint(__ldg(&tris[3 * tri]).w); found = true;
                    if (ANY_HIT) return false;
                }
            }
        }
        if (ng.y <= 0x00FFFFFFu) {
            if (sp == 0) return false;
            --sp;
            ng = st.get(sp);
        }
        return true;
    }
};

// Whole traversal in one call.  tmax in: upper bound (exclusive); out: hit
// distance when found.  Returns true on a hit; id / u / v are written only
// then.  `cnt`, when not null, accumulates the work done.
template <int TRI_FMT, bool ANY_HIT>
__device__ __forceinline__ bool cwbvh_trace(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                                            V3 O, V3 D, float tmin, float& tmax, uint32_t& id, float& hu,
                                            float& hv, TravStack& st, TravCounts* cnt) {
    CwbvhRay<TRI_FMT, ANY_HIT> r;
    r.init(O, D, tmin, tmax);
    while (r.step(nodes, tris, st)) {
    }
    if (cnt) { cnt->nodes += r.nsteps; cnt->tris += r.ntris; }
    if (!r.found) return false;
    tmax = r.tmax; id = r.id; hu = r.hu; hv = r.hv;
    return true;
}

}  // namespace tfg
