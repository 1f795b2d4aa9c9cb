// CWBVH build on the GPU, for scenes that change or arrive in batches: the
// same node and triangle layouts as the host builder (cwbvh_build.cpp; the
// layouts the reference traversal decodes, traverse_cwbvh.cuh:77-209), built
// without leaving the device.
//
//   1. compact the TRIANGULO primitives in input order (their index is the
//      prim id, as tinybvh_wrapper.cpp:36-44 numbers them), FP32 vertices;
//   2. 30-bit Morton codes of the triangle centroids, radix-sorted;
//   3. binary radix tree over the sorted codes (Karras 2012, "Maximizing
//      Parallelism in the Construction of BVHs, Octrees, and k-d Trees"),
//      duplicate codes ordered by index;
//   4. boxes and triangle counts bottom-up, one thread per leaf climbing
//      while it is the second child to finish;
//   5. one kernel per wide level: every wide node gathers up to 8 children
//      by opening the largest-area interior child (a subtree of <= 3
//      triangles becomes a leaf slot), assigns octant slots greedily,
//      quantises the child boxes to 8 bits and reserves contiguous blocks
//      for its inner children and leaf triangles with atomics;
//   6. the reference transform triangles and the watertight triangles in
//      leaf order.
// The tree is a Morton-order (LBVH) tree: it builds in milliseconds, and
// traverses slower than the host builder's binned-SAH tree.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/tfg_pt.h"
#include "tfg_errors.h"
#include "tfg_runtime.h"

namespace tfg {
namespace {

constexpr int kMaxLeaf = 3;   // the 3-bit unary meta count limits a leaf to 3 triangles

struct Box6 {
    float lo[3], hi[3];
};

// Collapse plan of a binary node, as in the host builder (cwbvh_build.cpp):
// for a budget of i = 1..8 slots of the wide parent, the least SAH cost of
// the node's subtree and how it is reached (leaf of <= 3 triangles, a wide
// node of its own, as with one slot less, or split with k slots to the left).
struct Plan2 {
    float cost[8];
    uint8_t how[8];
    uint8_t split8;       // as a wide node: slots given to the left child
    uint8_t pad[7];
};
constexpr uint8_t kLeaf = 0, kInternal = 1, kSame = 2, kSplit = 16;
constexpr float kCostWideNode = 1.0f, kCostWideTri = 0.3f;

__device__ __forceinline__ float box_area(const Box6& b) {
    const float dx = fmaxf(b.hi[0] - b.lo[0], 0.0f), dy = fmaxf(b.hi[1] - b.lo[1], 0.0f),
                dz = fmaxf(b.hi[2] - b.lo[2], 0.0f);
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {   // 10 bits -> every third bit
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_flag_triangles(const TfgPrimitiva* __restrict__ p, int n, uint32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flag[i] = p[i].tipo == TFG_TRIANGULO ? 1u : 0u;
}

// Compacted triangles: primitive copy, FP32 vertices, box.
__global__ void k_compact(const TfgPrimitiva* __restrict__ p, int n, const uint32_t* __restrict__ flag,
                          const uint32_t* __restrict__ pos, TfgPrimitiva* __restrict__ tris, float* __restrict__ verts,
                          Box6* __restrict__ box) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!flag[i]) continue;
        const uint32_t k = pos[i];
        tris[k] = p[i];
        const auto& t = p[i].u.triangulo;
        const TfgVec3d* v[3] = {&t.v0, &t.v1, &t.v2};
        Box6 b;
        for (int a = 0; a < 3; ++a) { b.lo[a] = INFINITY; b.hi[a] = -INFINITY; }
        for (int c = 0; c < 3; ++c) {
            const float x[3] = {(float)v[c]->x, (float)v[c]->y, (float)v[c]->z};
            for (int a = 0; a < 3; ++a) {
                verts[9 * (size_t)k + 3 * c + a] = x[a];
                b.lo[a] = fminf(b.lo[a], x[a]);
                b.hi[a] = fmaxf(b.hi[a], x[a]);
            }
        }
        box[k] = b;
    }
}

// Order-preserving float <-> uint mapping for atomic min / max.
__device__ __forceinline__ uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funkey(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__global__ void k_centroid_bounds(const Box6* __restrict__ box, uint32_t n, uint32_t* __restrict__ cb) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            const float c = 0.5f * (box[i].lo[a] + box[i].hi[a]);
            lo[a] = fminf(lo[a], c);
            hi[a] = fmaxf(hi[a], c);
        }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xFFFFFFFFu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xFFFFFFFFu, hi[a], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&cb[a], fkey(lo[a]));
            atomicMax(&cb[3 + a], fkey(hi[a]));
        }
    }
}

__global__ void k_morton(const Box6* __restrict__ box, uint32_t n, const uint32_t* __restrict__ cb,
                         uint32_t* __restrict__ code, uint32_t* __restrict__ idx) {
    float lo[3], inv[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = funkey(cb[a]);
        const float ext = funkey(cb[3 + a]) - lo[a];
        inv[a] = ext > 0.0f ? 1.0f / ext : 0.0f;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            const float c = (0.5f * (box[i].lo[a] + box[i].hi[a]) - lo[a]) * inv[a];
            q[a] = (uint32_t)fminf(fmaxf(c * 1024.0f, 0.0f), 1023.0f);
        }
        code[i] = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
        idx[i] = i;
    }
}

// Binary radix tree: internal nodes 0..n-2, leaf i (sorted position) is node
// n - 1 + i.  child[2i], child[2i+1]; parent of every node.
__device__ __forceinline__ int delta_of(const uint32_t* code, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = code[i], b = code[j];
    return a == b ? 32 + __clz((uint32_t)(i ^ j)) : __clz(a ^ b);
}

__global__ void k_radix_tree(const uint32_t* __restrict__ code, int n, int* __restrict__ child,
                             int* __restrict__ parent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = (delta_of(code, n, i, i + 1) - delta_of(code, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = delta_of(code, n, i, i - d);
        int lmax = 2;
        while (delta_of(code, n, i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (delta_of(code, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = delta_of(code, n, i, j);
        int s = 0;
        for (int t = (l + 1) / 2;; t = (t + 1) / 2) {
            if (delta_of(code, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        const int gamma = i + s * d + min(d, 0);
        const int left = min(i, j) == gamma ? (n - 1 + gamma) : gamma;
        const int right = max(i, j) == gamma + 1 ? (n - 1 + gamma + 1) : gamma + 1;
        child[2 * i] = left;
        child[2 * i + 1] = right;
        parent[left] = i;
        parent[right] = i;
    }
}

// Boxes and triangle counts bottom-up.  A thread stops at the first node whose
// other child is not finished yet; the second thread to arrive continues.
// The plan of binary node p from its area, triangle count and its children's
// plans (C(n, 1) = min(leaf, wide node); C(n, i) = min(C(n, i - 1), D(n, i));
// D(n, j) = min over k of C(left, k) + C(right, j - k)).
__device__ void plan_node(Plan2& P, float area, int count, const Plan2* L, const Plan2* R) {
    float dist[9];
    uint8_t split[9];
    for (int j = 0; j <= 8; ++j) { dist[j] = INFINITY; split[j] = 0; }
    if (L && R) {
        float lc[8], rc[8];
        for (int k = 0; k < 8; ++k) { lc[k] = __ldcg(&L->cost[k]); rc[k] = __ldcg(&R->cost[k]); }
        for (int j = 2; j <= 8; ++j)
            for (int k = 1; k < j; ++k) {
                const float c = lc[k - 1] + rc[j - k - 1];
                if (c < dist[j]) { dist[j] = c; split[j] = (uint8_t)k; }
            }
    }
    const float leaf = count <= kMaxLeaf ? area * (float)count * kCostWideTri : INFINITY;
    const float internal = dist[8] + area * kCostWideNode;
    P.split8 = split[8];
    if (leaf <= internal) { P.cost[0] = leaf; P.how[0] = kLeaf; }
    else { P.cost[0] = internal; P.how[0] = kInternal; }
    for (int i = 2; i <= 8; ++i) {
        if (dist[i] < P.cost[i - 2]) { P.cost[i - 1] = dist[i]; P.how[i - 1] = (uint8_t)(kSplit + split[i]); }
        else { P.cost[i - 1] = P.cost[i - 2]; P.how[i - 1] = kSame; }
    }
}

__global__ void k_refit(const Box6* __restrict__ tbox, const uint32_t* __restrict__ sorted, int n,
                        const int* __restrict__ child, const int* __restrict__ parent, Box6* box, int* count,
                        Plan2* plan, uint32_t* arrivals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int node = n - 1 + i;
        box[node] = tbox[sorted[i]];
        count[node] = 1;
        plan_node(plan[node], box_area(tbox[sorted[i]]), 1, nullptr, nullptr);
        __threadfence();
        while (node != 0) {
            const int p = parent[node];
            if (atomicAdd(&arrivals[p], 1u) == 0u) break;
            __threadfence();
            const int a = child[2 * p], b = child[2 * p + 1];
            Box6 ba, bb, r;
            for (int k = 0; k < 3; ++k) {
                ba.lo[k] = __ldcg(&box[a].lo[k]); ba.hi[k] = __ldcg(&box[a].hi[k]);
                bb.lo[k] = __ldcg(&box[b].lo[k]); bb.hi[k] = __ldcg(&box[b].hi[k]);
                r.lo[k] = fminf(ba.lo[k], bb.lo[k]);
                r.hi[k] = fmaxf(ba.hi[k], bb.hi[k]);
            }
            box[p] = r;
            const int cnt = __ldcg(&count[a]) + __ldcg(&count[b]);
            count[p] = cnt;
            plan_node(plan[p], box_area(r), cnt, &plan[a], &plan[b]);
            __threadfence();
            node = p;
        }
    }
}

struct WideArgs {
    const int* child;
    const Box6* box;
    const int* count;
    const Plan2* plan;
    const uint32_t* sorted;   // sorted position -> compacted triangle index
    int n;                    // triangles
    const int2* q_in;         // (binary node, wide index)
    uint32_t q_n;
    int2* q_out;
    uint32_t* q_out_n;
    uint32_t* next_node;
    uint32_t* next_tri;
    uint32_t* nodes;          // 20 words per wide node
    uint32_t* tri_order;      // leaf order -> compacted triangle index
};

__device__ __forceinline__ bool is_leaf2(int node, int n) { return node >= n - 1; }

__device__ int gather_leaf_tris(const WideArgs& a, int node, uint32_t* out) {
    int stack[8], sp = 0, cnt = 0;
    stack[sp++] = node;
    while (sp > 0 && cnt < kMaxLeaf) {
        const int m = stack[--sp];
        if (is_leaf2(m, a.n)) {
            out[cnt++] = a.sorted[m - (a.n - 1)];
        } else {
            stack[sp++] = a.child[2 * m + 1];
            stack[sp++] = a.child[2 * m];
        }
    }
    return cnt;
}

// One wide node per thread: the host builder's cost-optimal collapse (read
// from the plans), slot assignment and quantisation (cwbvh_build.cpp) on this
// level's queue.
__global__ void k_wide_level(WideArgs a) {
    const uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= a.q_n) return;
    const int node2 = a.q_in[qi].x;
    const uint32_t widx = (uint32_t)a.q_in[qi].y;
    int kid[8];
    bool leaf[8];
    int nk = 0;
    if (is_leaf2(node2, a.n)) {
        kid[0] = node2; leaf[0] = true; nk = 1;
    } else {
        // (binary node, slot budget) pairs, the left child on top; a split
        // pushes two entries and pops one, and the budgets sum to 8, so the
        // stack never holds more than 8
        int sn[8], sb[8], sp = 0;
        const int k8 = a.plan[node2].split8;
        sn[sp] = a.child[2 * node2 + 1]; sb[sp++] = 8 - k8;
        sn[sp] = a.child[2 * node2]; sb[sp++] = k8;
        while (sp > 0 && nk < 8) {
            const int m = sn[--sp];
            int b = sb[sp];
            const Plan2& P = a.plan[m];
            while (b > 1 && P.how[b - 1] == kSame) --b;
            const uint8_t h = P.how[b - 1];
            if (h == kLeaf || h == kInternal) {
                kid[nk] = m; leaf[nk] = h == kLeaf; ++nk;
            } else if (sp + 2 <= 8) {
                const int k = h - kSplit;
                sn[sp] = a.child[2 * m + 1]; sb[sp++] = b - k;
                sn[sp] = a.child[2 * m]; sb[sp++] = k;
            }
        }
    }
    const Box6 pb = a.box[node2];
    // Octant slot assignment, greedy on dot(c_child - c_parent, dir_s).
    double pc[3];
    for (int k = 0; k < 3; ++k) pc[k] = 0.5 * ((double)pb.lo[k] + (double)pb.hi[k]);
    double cost[8][8];
    for (int i = 0; i < nk; ++i) {
        const Box6 cb = a.box[kid[i]];
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = 0.5 * ((double)cb.lo[k] + (double)cb.hi[k]) - pc[k];
        for (int s = 0; s < 8; ++s)
            cost[i][s] = d[0] * ((s & 4) ? -1.0 : 1.0) + d[1] * ((s & 2) ? -1.0 : 1.0) + d[2] * ((s & 1) ? -1.0 : 1.0);
    }
    int slot_of[8], kid_in_slot[8];
    for (int s = 0; s < 8; ++s) { kid_in_slot[s] = -1; slot_of[s] = -1; }
    for (int round = 0; round < nk; ++round) {
        double best = INFINITY;
        int bi = -1, bs = -1;
        for (int i = 0; i < nk; ++i) {
            if (slot_of[i] >= 0) continue;
            for (int s = 0; s < 8; ++s) {
                if (kid_in_slot[s] >= 0) continue;
                if (cost[i][s] < best || bi < 0) { best = cost[i][s]; bi = i; bs = s; }
            }
        }
        slot_of[bi] = bs;
        kid_in_slot[bs] = bi;
    }
    // Quantisation grid.
    float p[3];
    int e[3];
    for (int k = 0; k < 3; ++k) {
        p[k] = pb.lo[k];
        const double ext = (double)pb.hi[k] - (double)pb.lo[k];
        int ex = -126;
        if (ext > 0.0) {
            ex = (int)ceil(log2(ext / 255.0));
            while (ldexp(255.0, ex) < ext) ++ex;
            ex = max(ex, -126);
        }
        e[k] = min(ex, 127);
    }
    // Reserve the inner children's node block and the leaf triangles' block.
    uint32_t inner = 0, ntri = 0;
    uint32_t leaf_tris[8][kMaxLeaf];
    int leaf_cnt[8];
    for (int i = 0; i < nk; ++i) {
        leaf_cnt[i] = 0;
        if (leaf[i]) { leaf_cnt[i] = gather_leaf_tris(a, kid[i], leaf_tris[i]); ntri += (uint32_t)leaf_cnt[i]; }
        else ++inner;
    }
    const uint32_t child_base = inner ? atomicAdd(a.next_node, inner) : 0u;
    const uint32_t tri_base = ntri ? atomicAdd(a.next_tri, ntri) : 0u;
    const uint32_t qbase = inner ? atomicAdd(a.q_out_n, inner) : 0u;
    uint8_t meta[8] = {0}, qlo[3][8] = {{0}}, qhi[3][8] = {{0}};
    uint32_t imask = 0, rank = 0, toff = 0;
    for (int s = 0; s < 8; ++s) {
        const int i = kid_in_slot[s];
        if (i < 0) continue;
        const Box6 cb = a.box[kid[i]];
        for (int k = 0; k < 3; ++k) {
            const double step = ldexp(1.0, e[k]);
            const double lo = floor(((double)cb.lo[k] - (double)p[k]) / step);
            const double hi = ceil(((double)cb.hi[k] - (double)p[k]) / step);
            qlo[k][s] = (uint8_t)fmin(fmax(lo, 0.0), 255.0);
            qhi[k][s] = (uint8_t)fmin(fmax(hi, 0.0), 255.0);
        }
        if (leaf[i]) {
            const uint32_t c = (uint32_t)leaf_cnt[i];
            meta[s] = (uint8_t)((((1u << c) - 1u) << 5) | toff);
            for (uint32_t k = 0; k < c; ++k) a.tri_order[tri_base + toff + k] = leaf_tris[i][k];
            toff += c;
        } else {
            imask |= 1u << s;
            meta[s] = (uint8_t)((1u << 5) | (24u + (uint32_t)s));
            a.q_out[qbase + rank] = make_int2(kid[i], (int)(child_base + rank));
            ++rank;
        }
    }
    uint32_t* w = a.nodes + 20 * (size_t)widx;
    w[0] = __float_as_uint(p[0]); w[1] = __float_as_uint(p[1]); w[2] = __float_as_uint(p[2]);
    w[3] = (uint32_t)(uint8_t)(int8_t)e[0] | ((uint32_t)(uint8_t)(int8_t)e[1] << 8) |
           ((uint32_t)(uint8_t)(int8_t)e[2] << 16) | (imask << 24);
    w[4] = inner ? child_base : 0u;
    w[5] = 4u * tri_base;
    auto pack4 = [](const uint8_t* b) {
        return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
    };
    w[6] = pack4(meta); w[7] = pack4(meta + 4);
    for (int k = 0; k < 3; ++k) {
        w[8 + 2 * k] = pack4(qlo[k]); w[9 + 2 * k] = pack4(qlo[k] + 4);
        w[14 + 2 * k] = pack4(qhi[k]); w[15 + 2 * k] = pack4(qhi[k] + 4);
    }
}

// Both triangle layouts in leaf order (the host builder's formulas).
__global__ void k_emit_tris(const float* __restrict__ verts, const uint32_t* __restrict__ order, uint32_t nt,
                            float* __restrict__ tris_ref, float* __restrict__ tris_wt) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += gridDim.x * blockDim.x) {
        const uint32_t t = order[k];
        const float* tv = &verts[9 * (size_t)t];
        float* W = &tris_wt[12 * (size_t)k];
        W[0] = tv[0]; W[1] = tv[1]; W[2] = tv[2]; W[3] = __uint_as_float(t);
        W[4] = tv[3]; W[5] = tv[4]; W[6] = tv[5]; W[7] = 0.0f;
        W[8] = tv[6]; W[9] = tv[7]; W[10] = tv[8]; W[11] = 0.0f;
        const double v0[3] = {tv[0], tv[1], tv[2]};
        const double e1[3] = {tv[3] - v0[0], tv[4] - v0[1], tv[5] - v0[2]};
        const double e2[3] = {tv[6] - v0[0], tv[7] - v0[1], tv[8] - v0[2]};
        auto cross = [](const double* x, const double* y, double* r) {
            r[0] = x[1] * y[2] - x[2] * y[1];
            r[1] = x[2] * y[0] - x[0] * y[2];
            r[2] = x[0] * y[1] - x[1] * y[0];
        };
        double nrm[3], r0[3], r1[3];
        cross(e1, e2, nrm);
        const double n2 = nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2];
        float* R = &tris_ref[16 * (size_t)k];
        if (!(n2 > 0.0) || !isfinite(n2)) {
            for (int j = 0; j < 12; ++j) R[j] = 0.0f;
            R[11] = 1.0f;
        } else {
            cross(e2, nrm, r0);
            cross(nrm, e1, r1);
            const double inv = 1.0 / n2;
            double rows[3][3];
            for (int c = 0; c < 3; ++c) { rows[0][c] = r0[c] * inv; rows[1][c] = r1[c] * inv; rows[2][c] = nrm[c] * inv; }
            for (int r = 0; r < 3; ++r) {
                const double wv = -(rows[r][0] * v0[0] + rows[r][1] * v0[1] + rows[r][2] * v0[2]);
                R[4 * r + 0] = (float)rows[r][0];
                R[4 * r + 1] = (float)rows[r][1];
                R[4 * r + 2] = (float)rows[r][2];
                R[4 * r + 3] = (float)wv;
            }
        }
        R[12] = 0.0f; R[13] = 0.0f; R[14] = 0.0f; R[15] = __uint_as_float(t);
    }
}

// Scratch of one build, freed on every exit path.
struct Scratch {
    static constexpr int kSlots = 32;
    void* p[kSlots] = {nullptr};
    int n = 0;
    cudaError_t err = cudaSuccess;
    template <typename T>
    T* get(size_t count) {
        if (err != cudaSuccess) return nullptr;
        if (n == kSlots) { err = cudaErrorMemoryAllocation; return nullptr; }
        void* q = nullptr;
        err = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (err == cudaSuccess) p[n++] = q;
        return static_cast<T*>(q);
    }
    ~Scratch() {
        for (int i = 0; i < n; ++i) cudaFree(p[i]);
    }
};

}  // namespace
}  // namespace tfg

extern "C" int tfgTinyBVHConstruirGPU(const TfgPrimitiva* d_prims, int32_t n, TfgTinyBVH* out, void* stream) {
    using namespace tfg;
    if (!out) return fail(TFG_E_INVALID, "tfgTinyBVHConstruirGPU: out is null");
    std::memset(out, 0, sizeof(*out));
    if (n < 0 || (n > 0 && !d_prims)) return fail(TFG_E_INVALID, "tfgTinyBVHConstruirGPU: bad primitive array");
    if (n == 0) return ok();
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail((int)e, cudaGetErrorString(e));
    if (int rc = require_sm100(dev)) return rc;
    const uint32_t blocks = std::min<uint32_t>(((uint32_t)n + 255) / 256, 148u * 8u);
    Scratch sc;
    uint32_t* flag = sc.get<uint32_t>(n);
    uint32_t* pos = sc.get<uint32_t>(n);
    size_t tmp_bytes = 0;
    if (sc.err == cudaSuccess) sc.err = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flag, pos, n, s);
    void* tmp = sc.get<uint8_t>(tmp_bytes);
    if (sc.err != cudaSuccess) return fail((int)sc.err, std::string("tfgTinyBVHConstruirGPU: ") + cudaGetErrorString(sc.err));
    k_flag_triangles<<<blocks, 256, 0, s>>>(d_prims, n, flag);
    if (sc.err == cudaSuccess) sc.err = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flag, pos, n, s);
    uint32_t nt = 0, last_flag = 0;
    if (sc.err == cudaSuccess) sc.err = cudaMemcpyAsync(&nt, pos + n - 1, 4, cudaMemcpyDeviceToHost, s);
    if (sc.err == cudaSuccess) sc.err = cudaMemcpyAsync(&last_flag, flag + n - 1, 4, cudaMemcpyDeviceToHost, s);
    if (sc.err == cudaSuccess) sc.err = cudaStreamSynchronize(s);
    if (sc.err != cudaSuccess) return fail((int)sc.err, std::string("tfgTinyBVHConstruirGPU: ") + cudaGetErrorString(sc.err));
    nt += last_flag;
    if (nt == 0) return ok();   // no triangles: an empty BVH, as the host path
    if (nt > (1u << 29)) return fail(TFG_E_INVALID, "tfgTinyBVHConstruirGPU: too many triangles");

    TfgPrimitiva* tris = nullptr;
    e = cudaMalloc((void**)&tris, (size_t)nt * sizeof(TfgPrimitiva));
    if (e != cudaSuccess) return fail((int)e, std::string("tfgTinyBVHConstruirGPU: ") + cudaGetErrorString(e));
    out->d_primitivas = tris;
    out->num_primitivas = nt;
    auto bail = [&](cudaError_t err) {
        tfgTinyBVHLiberar(out);
        return fail((int)err, std::string("tfgTinyBVHConstruirGPU: ") + cudaGetErrorString(err));
    };
    float* verts = sc.get<float>(9 * (size_t)nt);
    Box6* tbox = sc.get<Box6>(nt);
    uint32_t* cb = sc.get<uint32_t>(6);
    uint32_t* code = sc.get<uint32_t>(nt);
    uint32_t* code_s = sc.get<uint32_t>(nt);
    uint32_t* idx = sc.get<uint32_t>(nt);
    uint32_t* idx_s = sc.get<uint32_t>(nt);
    const uint32_t nn = 2 * nt - 1;
    int* child = sc.get<int>(2 * (size_t)nt);
    int* parent = sc.get<int>(nn);
    Box6* box = sc.get<Box6>(nn);
    int* count = sc.get<int>(nn);
    Plan2* plan = sc.get<Plan2>(nn);
    uint32_t* arrivals = sc.get<uint32_t>(nt);
    int2* q[2] = {sc.get<int2>(nt + 1), sc.get<int2>(nt + 1)};
    uint32_t* ctr = sc.get<uint32_t>(3);   // next_node, next_tri, queue length
    uint32_t* nodes = sc.get<uint32_t>(20 * ((size_t)nt + 1));
    uint32_t* tri_order = sc.get<uint32_t>(nt);
    if (sc.err != cudaSuccess) return bail(sc.err);

    const uint32_t tb = std::min<uint32_t>((nt + 255) / 256, 148u * 8u);
    k_compact<<<blocks, 256, 0, s>>>(d_prims, n, flag, pos, tris, verts, tbox);
    const uint32_t init_cb[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
    e = cudaMemcpyAsync(cb, init_cb, sizeof(init_cb), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return bail(e);
    k_centroid_bounds<<<tb, 256, 0, s>>>(tbox, nt, cb);
    k_morton<<<tb, 256, 0, s>>>(tbox, nt, cb, code, idx);
    size_t sort_bytes = 0;
    e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, code, code_s, idx, idx_s, (int)nt, 0, 30, s);
    if (e != cudaSuccess) return bail(e);
    void* sort_tmp = sc.get<uint8_t>(sort_bytes);
    if (sc.err != cudaSuccess) return bail(sc.err);
    e = cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, code, code_s, idx, idx_s, (int)nt, 0, 30, s);
    if (e != cudaSuccess) return bail(e);
    if (nt > 1) {
        k_radix_tree<<<tb, 256, 0, s>>>(code_s, (int)nt, child, parent);
        e = cudaMemsetAsync(arrivals, 0, (size_t)nt * sizeof(uint32_t), s);
        if (e != cudaSuccess) return bail(e);
    }
    k_refit<<<tb, 256, 0, s>>>(tbox, idx_s, (int)nt, child, parent, box, count, plan, arrivals);
    // Level-by-level collapse; the root is binary node 0 (or the single leaf).
    const int2 r0 = make_int2(0, 0);   // binary node 0: the root (with one triangle, its leaf)
    const uint32_t init_ctr[3] = {1u, 0u, 0u};
    e = cudaMemcpyAsync(q[0], &r0, sizeof(r0), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctr, init_ctr, sizeof(init_ctr), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return bail(e);
    uint32_t qn = 1, depth = 0;
    while (qn > 0) {
        ++depth;
        if (depth > 64) {   // a valid tree is far shallower
            tfgTinyBVHLiberar(out);
            return fail(TFG_E_BUILD, "tfgTinyBVHConstruirGPU: tree deeper than 64 levels");
        }
        WideArgs wa;
        wa.child = child; wa.box = box; wa.count = count; wa.plan = plan; wa.sorted = idx_s; wa.n = (int)nt;
        wa.q_in = q[(depth - 1) & 1]; wa.q_n = qn; wa.q_out = q[depth & 1]; wa.q_out_n = ctr + 2;
        wa.next_node = ctr; wa.next_tri = ctr + 1; wa.nodes = nodes; wa.tri_order = tri_order;
        e = cudaMemsetAsync(ctr + 2, 0, 4, s);
        if (e != cudaSuccess) return bail(e);
        k_wide_level<<<(qn + 127) / 128, 128, 0, s>>>(wa);
        e = cudaMemcpyAsync(&qn, ctr + 2, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return bail(e);
    }
    uint32_t counts[2] = {0, 0};
    e = cudaMemcpy(counts, ctr, sizeof(counts), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return bail(e);
    if (counts[1] != nt) {
        tfgTinyBVHLiberar(out);
        return fail(TFG_E_BUILD, "tfgTinyBVHConstruirGPU: leaves do not cover every triangle");
    }
    const uint32_t num_nodes = counts[0];
    e = cudaMalloc((void**)&out->ref.d_nodos, (size_t)num_nodes * 80);
    if (e == cudaSuccess) e = cudaMalloc((void**)&out->ref.d_tris, (size_t)nt * 64);
    if (e == cudaSuccess) e = cudaMalloc((void**)&out->d_tris_wt, (size_t)nt * 48);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out->ref.d_nodos, nodes, (size_t)num_nodes * 80, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return bail(e);
    k_emit_tris<<<tb, 256, 0, s>>>(verts, tri_order, nt, reinterpret_cast<float*>(out->ref.d_tris), out->d_tris_wt);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bail(e);
    out->ref.num_nodos = num_nodes;
    out->ref.num_tris = nt;
    out->max_depth = depth;
    return ok();
}
