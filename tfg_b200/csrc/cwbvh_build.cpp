// CWBVH builder: binned-SAH binary BVH -> cost-optimal 8-wide collapse -> 8-bit
// quantisation, emitted in the compressed-wide-BVH node layout that the
// reference traversal decodes (traverse_cwbvh.cuh:77-181; Ylitie, Karras,
// Laine 2017, "Efficient Incoherent Ray Traversal on GPUs Through Compressed
// Wide BVHs").  It replaces the tinybvh BVH8_CWBVH::Build call in
// tinybvh_wrapper.cpp:53, whose source is not part of the reference.
//
// Node (20 x 32-bit words, 80 B):
//   w0..2  p.xyz (float)          origin of the quantisation grid
//   w3     bytes e.x, e.y, e.z (int8 exponents), imask (inner-child slots)
//   w4     child node base (node units); inner children are stored
//          contiguously in slot order
//   w5     triangle base in float4 units (4 * BVH-order triangle index)
//   w6,w7  meta byte per slot: 0 = empty; inner = 0b001_11sss (24 + slot);
//          leaf = unary triangle count in bits 5..7, triangle offset in 0..4
//   w8..19 q_lo_x[8] q_lo_y[8] q_lo_z[8] q_hi_x[8] q_hi_y[8] q_hi_z[8]
//          (the reference reads q_lo_x from n2.x/n2.y, q_lo_y n2.z/n2.w,
//           q_lo_z n3.x/n3.y, q_hi_x n3.z/n3.w, q_hi_y n4.x/n4.y,
//           q_hi_z n4.z/n4.w, traverse_cwbvh.cuh:102-107,145-150)
// Slot s holds the child that rays of octant s (x<0 -> 4, y<0 -> 2,
// z<0 -> 1) should visit first, so the traversal's octant-xor ordering
// (traverse_cwbvh.cuh:59,73) yields near front-to-back order.

#include "../../include/tfg_pt.h"
#include "tfg_errors.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

namespace {

struct Box {
    float lo[3], hi[3];
    void reset() {
        for (int a = 0; a < 3; ++a) { lo[a] = std::numeric_limits<float>::infinity(); hi[a] = -lo[a]; }
    }
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
    }
    double area() const {
        double d[3];
        for (int a = 0; a < 3; ++a) d[a] = std::max(0.0, (double)hi[a] - (double)lo[a]);
        return 2.0 * (d[0] * d[1] + d[0] * d[2] + d[1] * d[2]);
    }
    bool valid() const { return lo[0] <= hi[0]; }
};

// Binary node of the intermediate BVH.
struct Node2 {
    Box box;
    int left = -1, right = -1;   // children (interior)
    int first = 0, count = 0;    // triangle range in `order` (leaf when count > 0)
    int tris_below = 0;
};

constexpr int kBins = 32;
constexpr int kMaxLeaf = 3;   // the 3-bit unary meta count limits a leaf to 3 triangles
constexpr double kCostTrav = 1.0, kCostTri = 1.0;
// Wide-node collapse costs: one 8-wide node decode against one triangle test
// (about 200 against 60 instructions in the traversal kernels).
constexpr double kCostWideNode = 1.0, kCostWideTri = 0.3;

// Collapse plan of one binary node: for a budget of i = 1..8 slots of the
// wide parent, the least cost of its subtree and how it is reached.
struct Plan {
    double cost[8];
    uint8_t how[8];     // kLeaf / kInternal (i = 1), kSame (as with i - 1 slots), or kSplit + k
    uint8_t split8;     // as a wide node of its own: slots given to the left child
};
constexpr uint8_t kLeaf = 0, kInternal = 1, kSame = 2, kSplit = 16;

class Builder {
public:
    Builder(const float* verts, uint32_t n) : v_(verts), n_(n) {}

    bool build(TfgCWBVHHost* out);

private:
    const float* v_;
    uint32_t n_;
    std::vector<Box> tbox_;
    std::vector<float> cen_;   // 3 per triangle
    std::vector<uint32_t> order_;
    std::vector<Node2> nodes2_;

    int build2(int first, int count, int depth);

    // Wide-node emission.
    struct Child { int node2; bool leaf; };
    std::vector<float> out_nodes_;
    std::vector<uint32_t> out_tri_order_;
    uint32_t max_depth_ = 0;
    std::vector<Plan> plan_;
    void plan_collapse();
    void gather_slots(int node2, int budget, std::vector<Child>& kids) const;
    void collapse(int node2, std::vector<Child>& kids);
    void gather_tris(int node2, std::vector<uint32_t>& dst);
};

int Builder::build2(int first, int count, int depth) {
    int idx = (int)nodes2_.size();
    nodes2_.emplace_back();
    Box box; box.reset();
    Box cbox; cbox.reset();
    for (int i = first; i < first + count; ++i) {
        uint32_t t = order_[i];
        box.grow(tbox_[t]);
        cbox.grow(&cen_[3 * t]);
    }
    nodes2_[idx].box = box;
    nodes2_[idx].tris_below = count;

    auto make_leaf = [&]() {
        nodes2_[idx].first = first;
        nodes2_[idx].count = count;
        return idx;
    };
    if (count == 1) return make_leaf();

    // Binned SAH over the centroid bounds.
    double best_cost = std::numeric_limits<double>::infinity();
    int best_axis = -1, best_split = -1;
    for (int a = 0; a < 3; ++a) {
        double ext = (double)cbox.hi[a] - (double)cbox.lo[a];
        if (!(ext > 0.0)) continue;
        Box bb[kBins]; int bc[kBins];
        for (int b = 0; b < kBins; ++b) { bb[b].reset(); bc[b] = 0; }
        double scale = kBins / ext;
        for (int i = first; i < first + count; ++i) {
            uint32_t t = order_[i];
            int b = (int)(((double)cen_[3 * t + a] - cbox.lo[a]) * scale);
            b = std::min(std::max(b, 0), kBins - 1);
            bb[b].grow(tbox_[t]); bc[b]++;
        }
        double rarea[kBins]; int rcount[kBins];
        Box acc; acc.reset(); int c = 0;
        for (int b = kBins - 1; b > 0; --b) {
            if (bc[b]) acc.grow(bb[b]);
            c += bc[b];
            rarea[b] = acc.valid() ? acc.area() : 0.0; rcount[b] = c;
        }
        acc.reset(); c = 0;
        for (int b = 0; b < kBins - 1; ++b) {
            if (bc[b]) acc.grow(bb[b]);
            c += bc[b];
            if (c == 0 || rcount[b + 1] == 0) continue;
            double cost = (acc.area() * c + rarea[b + 1] * rcount[b + 1]);
            if (cost < best_cost) { best_cost = cost; best_axis = a; best_split = b; }
        }
    }
    double parea = box.area();
    double split_cost = kCostTrav + (parea > 0.0 ? best_cost / parea : 0.0) * kCostTri;
    double leaf_cost = count * kCostTri;

    int mid;
    if (best_axis < 0) {
        // All centroids coincide: split by index so the tree still terminates.
        if (count <= kMaxLeaf) return make_leaf();
        mid = first + count / 2;
    } else {
        if (count <= kMaxLeaf && leaf_cost <= split_cost) return make_leaf();
        double ext = (double)cbox.hi[best_axis] - (double)cbox.lo[best_axis];
        double scale = kBins / ext;
        auto it = std::partition(order_.begin() + first, order_.begin() + first + count, [&](uint32_t t) {
            int b = (int)(((double)cen_[3 * t + best_axis] - cbox.lo[best_axis]) * scale);
            b = std::min(std::max(b, 0), kBins - 1);
            return b <= best_split;
        });
        mid = (int)(it - order_.begin());
        if (mid == first || mid == first + count) mid = first + count / 2;
    }
    int l = build2(first, mid - first, depth + 1);
    int r = build2(mid, first + count - mid, depth + 1);
    nodes2_[idx].left = l;
    nodes2_[idx].right = r;
    return idx;
}

// Cost-optimal collapse of the binary tree into 8-wide nodes (Ylitie,
// Karras, Laine 2017, section 3.1).  With A(n) the surface area of binary node
// n and p(n) its triangle count, the cost of n's subtree given at most i
// slots of the wide parent is
//   C(n, 1) = min(leaf: A(n) p(n) c_tri if p(n) <= 3, wide node: A(n) c_node + D(n, 8))
//   C(n, i) = min(C(n, i - 1), D(n, i))                        for i = 2..8
//   D(n, j) = min over k = 1..j-1 of C(left, k) + C(right, j - k)
// computed children first (a child's index is always above its parent's).
void Builder::plan_collapse() {
    const double inf = std::numeric_limits<double>::infinity();
    plan_.assign(nodes2_.size(), Plan{});
    for (int n = (int)nodes2_.size() - 1; n >= 0; --n) {
        const Node2& m = nodes2_[n];
        Plan& P = plan_[n];
        const double area = m.box.area();
        const double leaf = m.tris_below <= kMaxLeaf ? area * (double)m.tris_below * kCostWideTri : inf;
        double dist[9];
        uint8_t split[9] = {0};
        for (int j = 0; j <= 8; ++j) dist[j] = inf;
        if (m.count == 0) {
            const Plan& L = plan_[m.left];
            const Plan& R = plan_[m.right];
            for (int j = 2; j <= 8; ++j)
                for (int k = 1; k < j; ++k) {
                    const double c = L.cost[k - 1] + R.cost[j - k - 1];
                    if (c < dist[j]) { dist[j] = c; split[j] = (uint8_t)k; }
                }
        }
        const double internal = dist[8] + area * kCostWideNode;
        P.split8 = split[8];
        if (leaf <= internal) { P.cost[0] = leaf; P.how[0] = kLeaf; }
        else { P.cost[0] = internal; P.how[0] = kInternal; }
        for (int i = 2; i <= 8; ++i) {
            if (dist[i] < P.cost[i - 2]) { P.cost[i - 1] = dist[i]; P.how[i - 1] = (uint8_t)(kSplit + split[i]); }
            else { P.cost[i - 1] = P.cost[i - 2]; P.how[i - 1] = kSame; }
        }
    }
}

// The slots that binary node `node2` fills with a budget of `budget` slots.
void Builder::gather_slots(int node2, int budget, std::vector<Child>& kids) const {
    const Plan& P = plan_[node2];
    while (budget > 1 && P.how[budget - 1] == kSame) --budget;
    const uint8_t h = P.how[budget - 1];
    if (h == kLeaf) { kids.push_back({node2, true}); return; }
    if (h == kInternal) { kids.push_back({node2, false}); return; }
    const int k = h - kSplit;
    gather_slots(nodes2_[node2].left, k, kids);
    gather_slots(nodes2_[node2].right, budget - k, kids);
}

// The children (2..8) of the wide node that replaces binary node `node2`.
void Builder::collapse(int node2, std::vector<Child>& kids) {
    kids.clear();
    const Node2& n = nodes2_[node2];
    if (n.count > 0) { kids.push_back({node2, true}); return; }
    const int k = plan_[node2].split8;
    gather_slots(n.left, k, kids);
    gather_slots(n.right, 8 - k, kids);
}

void Builder::gather_tris(int node2, std::vector<uint32_t>& dst) {
    const Node2& n = nodes2_[node2];
    if (n.count > 0) {
        for (int i = n.first; i < n.first + n.count; ++i) dst.push_back(order_[i]);
        return;
    }
    gather_tris(n.left, dst);
    gather_tris(n.right, dst);
}

static inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

bool Builder::build(TfgCWBVHHost* out) {
    tbox_.resize(n_);
    cen_.resize(3 * (size_t)n_);
    order_.resize(n_);
    for (uint32_t t = 0; t < n_; ++t) {
        Box b; b.reset();
        for (int k = 0; k < 3; ++k) b.grow(&v_[9 * (size_t)t + 3 * k]);
        tbox_[t] = b;
        for (int a = 0; a < 3; ++a) cen_[3 * (size_t)t + a] = 0.5f * (b.lo[a] + b.hi[a]);
        order_[t] = t;
    }
    nodes2_.reserve(2 * (size_t)n_);
    int root2 = build2(0, (int)n_, 0);
    plan_collapse();

    // Breadth-first emission: node i's inner children get consecutive indices.
    struct Pending { int node2; uint32_t index; uint32_t depth; };
    std::vector<Pending> queue;
    queue.push_back({root2, 0u, 1u});
    uint32_t next_node = 1;
    out_nodes_.assign(20, 0.0f);
    std::vector<Child> kids;
    std::vector<uint32_t> leaf_tris;
    for (size_t qi = 0; qi < queue.size(); ++qi) {
        Pending pd = queue[qi];
        max_depth_ = std::max(max_depth_, pd.depth);
        collapse(pd.node2, kids);
        const Box& pb = nodes2_[pd.node2].box;

        // Octant slot assignment, greedy on the cost dot(c_child - c_parent, dir_s).
        double pc[3];
        for (int a = 0; a < 3; ++a) pc[a] = 0.5 * ((double)pb.lo[a] + (double)pb.hi[a]);
        int nk = (int)kids.size();
        double cost[8][8];
        for (int i = 0; i < nk; ++i) {
            const Box& cb = nodes2_[kids[i].node2].box;
            double d[3];
            for (int a = 0; a < 3; ++a) d[a] = 0.5 * ((double)cb.lo[a] + (double)cb.hi[a]) - pc[a];
            for (int s = 0; s < 8; ++s) {
                double dx = (s & 4) ? -1.0 : 1.0, dy = (s & 2) ? -1.0 : 1.0, dz = (s & 1) ? -1.0 : 1.0;
                cost[i][s] = d[0] * dx + d[1] * dy + d[2] * dz;
            }
        }
        int slot_of[8]; int kid_in_slot[8];
        for (int s = 0; s < 8; ++s) kid_in_slot[s] = -1;
        for (int i = 0; i < nk; ++i) slot_of[i] = -1;
        for (int round = 0; round < nk; ++round) {
            double best = std::numeric_limits<double>::infinity(); int bi = -1, bs = -1;
            for (int i = 0; i < nk; ++i) {
                if (slot_of[i] >= 0) continue;
                for (int s = 0; s < 8; ++s) {
                    if (kid_in_slot[s] >= 0) continue;
                    if (cost[i][s] < best || bi < 0) { best = cost[i][s]; bi = i; bs = s; }
                }
            }
            slot_of[bi] = bs; kid_in_slot[bs] = bi;
        }

        // Quantisation grid.
        float p[3]; int8_t e[3];
        for (int a = 0; a < 3; ++a) {
            p[a] = pb.lo[a];
            double ext = (double)pb.hi[a] - (double)pb.lo[a];
            int ex = -126;
            if (ext > 0.0) {
                ex = (int)std::ceil(std::log2(ext / 255.0));
                while (std::ldexp(255.0, ex) < ext) ++ex;
                ex = std::max(ex, -126);
            }
            e[a] = (int8_t)std::min(ex, 127);
        }

        uint32_t node_words[20];
        std::memset(node_words, 0, sizeof(node_words));
        node_words[0] = f2u(p[0]); node_words[1] = f2u(p[1]); node_words[2] = f2u(p[2]);
        uint8_t imask = 0;
        uint8_t meta[8] = {0};
        uint8_t qlo[3][8] = {{0}}, qhi[3][8] = {{0}};
        uint32_t child_base = next_node;
        uint32_t tri_base = (uint32_t)out_tri_order_.size();
        uint32_t inner_count = 0, tri_off = 0;
        for (int s = 0; s < 8; ++s) {
            int i = kid_in_slot[s];
            if (i < 0) continue;
            const Box& cb = nodes2_[kids[i].node2].box;
            for (int a = 0; a < 3; ++a) {
                double step = std::ldexp(1.0, e[a]);
                double lo = std::floor(((double)cb.lo[a] - (double)p[a]) / step);
                double hi = std::ceil(((double)cb.hi[a] - (double)p[a]) / step);
                qlo[a][s] = (uint8_t)std::min(std::max(lo, 0.0), 255.0);
                qhi[a][s] = (uint8_t)std::min(std::max(hi, 0.0), 255.0);
            }
            if (kids[i].leaf) {
                leaf_tris.clear();
                gather_tris(kids[i].node2, leaf_tris);
                uint32_t cnt = (uint32_t)leaf_tris.size();   // 1..3
                meta[s] = (uint8_t)((((1u << cnt) - 1u) << 5) | tri_off);
                for (uint32_t t : leaf_tris) out_tri_order_.push_back(t);
                tri_off += cnt;
            } else {
                imask |= (uint8_t)(1u << s);
                meta[s] = (uint8_t)((1u << 5) | (24u + (uint32_t)s));
                queue.push_back({kids[i].node2, child_base + inner_count, pd.depth + 1});
                ++inner_count;
            }
        }
        next_node += inner_count;
        node_words[3] = (uint32_t)(uint8_t)e[0] | ((uint32_t)(uint8_t)e[1] << 8) |
                        ((uint32_t)(uint8_t)e[2] << 16) | ((uint32_t)imask << 24);
        node_words[4] = inner_count ? child_base : 0u;
        node_words[5] = 4u * tri_base;
        std::memcpy(&node_words[6], meta, 8);
        // q arrays in order lo_x, lo_y, lo_z, hi_x, hi_y, hi_z, 8 bytes each.
        std::memcpy(&node_words[8], qlo[0], 8);
        std::memcpy(&node_words[10], qlo[1], 8);
        std::memcpy(&node_words[12], qlo[2], 8);
        std::memcpy(&node_words[14], qhi[0], 8);
        std::memcpy(&node_words[16], qhi[1], 8);
        std::memcpy(&node_words[18], qhi[2], 8);
        if (out_nodes_.size() < 20 * (size_t)(pd.index + 1)) out_nodes_.resize(20 * (size_t)(pd.index + 1), 0.0f);
        for (int w = 0; w < 20; ++w) out_nodes_[20 * (size_t)pd.index + w] = u2f(node_words[w]);
    }
    if (out_nodes_.size() < 20 * (size_t)next_node) out_nodes_.resize(20 * (size_t)next_node, 0.0f);

    const uint32_t nt = (uint32_t)out_tri_order_.size();
    out->num_nodes = next_node;
    out->num_tris = nt;
    out->max_depth = max_depth_;
    out->nodes = (float*)std::malloc(out_nodes_.size() * sizeof(float));
    out->tris_ref = (float*)std::malloc((size_t)nt * 16 * sizeof(float) + 16);
    out->tris_wt = (float*)std::malloc((size_t)nt * 12 * sizeof(float) + 16);
    if (!out->nodes || !out->tris_ref || !out->tris_wt) return false;
    std::memcpy(out->nodes, out_nodes_.data(), out_nodes_.size() * sizeof(float));

    for (uint32_t k = 0; k < nt; ++k) {
        uint32_t t = out_tri_order_[k];
        const float* tv = &v_[9 * (size_t)t];
        float* W = &out->tris_wt[12 * (size_t)k];
        W[0] = tv[0]; W[1] = tv[1]; W[2] = tv[2]; W[3] = u2f(t);
        W[4] = tv[3]; W[5] = tv[4]; W[6] = tv[5]; W[7] = 0.0f;
        W[8] = tv[6]; W[9] = tv[7]; W[10] = tv[8]; W[11] = 0.0f;

        // World -> triangle transform (u along v1-v0, v along v2-v0, w along
        // the normal): rows (e2 x n), (n x e1), n, each divided by |n|^2.
        double v0[3] = {tv[0], tv[1], tv[2]};
        double e1[3] = {tv[3] - v0[0], tv[4] - v0[1], tv[5] - v0[2]};
        double e2[3] = {tv[6] - v0[0], tv[7] - v0[1], tv[8] - v0[2]};
        auto cross = [](const double* a, const double* b, double* r) {
            r[0] = a[1] * b[2] - a[2] * b[1];
            r[1] = a[2] * b[0] - a[0] * b[2];
            r[2] = a[0] * b[1] - a[1] * b[0];
        };
        double nrm[3], r0[3], r1[3];
        cross(e1, e2, nrm);
        double n2 = nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2];
        float* R = &out->tris_ref[16 * (size_t)k];
        if (!(n2 > 0.0) || !std::isfinite(n2)) {
            // Degenerate triangle: a plane row that always yields d = -inf (rejected).
            for (int j = 0; j < 12; ++j) R[j] = 0.0f;
            R[11] = 1.0f;
        } else {
            cross(e2, nrm, r0);
            cross(nrm, e1, r1);
            double inv = 1.0 / n2;
            double rows[3][3];
            for (int a = 0; a < 3; ++a) { rows[0][a] = r0[a] * inv; rows[1][a] = r1[a] * inv; rows[2][a] = nrm[a] * inv; }
            for (int r = 0; r < 3; ++r) {
                double w = -(rows[r][0] * v0[0] + rows[r][1] * v0[1] + rows[r][2] * v0[2]);
                R[4 * r + 0] = (float)rows[r][0];
                R[4 * r + 1] = (float)rows[r][1];
                R[4 * r + 2] = (float)rows[r][2];
                R[4 * r + 3] = (float)w;
            }
        }
        R[12] = 0.0f; R[13] = 0.0f; R[14] = 0.0f; R[15] = u2f(t);
    }
    return true;
}

}  // namespace

extern "C" int tfgCWBVHBuild(const float* verts, uint32_t num_tris, TfgCWBVHHost* out) {
    if (!out) return tfg::fail(TFG_E_INVALID, "tfgCWBVHBuild: out is null");
    std::memset(out, 0, sizeof(*out));
    if (num_tris == 0) return tfg::fail(TFG_E_INVALID, "tfgCWBVHBuild: no triangles");
    if (!verts) return tfg::fail(TFG_E_INVALID, "tfgCWBVHBuild: verts is null");
    if (num_tris > (1u << 29)) return tfg::fail(TFG_E_INVALID, "tfgCWBVHBuild: too many triangles");
    try {
        Builder b(verts, num_tris);
        if (!b.build(out)) {
            tfgCWBVHFree(out);
            return tfg::fail(TFG_E_BUILD, "tfgCWBVHBuild: out of host memory");
        }
    } catch (const std::bad_alloc&) {
        tfgCWBVHFree(out);
        return tfg::fail(TFG_E_BUILD, "tfgCWBVHBuild: out of host memory");
    }
    return tfg::ok();
}

extern "C" void tfgCWBVHFree(TfgCWBVHHost* bvh) {
    if (!bvh) return;
    std::free(bvh->nodes);
    std::free(bvh->tris_ref);
    std::free(bvh->tris_wt);
    std::memset(bvh, 0, sizeof(*bvh));
}
