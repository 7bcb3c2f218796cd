// Binned-SAH BVH builder emitting the traversal layout of rl_device.cuh:
// 64-byte nodes holding both children's boxes, 48-byte triangle records
// (v0, e1, e2) in leaf order.  Surface-area heuristic with 32 bins per axis
// on triangle centroids (Wald, "On fast construction of SAH-based bounding
// volume hierarchies", 2007); leaves hold at most 4 triangles unless the
// centroids cannot be separated (at most 8, the leaf encoding's limit).
#include "rl_bvh.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

namespace rl {
namespace {

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const Box& b) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], b.lo[k]);
            hi[k] = std::max(hi[k], b.hi[k]);
        }
    }
    void grow(const float* p) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], p[k]);
            hi[k] = std::max(hi[k], p[k]);
        }
    }
    float area() const {
        float d[3];
        for (int k = 0; k < 3; k++) d[k] = std::max(0.0f, hi[k] - lo[k]);
        return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
    bool empty() const { return lo[0] > hi[0]; }
};

struct Node {
    Box box;
    int child[2] = {-1, -1};  // inner: build-node ids
    int first = 0, count = 0; // leaf: range in prims
};

constexpr int kBins = 32;
constexpr int kMaxLeaf = 4;
constexpr int kHardLeaf = 8;
constexpr int kDepthLimit = 40;

struct Builder {
    std::vector<Box> tbox;
    std::vector<float> cent;  // 3 per triangle
    std::vector<int> prims;
    std::vector<Node> nodes;
    int max_depth = 0;

    Box range_box(int b, int e, Box* cbox) const {
        Box bx, cb;
        for (int i = b; i < e; i++) {
            int t = prims[i];
            bx.grow(tbox[t]);
            cb.grow(&cent[3 * t]);
        }
        *cbox = cb;
        return bx;
    }

    // Split prims[b, e) and return the split index (b < m < e), or -1 for a leaf.
    int split(int b, int e, const Box& bx, const Box& cb, int depth) {
        int n = e - b;
        if (n <= 1) return -1;
        int axis = 0;
        float ext[3];
        for (int k = 0; k < 3; k++) ext[k] = cb.hi[k] - cb.lo[k];
        if (ext[1] > ext[axis]) axis = 1;
        if (ext[2] > ext[axis]) axis = 2;
        auto median_split = [&](int ax) {
            int m = b + n / 2;
            std::nth_element(prims.begin() + b, prims.begin() + m, prims.begin() + e,
                             [&](int x, int y) { return cent[3 * x + ax] < cent[3 * y + ax]; });
            return m;
        };
        if (depth >= kDepthLimit) return median_split(axis);
        float best_cost = FLT_MAX;
        int best_axis = -1, best_bin = -1;
        for (int ax = 0; ax < 3; ax++) {
            if (!(ext[ax] > 0.0f)) continue;
            Box bb[kBins];
            int bc[kBins] = {0};
            float scale = kBins / ext[ax];
            for (int i = b; i < e; i++) {
                int t = prims[i];
                int k = std::min(kBins - 1, std::max(0, (int)((cent[3 * t + ax] - cb.lo[ax]) * scale)));
                bc[k]++;
                bb[k].grow(tbox[t]);
            }
            float left_area[kBins];
            int left_count[kBins];
            Box acc;
            int cnt = 0;
            for (int k = 0; k < kBins - 1; k++) {
                acc.grow(bb[k]);
                cnt += bc[k];
                left_area[k] = acc.area();
                left_count[k] = cnt;
            }
            Box racc;
            int rcnt = 0;
            for (int k = kBins - 1; k > 0; k--) {
                racc.grow(bb[k]);
                rcnt += bc[k];
                int lc = left_count[k - 1];
                if (lc == 0 || rcnt == 0) continue;
                float cost = left_area[k - 1] * lc + racc.area() * rcnt;
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = ax;
                    best_bin = k;
                }
            }
        }
        float leaf_cost = bx.area() * n;
        if (best_axis < 0) {
            if (n <= kHardLeaf) return -1;
            return median_split(axis);
        }
        if (n <= kMaxLeaf && best_cost >= leaf_cost) return -1;
        float scale = kBins / ext[best_axis];
        auto mid = std::partition(prims.begin() + b, prims.begin() + e, [&](int t) {
            int k = std::min(kBins - 1, std::max(0, (int)((cent[3 * t + best_axis] - cb.lo[best_axis]) * scale)));
            return k < best_bin;
        });
        int m = (int)(mid - prims.begin());
        if (m == b || m == e) return median_split(best_axis);
        return m;
    }

    int build(int b, int e, int depth) {
        int id = (int)nodes.size();
        nodes.emplace_back();
        Box cb;
        Box bx = range_box(b, e, &cb);
        nodes[id].box = bx;
        max_depth = std::max(max_depth, depth);
        int m = split(b, e, bx, cb, depth);
        if (m < 0) {
            nodes[id].first = b;
            nodes[id].count = e - b;
            return id;
        }
        int l = build(b, m, depth + 1);
        int r = build(m, e, depth + 1);
        nodes[id].child[0] = l;
        nodes[id].child[1] = r;
        return id;
    }
};

// 4-wide node: f4[0..5] = lo.x, hi.x, lo.y, hi.y, lo.z, hi.z of the four
// children; f4[6] = child codes; f4[7] unused.  Empty slots get a far point
// box and the code kEmpty4.
constexpr int kEmpty4 = (int)0x80000000;

void put_child_box4(float* dst, int slot, const Box& b) {
    for (int k = 0; k < 3; k++) {
        dst[(2 * k) * 4 + slot] = b.lo[k];
        dst[(2 * k + 1) * 4 + slot] = b.hi[k];
    }
}

void put_child_box(float* dst, int slot, const Box& b) {
    // n0 / n1: lo.x hi.x lo.y hi.y for child 0 / 1; n2: c0 lo.z hi.z, c1 lo.z hi.z
    float* xy = dst + 4 * slot;
    xy[0] = b.lo[0]; xy[1] = b.hi[0]; xy[2] = b.lo[1]; xy[3] = b.hi[1];
    dst[8 + 2 * slot] = b.lo[2];
    dst[8 + 2 * slot + 1] = b.hi[2];
}

}  // namespace

bool build_bvh_sah(const float* pos, int nverts, const int32_t* tris, int ntris, BvhBuild& out, const char** err) {
    out = BvhBuild();
    if (ntris <= 0) return true;
    if ((int64_t)ntris >= (1ll << 28)) {
        *err = "too many triangles for the 28-bit leaf encoding";
        return false;
    }
    Builder B;
    B.tbox.resize(ntris);
    B.cent.resize(3 * (size_t)ntris);
    B.prims.resize(ntris);
    for (int t = 0; t < ntris; t++) {
        Box bx;
        for (int k = 0; k < 3; k++) {
            int v = tris[3 * t + k];
            if (v < 0 || v >= nverts) {
                *err = "triangle vertex index out of range";
                return false;
            }
            bx.grow(pos + 3 * (size_t)v);
        }
        // Pad outward: a Moeller-Trumbore hit whose t carries rounding error
        // must still lie inside every ancestor box.
        for (int k = 0; k < 3; k++) {
            float m = std::max(std::fabs(bx.lo[k]), std::fabs(bx.hi[k]));
            float pad = 1e-5f * std::max(1.0f, m);
            bx.lo[k] -= pad;
            bx.hi[k] += pad;
        }
        B.tbox[t] = bx;
        for (int k = 0; k < 3; k++) B.cent[3 * t + k] = 0.5f * (bx.lo[k] + bx.hi[k]);
        B.prims[t] = t;
    }
    B.nodes.reserve(2 * (size_t)ntris);
    B.build(0, ntris, 0);
    out.depth = B.max_depth;

    // Triangle records in prims order (leaves reference contiguous ranges).
    out.tris.resize(12 * (size_t)ntris);
    for (int i = 0; i < ntris; i++) {
        int t = B.prims[i];
        const float* p0 = pos + 3 * (size_t)tris[3 * t];
        const float* p1 = pos + 3 * (size_t)tris[3 * t + 1];
        const float* p2 = pos + 3 * (size_t)tris[3 * t + 2];
        float* r = &out.tris[12 * (size_t)i];
        r[0] = p0[0]; r[1] = p0[1]; r[2] = p0[2];
        std::memcpy(&r[3], &t, 4);
        for (int k = 0; k < 3; k++) {
            r[4 + k] = p1[k] - p0[k];
            r[8 + k] = p2[k] - p0[k];
        }
        r[7] = 0.0f;
        r[11] = 0.0f;
    }

    // Emit inner nodes in depth-first order; the root is always inner.
    std::vector<int> gpu_id(B.nodes.size(), -1);
    std::vector<int> order;
    std::vector<int> st = {0};
    while (!st.empty()) {
        int id = st.back();
        st.pop_back();
        if (B.nodes[id].count > 0) continue;
        gpu_id[id] = (int)order.size();
        order.push_back(id);
        st.push_back(B.nodes[id].child[1]);
        st.push_back(B.nodes[id].child[0]);
    }
    auto code_of = [&](int id) -> int {
        const Node& n = B.nodes[id];
        if (n.count > 0) return ~((n.first << 3) | (n.count - 1));
        return gpu_id[id];
    };
    float root_area = std::max(B.nodes[0].box.area(), 1e-30f);
    if (order.empty()) {
        // a single-leaf tree: an inner root whose two children are that leaf
        out.nodes.assign(16, 0.0f);
        put_child_box(out.nodes.data(), 0, B.nodes[0].box);
        put_child_box(out.nodes.data(), 1, B.nodes[0].box);
        int c = code_of(0);
        std::memcpy(&out.nodes[12], &c, 4);
        std::memcpy(&out.nodes[13], &c, 4);
        out.leaves = 1;
        out.sah = 1.0 + B.nodes[0].count;
        out.nodes4.assign(32, 0.0f);
        Box far;
        for (int a = 0; a < 3; a++) { far.lo[a] = 1e30f; far.hi[a] = 1e30f; }
        int codes4[4] = {c, kEmpty4, kEmpty4, kEmpty4};
        for (int k = 0; k < 4; k++) {
            put_child_box4(out.nodes4.data(), k, k == 0 ? B.nodes[0].box : far);
            std::memcpy(&out.nodes4[24 + k], &codes4[k], 4);
        }
        out.nodes4_count = 1;
        return true;
    }
    out.nodes.assign(16 * order.size(), 0.0f);
    double sah = 0.0;
    for (size_t g = 0; g < order.size(); g++) {
        const Node& n = B.nodes[order[g]];
        float* dst = &out.nodes[16 * g];
        sah += n.box.area() / root_area;
        for (int s = 0; s < 2; s++) {
            const Node& c = B.nodes[n.child[s]];
            put_child_box(dst, s, c.box);
            int code = code_of(n.child[s]);
            std::memcpy(&dst[12 + s], &code, 4);
            if (c.count > 0) {
                out.leaves++;
                sah += (double)c.box.area() / root_area * c.count;
            }
        }
    }
    out.sah = sah;

    // Collapse into a 4-wide tree: each 4-wide node takes a binary inner node
    // and repeatedly opens its largest-area inner child until it has four.
    struct Collapse {
        const std::vector<Node>& bn;
        std::vector<float>& n4;
        int (*leaf_code)(const Node&);
        int emit(int id) {
            int me = (int)(n4.size() / 32);
            n4.resize(n4.size() + 32, 0.0f);
            int kids[4] = {bn[id].child[0], bn[id].child[1], -1, -1};
            int nk = 2;
            while (nk < 4) {
                int pick = -1;
                float best = -1.0f;
                for (int k = 0; k < nk; k++) {
                    const Node& c = bn[kids[k]];
                    if (c.count == 0 && c.box.area() > best) { best = c.box.area(); pick = k; }
                }
                if (pick < 0) break;
                int opened = kids[pick];
                kids[pick] = bn[opened].child[0];
                kids[nk++] = bn[opened].child[1];
            }
            int codes[4];
            for (int k = 0; k < 4; k++) {
                if (k >= nk) { codes[k] = kEmpty4; continue; }
                const Node& c = bn[kids[k]];
                codes[k] = c.count > 0 ? leaf_code(c) : emit(kids[k]);
            }
            float* dst = &n4[32 * (size_t)me];
            Box far;
            for (int a = 0; a < 3; a++) { far.lo[a] = 1e30f; far.hi[a] = 1e30f; }
            for (int k = 0; k < 4; k++) {
                put_child_box4(dst, k, k < nk ? bn[kids[k]].box : far);
                std::memcpy(&dst[24 + k], &codes[k], 4);
            }
            return me;
        }
    };
    auto lc = [](const Node& n) -> int { return ~((n.first << 3) | (n.count - 1)); };
    Collapse col{B.nodes, out.nodes4, +lc};
    if (B.nodes[0].count > 0) {
        // single leaf: one 4-wide node holding it
        out.nodes4.assign(32, 0.0f);
        Box far;
        for (int a = 0; a < 3; a++) { far.lo[a] = 1e30f; far.hi[a] = 1e30f; }
        int codes[4] = {lc(B.nodes[0]), kEmpty4, kEmpty4, kEmpty4};
        for (int k = 0; k < 4; k++) {
            put_child_box4(out.nodes4.data(), k, k == 0 ? B.nodes[0].box : far);
            std::memcpy(&out.nodes4[24 + k], &codes[k], 4);
        }
    } else {
        col.emit(0);
    }
    out.nodes4_count = (int64_t)(out.nodes4.size() / 32);
    return true;
}

}  // namespace rl
