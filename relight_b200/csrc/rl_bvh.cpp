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
// SAH cost of visiting a node, in triangle tests: a split is worth
// kTraversalCost * area(node) + area(L) * n(L) + area(R) * n(R) against
// area(node) * n for a leaf.  Without the term every pair of triangles is
// split into one-triangle leaves; with it (any value in 0.25..1 builds nearly
// the same tree) the terrain tree has 77k instead of 114k nodes and the
// final gather runs 11% faster (48.0 -> 42.8 ms).  Hits do not depend on it.
constexpr float kTraversalCost = 1.0f;
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
                float cost = kTraversalCost * bx.area() + left_area[k - 1] * lc + racc.area() * rcnt;
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

// ---------------------------------------------------- compressed 8-wide
//
// Node (20 words): p.xyz (float), exponent bytes ex | ey << 8 | ez << 16 |
// internal-child mask << 24, child base, triangle base, meta[8] (2 words),
// then the quantised child bounds qlo.x[8] qlo.y[8] qlo.z[8] qhi.x[8]
// qhi.y[8] qhi.z[8] (one byte each).  Child c's box is
// p + q * 2^(e - 127) per axis; internal children are stored contiguously
// from the child base in slot order (rank = internal slots below c); a leaf
// slot's meta is count << 5 | offset, its triangles at triangle base +
// offset (count <= 4, offset <= 28); meta 0 on a non-internal slot = empty.
// Children go to slots by octant (the child lying most towards corner s of
// the node gets slot s), so a ray that visits slots in the order slot ^
// (its direction sign bits) meets them roughly front to back.

struct Collapse8 {
    const std::vector<Node>& bn;
    const std::vector<float>& tris;   // records in leaf (prims) order
    std::vector<uint32_t>& n8;
    std::vector<float>& t8;

    struct Slot {
        int node = -1;       // binary node id (inner child), or the leaf node
        int first = 0, count = 0;  // leaf chunk in prims order
        Box box;
        bool inner = false;
    };

    // Smallest exponent e (scale 2^e) with every child's float decode
    // p + q * 2^e (one rounding) conservative for q in [0, 255].
    static void quantize(float p, const float* lo, const float* hi, int n, float ext, int& e, uint8_t* qlo,
                         uint8_t* qhi) {
        int ee = ext > 0.0f ? (int)std::ceil(std::log2((double)ext / 255.0)) : -126;
        ee = std::max(-126, std::min(127, ee));
        for (;; ee++) {
            float sc = std::ldexp(1.0f, ee);
            bool ok = true;
            for (int c = 0; c < n && ok; c++) {
                float ql = std::floor((lo[c] - p) / sc);
                ql = std::max(0.0f, std::min(255.0f, ql));
                while (ql > 0.0f && p + ql * sc > lo[c]) ql -= 1.0f;
                float qh = std::ceil((hi[c] - p) / sc);
                qh = std::max(0.0f, qh);
                while (qh <= 255.0f && p + qh * sc < hi[c]) qh += 1.0f;
                if (qh > 255.0f || p + ql * sc > lo[c]) {
                    ok = false;
                    break;
                }
                qlo[c] = (uint8_t)ql;
                qhi[c] = (uint8_t)qh;
            }
            if (ok || ee >= 127) {
                e = ee;
                return;
            }
        }
    }

    // Write binary inner node `id` as the 8-wide node at index `at`.
    void emit(int id, uint32_t at) {
        std::vector<int> items = {bn[id].child[0], bn[id].child[1]};
        auto slots_of = [&](int k) { return bn[k].count > 0 ? (bn[k].count + 3) / 4 : 1; };
        for (;;) {
            int used = 0, pick = -1;
            float best = -1.0f;
            for (int k : items) used += slots_of(k);
            for (size_t q = 0; q < items.size(); q++) {
                const Node& c = bn[items[q]];
                if (c.count == 0 && c.box.area() > best) {
                    int grow = slots_of(c.child[0]) + slots_of(c.child[1]) - 1;
                    if (used + grow <= 8) { best = c.box.area(); pick = (int)q; }
                }
            }
            if (pick < 0) break;
            int opened = items[pick];
            items[pick] = bn[opened].child[0];
            items.push_back(bn[opened].child[1]);
        }
        std::vector<Slot> sl;
        for (int k : items) {
            const Node& c = bn[k];
            if (c.count == 0) {
                Slot s;
                s.node = k; s.inner = true; s.box = c.box;
                sl.push_back(s);
            } else {
                for (int f = 0; f < c.count; f += 4) {
                    Slot s;
                    s.node = k; s.first = c.first + f; s.count = std::min(4, c.count - f); s.box = c.box;
                    sl.push_back(s);
                }
            }
        }
        // octant slot assignment, greedy on the best remaining (child, slot) score
        Box nb;
        for (const Slot& s : sl) nb.grow(s.box);
        float cen[3];
        for (int a = 0; a < 3; a++) cen[a] = 0.5f * (nb.lo[a] + nb.hi[a]);
        int slot_of[8] = {-1, -1, -1, -1, -1, -1, -1, -1};  // slot -> index in sl
        std::vector<bool> placed(sl.size(), false);
        for (size_t round = 0; round < sl.size(); round++) {
            float bs = -FLT_MAX;
            int bi = -1, bslot = -1;
            for (size_t i = 0; i < sl.size(); i++) {
                if (placed[i]) continue;
                for (int q = 0; q < 8; q++) {
                    if (slot_of[q] >= 0) continue;
                    float sc = 0.0f;
                    for (int a = 0; a < 3; a++) {
                        float d = 0.5f * (sl[i].box.lo[a] + sl[i].box.hi[a]) - cen[a];
                        sc += ((q >> a) & 1) ? d : -d;
                    }
                    if (sc > bs) { bs = sc; bi = (int)i; bslot = q; }
                }
            }
            placed[bi] = true;
            slot_of[bslot] = bi;
        }
        // children block and triangle run
        uint32_t imask = 0;
        int ninner = 0;
        for (int q = 0; q < 8; q++)
            if (slot_of[q] >= 0 && sl[slot_of[q]].inner) { imask |= 1u << q; ninner++; }
        uint32_t child_base = (uint32_t)(n8.size() / 20);
        n8.resize(n8.size() + 20 * (size_t)ninner, 0u);
        uint32_t tri_base = (uint32_t)(t8.size() / 12);
        uint8_t meta[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int off = 0;
        for (int q = 0; q < 8; q++) {
            if (slot_of[q] < 0 || sl[slot_of[q]].inner) continue;
            const Slot& s = sl[slot_of[q]];
            for (int i = 0; i < s.count; i++)
                t8.insert(t8.end(), tris.begin() + 12 * (size_t)(s.first + i), tris.begin() + 12 * (size_t)(s.first + i + 1));
            meta[q] = (uint8_t)((s.count << 5) | off);
            off += s.count;
        }
        // quantised boxes
        uint8_t qlo[3][8], qhi[3][8];
        int ex[3];
        for (int a = 0; a < 3; a++) {
            float lo[8], hi[8];
            int n = 0, map[8];
            for (int q = 0; q < 8; q++) {
                qlo[a][q] = 255;
                qhi[a][q] = 0;
                if (slot_of[q] < 0) continue;
                lo[n] = sl[slot_of[q]].box.lo[a];
                hi[n] = sl[slot_of[q]].box.hi[a];
                map[n++] = q;
            }
            uint8_t l8[8], h8[8];
            quantize(nb.lo[a], lo, hi, n, nb.hi[a] - nb.lo[a], ex[a], l8, h8);
            for (int c = 0; c < n; c++) { qlo[a][map[c]] = l8[c]; qhi[a][map[c]] = h8[c]; }
        }
        uint32_t* w = &n8[20 * (size_t)at];
        for (int a = 0; a < 3; a++) std::memcpy(&w[a], &nb.lo[a], 4);
        w[3] = (uint32_t)(ex[0] + 127) | ((uint32_t)(ex[1] + 127) << 8) | ((uint32_t)(ex[2] + 127) << 16) | (imask << 24);
        w[4] = child_base;
        w[5] = tri_base;
        std::memcpy(&w[6], meta, 8);
        uint8_t* qb = reinterpret_cast<uint8_t*>(&w[8]);
        for (int a = 0; a < 3; a++) std::memcpy(qb + 8 * a, qlo[a], 8);
        for (int a = 0; a < 3; a++) std::memcpy(qb + 24 + 8 * a, qhi[a], 8);
        int r = 0;
        for (int q = 0; q < 8; q++)
            if (imask >> q & 1u) emit(sl[slot_of[q]].node, child_base + r++);
    }
};

}  // namespace

bool build_bvh_sah(const float* pos, int nverts, const int32_t* tris, int ntris, BvhBuild& out, const char** err,
                   bool wide8) {
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

    // Compressed 8-wide tree (a single-leaf tree gets none: the binary walk serves it).
    if (wide8 && B.nodes[0].count == 0) {
        Collapse8 c8{B.nodes, out.tris, out.nodes8, out.tris8};
        out.nodes8.assign(20, 0u);
        c8.emit(0, 0);
        out.nodes8_count = (int64_t)(out.nodes8.size() / 20);
    }
    return true;
}

}  // namespace rl
