// k-nearest-neighbour photon estimate over a uniform grid.
//
// The reference estimates irradiance with a disc gather in texel space
// (Photonmap::gather, Lightmap.cpp:376-413): the mean photon colour over
// the texels within a radius.  This is the world-space counterpart with
// the same meaning: at each valid lumel of a photonmap, the mean colour of
// the k photon deposits nearest to the lumel's position (within a radius
// cap), the deposits being exactly those Photons::store adds to that
// photonmap (rl_emit_photons_records keeps each one as a record).
//
//   build:  the records of the requested slot span a box; a dense grid of
//           cells (1.25 radii wide by default, RL_TUNE_KNN_CELL) covers it;
//           cells grow when the box would need more than 2^24 of them.  One radix sort orders the
//           records by cell, x fastest, so that every row of cells along x
//           is one contiguous range; start[c] = first record of cell c.
//   query:  one warp per lumel (8x8 lumel tiles per block, a tile row per
//           warp).  The warp visits shells of cells at growing distance,
//           32 records at a time, and appends those within the radius to a
//           buffer in shared memory; when the buffer fills it is sorted and
//           cut to the k nearest, which then bound admission.  After each
//           shell every record not yet seen is provably farther than the
//           shell's half-width, so the search stops once that passes the
//           admission bound.  The k nearest by (squared distance, record
//           id) come from binary searches over the buffer's distance bits
//           (and record ids on exact ties).  Their colours are summed in
//           64-bit fixed point (2^s per unit, s set per gather from the
//           largest colour so that no sum can overflow) and the mean taken
//           in double precision, so the result depends only on which
//           records are selected: not on emission order, sort order, cell
//           width or thread timing.
// Lumels that are not valid keep the disc gather's value.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/relight_b200.h"
#include "rl_device.cuh"
#include "rl_photon_records.h"

int rl_internal_fail(int code, const char* msg);
const rl::DevMap* rl_internal_map(const rl_map* m);
int rl_internal_tune(int param);

namespace {

// Grid of one gather: origin, cell size, dimensions; n = records kept
// (min(count, capacity)), count = deposits of the emission.
struct KnnGrid {
    float ox, oy, oz, cell, inv;
    int nx, ny, nz;
    int n;
    unsigned long long count;
    float scale;     // 2^s: colour -> fixed point
    double unscale;  // 2^-s
};

// Box of one slot's records: ordered-integer images of the floats, so that
// atomicMax finds both ends (the low end through the complement).
struct KnnBounds {
    uint32_t lo[3];  // ~max(~key)
    uint32_t hi[3];
    uint32_t cmax;   // bits of the largest |colour component|
};

}  // namespace

struct rl_photons {
    PhotonRecord* rec = nullptr;     // emission order
    PhotonRecord* sorted = nullptr;  // grid order
    float4* pos = nullptr;           // grid order: x, y, z of `sorted`
    unsigned long long* d_count = nullptr;
    long long capacity = 0;
    uint32_t *keys = nullptr, *keys_out = nullptr;
    uint32_t *idx = nullptr, *idx_out = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    uint32_t* start = nullptr;  // [cells + 1]
    long long start_cap = 0;
    KnnBounds* d_bounds = nullptr;
    KnnGrid* d_grid = nullptr;
    ~rl_photons() {
        cudaFree(rec);
        cudaFree(sorted);
        cudaFree(pos);
        cudaFree(d_count);
        cudaFree(keys);
        cudaFree(keys_out);
        cudaFree(idx);
        cudaFree(idx_out);
        cudaFree(temp);
        cudaFree(start);
        cudaFree(d_bounds);
        cudaFree(d_grid);
    }
};

namespace {

int kfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return rl_internal_fail(code, buf);
}

#define KCK(call)                                                                                    \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return kfail(RL_CUDA_ERROR, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

constexpr int kMaxK = 128;
constexpr int kKnnTile = 8;  // lumels per block: kKnnTile x kKnnTile
constexpr long long kMaxCells = (1ll << 24) - 1;

__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// The records a gather of `slot` uses: that slot's, with finite position
// and colour.
__device__ __forceinline__ bool eligible(const PhotonRecord& r, int slot) {
    return r.slot == slot && isfinite(r.x) && isfinite(r.y) && isfinite(r.z) && isfinite(r.r) && isfinite(r.g) &&
           isfinite(r.b);
}

__device__ __forceinline__ long long kept(const unsigned long long* count, long long capacity) {
    const unsigned long long c = *count;
    return c < (unsigned long long)capacity ? (long long)c : capacity;
}

__global__ void k_knn_bounds(const PhotonRecord* rec, const unsigned long long* count, long long capacity, int slot,
                             KnnBounds* b) {
    const long long n = kept(count, capacity);
    uint32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, cmax = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const PhotonRecord r = rec[i];
        if (!eligible(r, slot)) continue;
        const uint32_t k[3] = {ordered(r.x), ordered(r.y), ordered(r.z)};
        for (int a = 0; a < 3; a++) {
            lo[a] = max(lo[a], ~k[a]);
            hi[a] = max(hi[a], k[a]);
        }
        // non-negative float bits order like the floats
        cmax = max(cmax, max(__float_as_uint(fabsf(r.r)), max(__float_as_uint(fabsf(r.g)), __float_as_uint(fabsf(r.b)))));
    }
    for (int a = 0; a < 3; a++)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = max(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    for (int o = 16; o > 0; o >>= 1) cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; a++) {
            if (lo[a]) atomicMax(&b->lo[a], lo[a]);
            if (hi[a]) atomicMax(&b->hi[a], hi[a]);
        }
        if (cmax) atomicMax(&b->cmax, cmax);
    }
}

// One thread: the grid of the box.  No records -> zero cells.
__global__ void k_knn_grid(const KnnBounds* b, const unsigned long long* count, long long capacity, float radius,
                           float cell_frac, KnnGrid* g) {
    KnnGrid o{};
    o.count = *count;
    o.n = (int)kept(count, capacity);
    o.nx = o.ny = o.nz = 0;
    // Fixed point for the colour sums: 2^s with |colour| * 2^s < 2^54, so
    // that kMaxK terms stay below 2^61.  s in [-100, 100] (2^s a normal float).
    int s = 0;
    if (b->cmax) {
        int e;
        frexp((double)__uint_as_float(b->cmax), &e);  // cmax < 2^e
        s = min(100, max(-100, 54 - e));
    }
    o.scale = ldexpf(1.0f, s);
    o.unscale = ldexp(1.0, -s);
    if (b->hi[0] != 0) {
        const float lo[3] = {unordered(~b->lo[0]), unordered(~b->lo[1]), unordered(~b->lo[2])};
        const float hi[3] = {unordered(b->hi[0]), unordered(b->hi[1]), unordered(b->hi[2])};
        double ext[3], cell = (double)radius * cell_frac, dims[3];
        for (int a = 0; a < 3; a++) ext[a] = (double)hi[a] - (double)lo[a];
        for (int it = 0; it < 64; it++) {
            double cells = 1.0;
            for (int a = 0; a < 3; a++) {
                dims[a] = floor(ext[a] / cell) + 1.0;
                cells *= dims[a];
            }
            if (cells <= (double)kMaxCells) break;
            cell *= cbrt(cells / (double)kMaxCells) * 1.01;
        }
        o.ox = lo[0];
        o.oy = lo[1];
        o.oz = lo[2];
        o.cell = (float)cell;
        o.inv = 1.0f / o.cell;
        o.nx = (int)dims[0];
        o.ny = (int)dims[1];
        o.nz = (int)dims[2];
    }
    *g = o;
}

// Cell index along one axis; monotone non-decreasing in v, clamped to the grid.
__device__ __forceinline__ int cell_axis(float v, float o, float inv, int n) {
    float t = (v - o) * inv;
    t = fminf(fmaxf(t, -1.f), (float)n);
    return min(max((int)floorf(t), 0), n - 1);
}

__global__ void k_knn_keys(const PhotonRecord* rec, long long capacity, int slot, KnnGrid g, uint32_t* keys,
                           uint32_t* idx) {
    const uint32_t none = (uint32_t)((long long)g.nx * g.ny * g.nz);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.n; i += (long long)gridDim.x * blockDim.x) {
        const PhotonRecord r = rec[i];
        uint32_t key = none;
        if (eligible(r, slot)) {
            const int ix = cell_axis(r.x, g.ox, g.inv, g.nx), iy = cell_axis(r.y, g.oy, g.inv, g.ny),
                      iz = cell_axis(r.z, g.oz, g.inv, g.nz);
            key = (uint32_t)(((long long)iz * g.ny + iy) * g.nx + ix);
        }
        keys[i] = key;
        idx[i] = (uint32_t)i;
    }
}

__global__ void k_knn_scatter(const PhotonRecord* rec, const uint32_t* keys, const uint32_t* idx, int n,
                              uint32_t none, PhotonRecord* sorted, float4* pos) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (keys[i] == none) continue;
        const PhotonRecord r = rec[idx[i]];
        sorted[i] = r;
        pos[i] = make_float4(r.x, r.y, r.z, 0.f);
    }
}

// start[c] = first sorted position whose key is >= c, for c in [0, cells].
__global__ void k_knn_start(const uint32_t* keys, int n, uint32_t cells, uint32_t* start) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c <= cells; c += (long long)gridDim.x * blockDim.x) {
        int a = 0, b = n;
        while (a < b) {
            const int m = (a + b) >> 1;
            if (keys[m] < (uint32_t)c) a = m + 1;
            else b = m;
        }
        start[c] = (uint32_t)a;
    }
}

// A box of cells, bounds inclusive (empty when lx > hx).
struct KnnBox {
    int lx, hx, ly, hy, lz, hz;
};

// The cells holding the records within h of (px, py, pz) along every axis.
// cell_axis is monotone, so the box only grows with h, and a record outside
// it lies below px - h or above px + h as rounded (or likewise along y, z).
__device__ __forceinline__ KnnBox box_around(const KnnGrid& g, float px, float py, float pz, float h) {
    return {cell_axis(px - h, g.ox, g.inv, g.nx), cell_axis(px + h, g.ox, g.inv, g.nx),
            cell_axis(py - h, g.oy, g.inv, g.ny), cell_axis(py + h, g.oy, g.inv, g.ny),
            cell_axis(pz - h, g.oz, g.inv, g.nz), cell_axis(pz + h, g.oz, g.inv, g.nz)};
}

constexpr int kKnnWarps = 8;              // warps per block: one row of an 8x8 lumel tile each
constexpr int kKnnBuf = 256;              // candidate entries per warp
constexpr int kKnnPer = kKnnBuf / 32;     // buffer entries per lane (entry lane + 32 q)
constexpr uint32_t kNoEntry = 0xffffffffu;  // distance bits above every real squared distance

__device__ __forceinline__ uint64_t warp_max64(uint64_t v) {
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t w = __shfl_xor_sync(0xffffffffu, (unsigned long long)v, o);
        v = w > v ? w : v;
    }
    return v;
}

// The k nearest of the n > k buffer entries, by (squared distance, record
// id): each lane's entries lane + 32 q get sel[q].  Distances are
// non-negative, so their bits order like them; a binary search on the bits
// finds the k-th distance v, then one on record ids settles ties at v.
// Returns the largest selected key in (*tau_d, *tau_id).
__device__ __forceinline__ void warp_select(const uint32_t (&bits)[kKnnPer], const uint32_t (&jj)[kKnnPer], int k,
                                            const PhotonRecord* __restrict__ rec, bool (&sel)[kKnnPer],
                                            float* tau_d, uint64_t* tau_id) {
    uint32_t v = 0;
    for (int bit = 30; bit >= 0; bit--) {
        const uint32_t t = v + (1u << bit) - 1u;
        int c = 0;
#pragma unroll
        for (int q = 0; q < kKnnPer; q++) c += bits[q] <= t;
        if ((int)__reduce_add_sync(0xffffffffu, (unsigned)c) < k) v += 1u << bit;
    }
    int cl = 0, ce = 0;
#pragma unroll
    for (int q = 0; q < kKnnPer; q++) {
        cl += bits[q] < v;
        ce += bits[q] == v;
    }
    cl = (int)__reduce_add_sync(0xffffffffu, (unsigned)cl);
    ce = (int)__reduce_add_sync(0xffffffffu, (unsigned)ce);
    const int slots = k - cl;  // 1 <= slots <= ce
    uint64_t ids[kKnnPer];
#pragma unroll
    for (int q = 0; q < kKnnPer; q++) ids[q] = bits[q] == v ? record_id(rec[jj[q]]) : ~0ull;
    uint64_t idmax;
    if (slots == ce) {
        uint64_t m = 0;
#pragma unroll
        for (int q = 0; q < kKnnPer; q++)
            if (bits[q] == v && ids[q] > m) m = ids[q];
        idmax = warp_max64(m);
    } else {
        // the slots-th smallest id at distance v (ids have 36 bits)
        uint64_t u = 0;
        for (int bit = 35; bit >= 0; bit--) {
            const uint64_t t = u + (1ull << bit) - 1ull;
            int c = 0;
#pragma unroll
            for (int q = 0; q < kKnnPer; q++) c += ids[q] <= t;
            if ((int)__reduce_add_sync(0xffffffffu, (unsigned)c) < slots) u += 1ull << bit;
        }
        idmax = u;
    }
#pragma unroll
    for (int q = 0; q < kKnnPer; q++) sel[q] = bits[q] < v || (bits[q] == v && ids[q] <= idmax);
    *tau_d = __uint_as_float(v);
    *tau_id = idmax;
}

// One warp per lumel, all lanes on the same lumel.
struct KnnWarp {
    float* bd;       // [kKnnBuf] squared distances
    uint32_t* bj;    // [kKnnBuf] grid positions
    const float4* __restrict__ pos;
    const PhotonRecord* __restrict__ rec;
    int lane, k, cnt;
    float r2;
    bool limited;    // the buffer was cut to k: admit only keys below (tau_d, tau_id)
    float tau_d;
    uint64_t tau_id;

    __device__ __forceinline__ void load(uint32_t (&bits)[kKnnPer], uint32_t (&jj)[kKnnPer]) const {
#pragma unroll
        for (int q = 0; q < kKnnPer; q++) {
            const int e = lane + 32 * q;
            bits[q] = e < cnt ? __float_as_uint(bd[e]) : kNoEntry;
            jj[q] = e < cnt ? bj[e] : 0u;
        }
    }

    // Cut the buffer to its k nearest entries.
    __device__ __forceinline__ void cut() {
        uint32_t bits[kKnnPer], jj[kKnnPer];
        bool sel[kKnnPer];
        __syncwarp();
        load(bits, jj);
        warp_select(bits, jj, k, rec, sel, &tau_d, &tau_id);
        __syncwarp();
        int at = 0;
#pragma unroll
        for (int q = 0; q < kKnnPer; q++) {
            const unsigned vote = __ballot_sync(0xffffffffu, sel[q]);
            if (sel[q]) {
                const int e = at + __popc(vote & ((1u << lane) - 1u));
                bd[e] = __uint_as_float(bits[q]);
                bj[e] = jj[q];
            }
            at += __popc(vote);
        }
        cnt = k;
        limited = true;
    }

    // The records of [a, b), 32 at a time; admitted ones join the buffer.
    __device__ __forceinline__ void scan(uint32_t a, uint32_t b, float px, float py, float pz) {
        for (uint32_t base = a; base < b; base += 32) {
            if (cnt + 32 > kKnnBuf) cut();
            const uint32_t j = base + lane;
            bool take = false;
            float d2 = 0.f;
            if (j < b) {
                const float4 q = __ldg(pos + j);
                const float ex = q.x - px, ey = q.y - py, ez = q.z - pz;
                d2 = ex * ex + ey * ey + ez * ez;
                take = d2 <= r2 && (!limited || d2 < tau_d || (d2 == tau_d && record_id(rec[j]) < tau_id));
            }
            const unsigned vote = __ballot_sync(0xffffffffu, take);
            if (take) {
                const int at = cnt + __popc(vote & ((1u << lane) - 1u));
                bd[at] = d2;
                bj[at] = j;
            }
            cnt += __popc(vote);
        }
    }
};

__device__ __forceinline__ long long fixed(float c, float scale) { return __float2ll_rn(c * scale); }

__device__ __forceinline__ long long warp_sum64(long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// 80 registers: 24 resident warps, no spills (launch bounds alone spill).
__global__ void __maxnreg__(80) k_knn_query(rl::DevMap m, const float4* __restrict__ pos,
                                                              const PhotonRecord* __restrict__ rec,
                                                              const uint32_t* __restrict__ start, KnnGrid g, float r2,
                                                              float radius, int k) {
    __shared__ float s_d[kKnnWarps][kKnnBuf];
    __shared__ uint32_t s_j[kKnnWarps][kKnnBuf];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int y = blockIdx.y * kKnnTile + w;
    if (y >= m.height) return;
    KnnWarp q{s_d[w], s_j[w], pos, rec, lane, k, 0, r2, false, 0.f, 0};
    for (int tx = 0; tx < kKnnTile; tx++) {
        const int x = blockIdx.x * kKnnTile + tx;
        if (x >= m.width) break;
        const long long i = (long long)y * m.width + x;
        if (!(m.flags[i] & 1)) continue;
        const float px = m.position[3 * i], py = m.position[3 * i + 1], pz = m.position[3 * i + 2];
        q.cnt = 0;
        q.limited = false;
        if (g.nx > 0) {
            // Shells of cells at growing distance: after the box of
            // half-width hl, every record not yet seen is farther than
            // gl = hl - margin along some axis, so its squared distance,
            // rounded, is at least gl * gl (margin covers the rounding of
            // px +- hl, many times over).  Stop once that bound passes the
            // admission bound (the radius, or the k-th key once the buffer
            // has been cut).  hmax: a record with a rounded squared distance
            // <= r2 lies within radius * (1 + 2^-22) along each axis, well
            // inside it.
            const float margin =
                (fabsf(px) + fabsf(py) + fabsf(pz) + radius + g.cell) * (1.0f / (1 << 20)) + 1e-30f;
            const float hmax = radius * (1.0f + 1.0f / 65536) + 4.f * margin;
            KnnBox in{1, 0, 1, 0, 1, 0};
            for (int l = 1;; l++) {
                float hl = g.cell * (float)l;
                const bool last = !(hl < hmax) || l >= 4096;
                if (last) hl = hmax;
                const KnnBox b = box_around(g, px, py, pz, hl);
                for (int cz = b.lz; cz <= b.hz; cz++)
                    for (int cy = b.ly; cy <= b.hy; cy++) {
                        const long long row = ((long long)cz * g.ny + cy) * g.nx;
                        if (cz >= in.lz && cz <= in.hz && cy >= in.ly && cy <= in.hy) {
                            q.scan(start[row + b.lx], start[row + in.lx], px, py, pz);
                            q.scan(start[row + in.hx + 1], start[row + b.hx + 1], px, py, pz);
                        } else {
                            q.scan(start[row + b.lx], start[row + b.hx + 1], px, py, pz);
                        }
                    }
                if (last) break;
                const float gl = hl - margin;
                const float tl = gl > 0.f ? gl * gl : 0.f;
                if (tl > (q.limited ? q.tau_d : r2)) break;
                in = b;
            }
        }
        // the k nearest (all, when there are no more than k), summed in
        // fixed point: exact, so the order of the terms does not matter
        __syncwarp();
        uint32_t bits[kKnnPer], jj[kKnnPer];
        bool sel[kKnnPer];
        q.load(bits, jj);
        const int n = q.cnt;
        if (n > k) {
            float td;
            uint64_t ti;
            warp_select(bits, jj, k, rec, sel, &td, &ti);
        } else {
#pragma unroll
            for (int e = 0; e < kKnnPer; e++) sel[e] = bits[e] != kNoEntry;
        }
        long long sr = 0, sg = 0, sb = 0;
#pragma unroll
        for (int e = 0; e < kKnnPer; e++)
            if (sel[e]) {
                const PhotonRecord& r = rec[jj[e]];
                sr += fixed(r.r, g.scale);
                sg += fixed(r.g, g.scale);
                sb += fixed(r.b, g.scale);
            }
        sr = warp_sum64(sr);
        sg = warp_sum64(sg);
        sb = warp_sum64(sb);
        if (lane == 0) {
            const int c = min(n, k);
            float* out = m.gathered + 3 * i;
            if (c > 0) {
                const double dc = (double)c;
                out[0] = __double2float_rn(__ll2double_rn(sr) * g.unscale / dc);
                out[1] = __double2float_rn(__ll2double_rn(sg) * g.unscale / dc);
                out[2] = __double2float_rn(__ll2double_rn(sb) * g.unscale / dc);
            } else {
                out[0] = out[1] = out[2] = 0.f;
            }
        }
        __syncwarp();
    }
}

int grid_blocks(long long n, int block) {
    return (int)std::max<long long>(1, std::min<long long>((n + block - 1) / block, 148LL * 16));
}

}  // namespace

int rl_internal_photon_sink(rl_photons* p, PhotonSink* sink, void* stream) {
    KCK(cudaMemsetAsync(p->d_count, 0, sizeof(unsigned long long), (cudaStream_t)stream));
    sink->rec = p->rec;
    sink->count = p->d_count;
    sink->capacity = (unsigned long long)p->capacity;
    return RL_OK;
}

extern "C" int rl_photons_create(int64_t capacity, rl_photons** out) {
    if (!out || capacity <= 0 || capacity >= (1ll << 31)) return kfail(RL_INVALID_CALL, "rl_photons_create: bad capacity");
    *out = nullptr;
    rl_photons* p = new (std::nothrow) rl_photons;
    if (!p) return kfail(RL_OUT_OF_MEMORY, "host allocation failed");
    p->capacity = capacity;
    size_t n = (size_t)capacity;
    cudaError_t e = cudaMalloc(&p->rec, n * sizeof(PhotonRecord));
    if (e == cudaSuccess) e = cudaMalloc(&p->sorted, n * sizeof(PhotonRecord));
    if (e == cudaSuccess) e = cudaMalloc(&p->pos, n * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_count, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&p->keys, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->keys_out, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->idx, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->idx_out, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_bounds, sizeof(KnnBounds));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_grid, sizeof(KnnGrid));
    if (e == cudaSuccess) e = cudaMemset(p->d_count, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) {
        size_t tb = 0;
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb, p->keys, p->keys_out, p->idx, p->idx_out, (int)capacity);
        p->temp_bytes = tb;
        if (e == cudaSuccess) e = cudaMalloc(&p->temp, tb);
    }
    if (e != cudaSuccess) {
        delete p;
        return kfail(e == cudaErrorMemoryAllocation ? RL_OUT_OF_MEMORY : RL_CUDA_ERROR, "rl_photons_create: %s",
                     cudaGetErrorString(e));
    }
    *out = p;
    return RL_OK;
}

extern "C" int rl_photons_destroy(rl_photons* p) {
    if (!p) return kfail(RL_INVALID_CALL, "null photon records");
    cudaDeviceSynchronize();
    delete p;
    return RL_OK;
}

extern "C" int rl_photons_count(const rl_photons* p, int64_t* emitted) {
    if (!p || !emitted) return kfail(RL_INVALID_CALL, "null argument");
    unsigned long long h = 0;
    KCK(cudaMemcpy(&h, p->d_count, sizeof h, cudaMemcpyDeviceToHost));
    *emitted = (int64_t)h;
    return RL_OK;
}

extern "C" int rl_photons_download(const rl_photons* p, float* xyzrgb, uint32_t* photon, int32_t* depth_slot) {
    if (!p) return kfail(RL_INVALID_CALL, "null photon records");
    unsigned long long h = 0;
    KCK(cudaMemcpy(&h, p->d_count, sizeof h, cudaMemcpyDeviceToHost));
    size_t n = (size_t)std::min<unsigned long long>(h, (unsigned long long)p->capacity);
    if (!n) return RL_OK;
    PhotonRecord* host = (PhotonRecord*)malloc(n * sizeof(PhotonRecord));
    if (!host) return kfail(RL_OUT_OF_MEMORY, "host allocation failed");
    cudaError_t e = cudaMemcpy(host, p->rec, n * sizeof(PhotonRecord), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        free(host);
        return kfail(RL_CUDA_ERROR, "rl_photons_download: %s", cudaGetErrorString(e));
    }
    for (size_t i = 0; i < n; i++) {
        const PhotonRecord& r = host[i];
        if (xyzrgb) {
            float* o = xyzrgb + 6 * i;
            o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.r; o[4] = r.g; o[5] = r.b;
        }
        if (photon) photon[i] = r.photon;
        if (depth_slot) {
            depth_slot[2 * i] = r.depth;
            depth_slot[2 * i + 1] = r.slot;
        }
    }
    free(host);
    return RL_OK;
}

extern "C" int rl_photons_upload(rl_photons* p, int64_t n, const float* xyzrgb, const uint32_t* photon,
                                 const int32_t* depth_slot) {
    if (!p || n < 0 || (n > 0 && (!xyzrgb || !photon || !depth_slot)))
        return kfail(RL_INVALID_CALL, "rl_photons_upload: null argument");
    if (n > p->capacity) return kfail(RL_CAPACITY, "rl_photons_upload: %lld records exceed the capacity %lld",
                                      (long long)n, p->capacity);
    PhotonRecord* host = nullptr;
    if (n > 0) {
        host = (PhotonRecord*)malloc((size_t)n * sizeof(PhotonRecord));
        if (!host) return kfail(RL_OUT_OF_MEMORY, "host allocation failed");
    }
    for (int64_t i = 0; i < n; i++) {
        const int32_t d = depth_slot[2 * i], sl = depth_slot[2 * i + 1];
        if (d < 0 || d > 0xffff || sl < 0 || sl > 0xffff) {
            free(host);
            return kfail(RL_INVALID_CALL, "rl_photons_upload: record %lld: depth and slot must be in [0, 65535]",
                         (long long)i);
        }
        PhotonRecord& r = host[i];
        const float* v = xyzrgb + 6 * i;
        r.x = v[0]; r.y = v[1]; r.z = v[2]; r.r = v[3]; r.g = v[4]; r.b = v[5];
        r.photon = photon[i];
        r.depth = (uint16_t)d;
        r.slot = (uint16_t)sl;
    }
    const unsigned long long count = (unsigned long long)n;
    cudaError_t e = n > 0 ? cudaMemcpy(p->rec, host, (size_t)n * sizeof(PhotonRecord), cudaMemcpyHostToDevice)
                          : cudaSuccess;
    free(host);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_count, &count, sizeof count, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return kfail(RL_CUDA_ERROR, "rl_photons_upload: %s", cudaGetErrorString(e));
    return RL_OK;
}

extern "C" int rl_photonmap_gather_knn(rl_map* map, int slot, rl_photons* p, int k, float radius, void* stream) {
    const rl::DevMap* m = rl_internal_map(map);
    if (!m || !p) return kfail(RL_INVALID_CALL, "rl_photonmap_gather_knn: null argument");
    if (k < 1 || k > kMaxK) return kfail(RL_INVALID_CALL, "rl_photonmap_gather_knn: k must be in [1, %d]", kMaxK);
    if (!(radius > 0.f) || !std::isfinite(radius))
        return kfail(RL_INVALID_CALL, "rl_photonmap_gather_knn: radius must be positive and finite");
    if (slot < 0 || slot > 0xffff) return kfail(RL_INVALID_CALL, "rl_photonmap_gather_knn: bad slot");
    cudaStream_t st = (cudaStream_t)stream;
    KCK(cudaMemsetAsync(p->d_bounds, 0, sizeof(KnnBounds), st));
    k_knn_bounds<<<grid_blocks(p->capacity, 256), 256, 0, st>>>(p->rec, p->d_count, p->capacity, slot, p->d_bounds);
    k_knn_grid<<<1, 1, 0, st>>>(p->d_bounds, p->d_count, p->capacity, radius,
                                rl_internal_tune(RL_TUNE_KNN_CELL) / 64.0f, p->d_grid);
    KnnGrid g;
    KCK(cudaMemcpyAsync(&g, p->d_grid, sizeof g, cudaMemcpyDeviceToHost, st));
    KCK(cudaStreamSynchronize(st));
    if (g.count > (unsigned long long)p->capacity)
        return kfail(RL_CAPACITY, "rl_photonmap_gather_knn: %llu deposits exceed the record capacity %lld", g.count,
                     p->capacity);
    const long long cells = (long long)g.nx * g.ny * g.nz;
    if (cells > kMaxCells) return kfail(RL_CUDA_ERROR, "rl_photonmap_gather_knn: grid of %lld cells", cells);
    if (cells > 0) {
        if (cells + 1 > p->start_cap) {
            cudaFree(p->start);
            p->start = nullptr;
            p->start_cap = 0;
            KCK(cudaMalloc(&p->start, (size_t)(cells + 1) * 4));
            p->start_cap = cells + 1;
        }
        int bits = 1;
        while ((1ll << bits) <= cells) bits++;
        const int n = g.n;
        k_knn_keys<<<grid_blocks(n, 256), 256, 0, st>>>(p->rec, p->capacity, slot, g, p->keys, p->idx);
        size_t tb = p->temp_bytes;
        KCK(cub::DeviceRadixSort::SortPairs(p->temp, tb, p->keys, p->keys_out, p->idx, p->idx_out, n, 0, bits, st));
        k_knn_scatter<<<grid_blocks(n, 256), 256, 0, st>>>(p->rec, p->keys_out, p->idx_out, n, (uint32_t)cells,
                                                           p->sorted, p->pos);
        k_knn_start<<<grid_blocks(cells + 1, 256), 256, 0, st>>>(p->keys_out, n, (uint32_t)cells, p->start);
    }
    const dim3 grid((unsigned)((m->width + kKnnTile - 1) / kKnnTile), (unsigned)((m->height + kKnnTile - 1) / kKnnTile));
    k_knn_query<<<grid, kKnnWarps * 32, 0, st>>>(*m, p->pos, p->sorted, p->start, g, radius * radius, radius, k);
    KCK(cudaGetLastError());
    return RL_OK;
}
