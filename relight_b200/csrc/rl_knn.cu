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
//           cells (half the radius wide by default, RL_TUNE_KNN_CELL) covers
//           it; cells grow when the box would need more than 2^24 of them.  One radix sort orders the
//           records by cell, x fastest, so that every row of cells along x
//           is one contiguous range; start[c] = first record of cell c.
//   query:  one thread per lumel, 8x8 lumel tiles per block.  Pass 1 scans
//           the cells within one cell of the lumel and keeps the k nearest
//           records in a max-heap in shared memory ordered by (squared
//           distance, record id).  Every record it skipped is farther than
//           one cell, so when the heap is full and its largest distance is
//           below one cell the selection is final.  Otherwise pass 2 scans
//           the rest of the cells within the radius.  The k records are
//           summed in ascending (distance, id) order, so the result does
//           not depend on emission order, sort order or thread timing.
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
};

// Box of one slot's records: ordered-integer images of the floats, so that
// atomicMax finds both ends (the low end through the complement).
struct KnnBounds {
    uint32_t lo[3];  // ~max(~key)
    uint32_t hi[3];
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
constexpr int kKnnBlock = kKnnTile * kKnnTile;
constexpr long long kMaxCells = (1ll << 24) - 1;

__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ bool finite3(const PhotonRecord& r) {
    return isfinite(r.x) && isfinite(r.y) && isfinite(r.z);
}

__device__ __forceinline__ long long kept(const unsigned long long* count, long long capacity) {
    const unsigned long long c = *count;
    return c < (unsigned long long)capacity ? (long long)c : capacity;
}

__global__ void k_knn_bounds(const PhotonRecord* rec, const unsigned long long* count, long long capacity, int slot,
                             KnnBounds* b) {
    const long long n = kept(count, capacity);
    uint32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const PhotonRecord r = rec[i];
        if (r.slot != slot || !finite3(r)) continue;
        const uint32_t k[3] = {ordered(r.x), ordered(r.y), ordered(r.z)};
        for (int a = 0; a < 3; a++) {
            lo[a] = max(lo[a], ~k[a]);
            hi[a] = max(hi[a], k[a]);
        }
    }
    for (int a = 0; a < 3; a++)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = max(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; a++) {
            if (lo[a]) atomicMax(&b->lo[a], lo[a]);
            if (hi[a]) atomicMax(&b->hi[a], hi[a]);
        }
}

// One thread: the grid of the box.  No records -> zero cells.
__global__ void k_knn_grid(const KnnBounds* b, const unsigned long long* count, long long capacity, float radius,
                           float cell_frac, KnnGrid* g) {
    KnnGrid o{};
    o.count = *count;
    o.n = (int)kept(count, capacity);
    o.nx = o.ny = o.nz = 0;
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
        if (r.slot == slot && finite3(r)) {
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

// Per-thread max-heap of (squared distance, sorted position) in shared
// memory, entry e of thread t at [e * kKnnBlock + t], ordered by
// (distance, record id); ids are read only on distance ties.
struct KnnHeap {
    float* d;
    uint32_t* j;
    const PhotonRecord* rec;
    int t, size, k;
    float top_d;  // largest entry, valid when size == k
    uint32_t top_j;

    __device__ __forceinline__ bool less(float da, uint32_t ja, float db, uint32_t jb) const {
        if (da != db) return da < db;
        return record_id(rec[ja]) < record_id(rec[jb]);
    }
    __device__ __forceinline__ float& D(int e) { return d[e * kKnnBlock + t]; }
    __device__ __forceinline__ uint32_t& J(int e) { return j[e * kKnnBlock + t]; }

    __device__ __forceinline__ void push(float dd, uint32_t jj) {
        int c = size++;
        while (c > 0) {
            const int p = (c - 1) >> 1;
            const float pd = D(p);
            const uint32_t pj = J(p);
            if (!less(pd, pj, dd, jj)) break;
            D(c) = pd;
            J(c) = pj;
            c = p;
        }
        D(c) = dd;
        J(c) = jj;
        if (size == k) {
            top_d = D(0);
            top_j = J(0);
        }
    }
    // Put (dd, jj) at the root of a heap of n entries and sift it down.
    __device__ __forceinline__ void sift_root(float dd, uint32_t jj, int n) {
        int c = 0;
        for (;;) {
            const int l = 2 * c + 1;
            if (l >= n) break;
            int g = l;
            if (l + 1 < n && less(D(l), J(l), D(l + 1), J(l + 1))) g = l + 1;
            if (!less(dd, jj, D(g), J(g))) break;
            D(c) = D(g);
            J(c) = J(g);
            c = g;
        }
        D(c) = dd;
        J(c) = jj;
    }
    __device__ __forceinline__ void offer(float dd, uint32_t jj, float r2) {
        if (!(dd <= r2)) return;
        if (size < k) {
            push(dd, jj);
        } else if (dd < top_d || (dd == top_d && record_id(rec[jj]) < record_id(rec[top_j]))) {
            sift_root(dd, jj, size);
            top_d = D(0);
            top_j = J(0);
        }
    }
};

__device__ __forceinline__ void scan_range(KnnHeap& h, const float4* __restrict__ pos, uint32_t a, uint32_t b,
                                           float px, float py, float pz, float r2) {
    uint32_t jj = a;
    for (; jj + 4 <= b; jj += 4) {
        float4 q[4];
#pragma unroll
        for (int u = 0; u < 4; u++) q[u] = __ldg(pos + jj + u);
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const float ex = q[u].x - px, ey = q[u].y - py, ez = q[u].z - pz;
            h.offer(ex * ex + ey * ey + ez * ez, jj + u, r2);
        }
    }
    for (; jj < b; jj++) {
        const float4 q = __ldg(pos + jj);
        const float ex = q.x - px, ey = q.y - py, ez = q.z - pz;
        h.offer(ex * ex + ey * ey + ez * ez, jj, r2);
    }
}

__global__ void __launch_bounds__(kKnnBlock) k_knn_query(rl::DevMap m, const float4* __restrict__ pos,
                                                         const PhotonRecord* __restrict__ rec,
                                                         const uint32_t* __restrict__ start, KnnGrid g, float r2,
                                                         float radius, int k) {
    extern __shared__ float smem[];
    const int t = threadIdx.x;
    const int x = blockIdx.x * kKnnTile + (t % kKnnTile), y = blockIdx.y * kKnnTile + (t / kKnnTile);
    if (x >= m.width || y >= m.height) return;
    const long long i = (long long)y * m.width + x;
    if (!(m.flags[i] & 1)) return;
    const float px = m.position[3 * i], py = m.position[3 * i + 1], pz = m.position[3 * i + 2];
    KnnHeap h{smem, reinterpret_cast<uint32_t*>(smem + (size_t)k * kKnnBlock), rec, t, 0, k, 0.f, 0u};
    if (g.nx > 0) {
        // pass 1: the cells within one cell of the lumel
        const float h1 = g.cell;
        // covers the rounding of px - h1 (and of g1 below), many times over
        const float margin = (fabsf(px) + fabsf(py) + fabsf(pz) + h1) * (1.0f / (1 << 20)) + 1e-30f;
        const int lx = cell_axis(px - h1, g.ox, g.inv, g.nx), hx = cell_axis(px + h1, g.ox, g.inv, g.nx);
        const int ly = cell_axis(py - h1, g.oy, g.inv, g.ny), hy = cell_axis(py + h1, g.oy, g.inv, g.ny);
        const int lz = cell_axis(pz - h1, g.oz, g.inv, g.nz), hz = cell_axis(pz + h1, g.oz, g.inv, g.nz);
        for (int cz = lz; cz <= hz; cz++)
            for (int cy = ly; cy <= hy; cy++) {
                const long long row = ((long long)cz * g.ny + cy) * g.nx;
                scan_range(h, pos, start[row + lx], start[row + hx + 1], px, py, pz, r2);
            }
        // cell_axis is monotone, so a record in a cell below lx lies below
        // px - h1 as rounded (above hx: above px + h1; the same along y and
        // z): it is farther than g1 along that axis, and its squared
        // distance, rounded, is at least g1 * g1.
        const float g1 = h1 - margin;
        const float t1 = g1 > 0.f ? g1 * g1 : 0.f;
        const bool done = t1 > r2 || (h.size == k && t1 > h.top_d);
        if (!done) {
            // pass 2: the cells within the radius, minus those of pass 1.  A
            // record with a rounded squared distance <= r2 lies within
            // radius * (1 + 2^-22) along each axis, well inside h2.
            const float h2 = radius * (1.0f + 1.0f / 65536) + 4.f * margin;
            const int Lx = min(lx, cell_axis(px - h2, g.ox, g.inv, g.nx)), Hx = max(hx, cell_axis(px + h2, g.ox, g.inv, g.nx));
            const int Ly = min(ly, cell_axis(py - h2, g.oy, g.inv, g.ny)), Hy = max(hy, cell_axis(py + h2, g.oy, g.inv, g.ny));
            const int Lz = min(lz, cell_axis(pz - h2, g.oz, g.inv, g.nz)), Hz = max(hz, cell_axis(pz + h2, g.oz, g.inv, g.nz));
            for (int cz = Lz; cz <= Hz; cz++)
                for (int cy = Ly; cy <= Hy; cy++) {
                    const long long row = ((long long)cz * g.ny + cy) * g.nx;
                    if (cz >= lz && cz <= hz && cy >= ly && cy <= hy) {
                        scan_range(h, pos, start[row + Lx], start[row + lx], px, py, pz, r2);
                        scan_range(h, pos, start[row + hx + 1], start[row + Hx + 1], px, py, pz, r2);
                    } else {
                        scan_range(h, pos, start[row + Lx], start[row + Hx + 1], px, py, pz, r2);
                    }
                }
        }
    }
    // heapsort: ascending (d2, id)
    for (int e = h.size - 1; e > 0; e--) {
        const float td = h.D(e);
        const uint32_t tj = h.J(e);
        h.D(e) = h.D(0);
        h.J(e) = h.J(0);
        h.sift_root(td, tj, e);
    }
    float sr = 0.f, sg = 0.f, sb = 0.f;
    for (int e = 0; e < h.size; e++) {
        const PhotonRecord& r = rec[h.J(e)];
        sr += r.r;
        sg += r.g;
        sb += r.b;
    }
    if (h.size > 0) {
        const float n = (float)h.size;
        m.gathered[3 * i] = sr / n;
        m.gathered[3 * i + 1] = sg / n;
        m.gathered[3 * i + 2] = sb / n;
    } else {
        m.gathered[3 * i] = m.gathered[3 * i + 1] = m.gathered[3 * i + 2] = 0.f;
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
    const size_t smem = (size_t)k * kKnnBlock * 8;
    static bool attr = false;
    if (!attr) {
        KCK(cudaFuncSetAttribute(k_knn_query, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxK * kKnnBlock * 8));
        attr = true;
    }
    const dim3 grid((unsigned)((m->width + kKnnTile - 1) / kKnnTile), (unsigned)((m->height + kKnnTile - 1) / kKnnTile));
    k_knn_query<<<grid, kKnnBlock, smem, st>>>(*m, p->pos, p->sorted, p->start, g, radius * radius, radius, k);
    KCK(cudaGetLastError());
    return RL_OK;
}
