// k-nearest-neighbour photon estimate over a hashed grid.
//
// The reference estimates irradiance with a disc gather in texel space
// (Photonmap::gather, Lightmap.cpp:376-413): the mean photon colour over
// the texels within a radius.  This is the world-space counterpart with
// the same meaning: at each valid lumel of a photonmap, the mean colour of
// the k photon deposits nearest to the lumel's position (within a radius
// cap), the deposits being exactly those Photons::store adds to that
// photonmap (rl_emit_photons_records keeps each one as a record).
//
//   build:  every record gets key = (bucket of its grid cell, record id);
//           one radix sort orders the records by bucket, then by id, and
//           each bucket's range [begin, end) is marked.  Cells are
//           `radius` wide and hashed into a power-of-two table, so the
//           grid needs no scene bounds.
//   query:  one thread per lumel visits the 27 cells around it (each
//           bucket once), keeps the k nearest records in a max-heap in
//           shared memory ordered by (squared distance, record id), and
//           sums their colours in that order, so the result does not
//           depend on emission order or thread timing.
// Lumels that are not valid keep the disc gather's value.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/relight_b200.h"
#include "rl_device.cuh"
#include "rl_photon_records.h"

int rl_internal_fail(int code, const char* msg);
const rl::DevMap* rl_internal_map(const rl_map* m);

struct rl_photons {
    PhotonRecord* rec = nullptr;     // emission order
    PhotonRecord* sorted = nullptr;  // grid order
    unsigned long long* d_count = nullptr;
    long long capacity = 0;
    uint64_t *keys = nullptr, *keys_out = nullptr;
    uint32_t *idx = nullptr, *idx_out = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    uint32_t *begin = nullptr, *end = nullptr;
    uint32_t table = 0;
    ~rl_photons() {
        cudaFree(rec);
        cudaFree(sorted);
        cudaFree(d_count);
        cudaFree(keys);
        cudaFree(keys_out);
        cudaFree(idx);
        cudaFree(idx_out);
        cudaFree(temp);
        cudaFree(begin);
        cudaFree(end);
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
constexpr int kKnnBlock = 64;

__device__ __forceinline__ uint32_t cell_bucket(int ix, int iy, int iz, uint32_t mask) {
    return (((uint32_t)ix * 73856093u) ^ ((uint32_t)iy * 19349663u) ^ ((uint32_t)iz * 83492791u)) & mask;
}

__device__ __forceinline__ int cell_of(float v, float cell) { return (int)floorf(v / cell); }

__global__ void k_knn_keys(const PhotonRecord* rec, long long n, float cell, uint32_t mask, uint64_t* keys,
                           uint32_t* idx) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const PhotonRecord& r = rec[i];
        uint32_t b = cell_bucket(cell_of(r.x, cell), cell_of(r.y, cell), cell_of(r.z, cell), mask);
        keys[i] = ((uint64_t)b << 36) | record_id(r);
        idx[i] = (uint32_t)i;
    }
}

__global__ void k_knn_scatter(const PhotonRecord* rec, const uint64_t* keys, const uint32_t* idx, long long n,
                              PhotonRecord* sorted, uint32_t* begin, uint32_t* end) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        sorted[i] = rec[idx[i]];
        uint32_t b = (uint32_t)(keys[i] >> 36);
        if (i == 0 || (uint32_t)(keys[i - 1] >> 36) != b) begin[b] = (uint32_t)i;
        if (i == n - 1 || (uint32_t)(keys[i + 1] >> 36) != b) end[b] = (uint32_t)(i + 1);
    }
}

// (d2, id) ordering of heap entries; ids are read only on distance ties.
__device__ __forceinline__ bool entry_less(float da, uint32_t ia, float db, uint32_t ib, const PhotonRecord* rec) {
    if (da != db) return da < db;
    return record_id(rec[ia]) < record_id(rec[ib]);
}

// One thread per lumel of the photonmap; heaps in shared memory, entry e
// of thread t at [e * kKnnBlock + t].
__global__ void __launch_bounds__(kKnnBlock) k_knn_query(rl::DevMap m, int slot, const PhotonRecord* rec,
                                                         const uint32_t* begin, const uint32_t* end, uint32_t mask,
                                                         float cell, float r2, int k) {
    extern __shared__ float smem[];
    float* hd = smem;
    uint32_t* hi = reinterpret_cast<uint32_t*>(smem + (size_t)k * kKnnBlock);
    const int t = threadIdx.x;
    const long long i = blockIdx.x * (long long)kKnnBlock + t;
    if (i >= (long long)m.width * m.height || !(m.flags[i] & 1)) return;
    const float px = m.position[3 * i], py = m.position[3 * i + 1], pz = m.position[3 * i + 2];
    const int cx = cell_of(px, cell), cy = cell_of(py, cell), cz = cell_of(pz, cell);
    uint32_t seen[27];
    int nseen = 0, hs = 0;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const uint32_t b = cell_bucket(cx + dx, cy + dy, cz + dz, mask);
                bool dup = false;
                for (int q = 0; q < nseen; q++) dup |= seen[q] == b;
                if (dup) continue;
                seen[nseen++] = b;
                for (uint32_t j = begin[b]; j < end[b]; j++) {
                    const PhotonRecord& r = rec[j];
                    if (r.slot != slot) continue;
                    const float ex = r.x - px, ey = r.y - py, ez = r.z - pz;
                    const float d2 = ex * ex + ey * ey + ez * ez;
                    if (!(d2 <= r2)) continue;
                    if (hs < k) {  // push, sift up
                        int c = hs++;
                        while (c > 0) {
                            int p = (c - 1) >> 1;
                            float pd = hd[p * kKnnBlock + t];
                            uint32_t pi = hi[p * kKnnBlock + t];
                            if (!entry_less(pd, pi, d2, j, rec)) break;
                            hd[c * kKnnBlock + t] = pd;
                            hi[c * kKnnBlock + t] = pi;
                            c = p;
                        }
                        hd[c * kKnnBlock + t] = d2;
                        hi[c * kKnnBlock + t] = j;
                    } else if (entry_less(d2, j, hd[t], hi[t], rec)) {  // replace the largest, sift down
                        int c = 0;
                        for (;;) {
                            int l = 2 * c + 1;
                            if (l >= hs) break;
                            int g = l;
                            if (l + 1 < hs && entry_less(hd[l * kKnnBlock + t], hi[l * kKnnBlock + t],
                                                         hd[(l + 1) * kKnnBlock + t], hi[(l + 1) * kKnnBlock + t], rec))
                                g = l + 1;
                            if (!entry_less(d2, j, hd[g * kKnnBlock + t], hi[g * kKnnBlock + t], rec)) break;
                            hd[c * kKnnBlock + t] = hd[g * kKnnBlock + t];
                            hi[c * kKnnBlock + t] = hi[g * kKnnBlock + t];
                            c = g;
                        }
                        hd[c * kKnnBlock + t] = d2;
                        hi[c * kKnnBlock + t] = j;
                    }
                }
            }
    // heapsort: ascending (d2, id)
    for (int e = hs - 1; e > 0; e--) {
        float td = hd[e * kKnnBlock + t];
        uint32_t ti = hi[e * kKnnBlock + t];
        hd[e * kKnnBlock + t] = hd[t];
        hi[e * kKnnBlock + t] = hi[t];
        int c = 0;
        for (;;) {
            int l = 2 * c + 1;
            if (l >= e) break;
            int g = l;
            if (l + 1 < e && entry_less(hd[l * kKnnBlock + t], hi[l * kKnnBlock + t], hd[(l + 1) * kKnnBlock + t],
                                        hi[(l + 1) * kKnnBlock + t], rec))
                g = l + 1;
            if (!entry_less(td, ti, hd[g * kKnnBlock + t], hi[g * kKnnBlock + t], rec)) break;
            hd[c * kKnnBlock + t] = hd[g * kKnnBlock + t];
            hi[c * kKnnBlock + t] = hi[g * kKnnBlock + t];
            c = g;
        }
        hd[c * kKnnBlock + t] = td;
        hi[c * kKnnBlock + t] = ti;
    }
    float sr = 0.f, sg = 0.f, sb = 0.f;
    for (int e = 0; e < hs; e++) {
        const PhotonRecord& r = rec[hi[e * kKnnBlock + t]];
        sr += r.r;
        sg += r.g;
        sb += r.b;
    }
    if (hs > 0) {
        float n = (float)hs;
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
    if (!out || capacity <= 0 || capacity > (1ll << 31)) return kfail(RL_INVALID_CALL, "rl_photons_create: bad capacity");
    *out = nullptr;
    rl_photons* p = new (std::nothrow) rl_photons;
    if (!p) return kfail(RL_OUT_OF_MEMORY, "host allocation failed");
    p->capacity = capacity;
    size_t n = (size_t)capacity;
    cudaError_t e = cudaMalloc(&p->rec, n * sizeof(PhotonRecord));
    if (e == cudaSuccess) e = cudaMalloc(&p->sorted, n * sizeof(PhotonRecord));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_count, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&p->keys, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&p->keys_out, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&p->idx, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->idx_out, n * 4);
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

extern "C" int rl_photonmap_gather_knn(rl_map* map, int slot, rl_photons* p, int k, float radius, void* stream) {
    const rl::DevMap* m = rl_internal_map(map);
    if (!m || !p) return kfail(RL_INVALID_CALL, "rl_photonmap_gather_knn: null argument");
    if (k < 1 || k > kMaxK) return kfail(RL_INVALID_CALL, "rl_photonmap_gather_knn: k must be in [1, %d]", kMaxK);
    if (!(radius > 0.f)) return kfail(RL_INVALID_CALL, "rl_photonmap_gather_knn: radius must be positive");
    if (slot < 0 || slot > 0xffff) return kfail(RL_INVALID_CALL, "rl_photonmap_gather_knn: bad slot");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long h = 0;
    KCK(cudaMemcpyAsync(&h, p->d_count, sizeof h, cudaMemcpyDeviceToHost, st));
    KCK(cudaStreamSynchronize(st));
    if (h > (unsigned long long)p->capacity)
        return kfail(RL_CAPACITY, "rl_photonmap_gather_knn: %llu deposits exceed the record capacity %lld", h,
                     p->capacity);
    const long long n = (long long)h;
    // hash table: a power of two >= 2n (>= 1024), at most 2^27 buckets
    uint32_t table = 1024;
    while ((long long)table < 2 * n && table < (1u << 27)) table <<= 1;
    if (table != p->table) {
        cudaFree(p->begin);
        cudaFree(p->end);
        p->begin = p->end = nullptr;
        p->table = 0;
        KCK(cudaMalloc(&p->begin, (size_t)table * 4));
        KCK(cudaMalloc(&p->end, (size_t)table * 4));
        p->table = table;
    }
    KCK(cudaMemsetAsync(p->begin, 0, (size_t)table * 4, st));
    KCK(cudaMemsetAsync(p->end, 0, (size_t)table * 4, st));
    if (n > 0) {
        int bits = 36;
        while ((1u << (bits - 36)) < table) bits++;
        k_knn_keys<<<grid_blocks(n, 256), 256, 0, st>>>(p->rec, n, radius, table - 1, p->keys, p->idx);
        size_t tb = p->temp_bytes;
        KCK(cub::DeviceRadixSort::SortPairs(p->temp, tb, p->keys, p->keys_out, p->idx, p->idx_out, (int)n, 0, bits, st));
        k_knn_scatter<<<grid_blocks(n, 256), 256, 0, st>>>(p->rec, p->keys_out, p->idx_out, n, p->sorted, p->begin,
                                                           p->end);
    }
    const size_t smem = (size_t)k * kKnnBlock * 8;
    static bool attr = false;
    if (!attr) {
        KCK(cudaFuncSetAttribute(k_knn_query, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxK * kKnnBlock * 8));
        attr = true;
    }
    const long long texels = (long long)m->width * m->height;
    k_knn_query<<<(unsigned)((texels + kKnnBlock - 1) / kKnnBlock), kKnnBlock, smem, st>>>(
        *m, slot, p->sorted, p->begin, p->end, table - 1, radius, radius * radius, k);
    KCK(cudaGetLastError());
    return RL_OK;
}
