// Device BVH builder: linear BVH over Morton-ordered triangle centroids
// (Karras, "Maximizing parallelism in the construction of BVHs, octrees, and
// k-d trees", HPG 2012), emitted in the traversal layout of rl_device.cuh
// (64-byte binary nodes with both children's boxes, 48-byte v0/e1/e2
// triangle records, one triangle per leaf).
//
//   k_lbvh_boxes   padded triangle boxes (the host builder's padding) and the
//                  centroid bounds (atomic min/max on order-preserving ints)
//   k_lbvh_morton  30-bit Morton code of each centroid, made unique by the
//                  triangle id in the low 32 bits; CUB radix sort
//   k_lbvh_karras  each internal node's key range, split and children
//   k_lbvh_up      bottom-up boxes: the second thread to reach a node writes it
//   k_lbvh_tris    triangle records in leaf order
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <cstdint>

#include "rl_lbvh.h"

namespace rl {
namespace {

__device__ __forceinline__ unsigned f2o(float f) {  // order-preserving float -> uint
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_lbvh_boxes(const float* pos, const int4* vidx, int n, float* box, unsigned* cbounds) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int4 f = vidx[t];
    int v[3] = {f.x, f.y, f.z};
    float lo[3], hi[3];
    for (int k = 0; k < 3; k++) { lo[k] = 3.402823466e+38f; hi[k] = -3.402823466e+38f; }
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 3; k++) {
            float p = pos[3 * v[c] + k];
            lo[k] = fminf(lo[k], p);
            hi[k] = fmaxf(hi[k], p);
        }
    for (int k = 0; k < 3; k++) {
        float m = fmaxf(fabsf(lo[k]), fabsf(hi[k]));
        float pad = 1e-5f * fmaxf(1.0f, m);
        lo[k] -= pad;
        hi[k] += pad;
        box[6 * (size_t)t + k] = lo[k];
        box[6 * (size_t)t + 3 + k] = hi[k];
        float c = 0.5f * (lo[k] + hi[k]);
        atomicMin(&cbounds[k], f2o(c));
        atomicMax(&cbounds[3 + k], f2o(c));
    }
}

__device__ __forceinline__ unsigned spread10(unsigned x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__global__ void k_lbvh_morton(const float* box, const unsigned* cbounds, int n, unsigned long long* keys) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    unsigned q[3];
    for (int k = 0; k < 3; k++) {
        float lo = o2f(cbounds[k]), hi = o2f(cbounds[3 + k]);
        float c = 0.5f * (box[6 * (size_t)t + k] + box[6 * (size_t)t + 3 + k]);
        float ext = hi - lo;
        float u = ext > 0.0f ? (c - lo) / ext : 0.0f;
        int qi = (int)(u * 1023.0f);
        q[k] = (unsigned)(qi < 0 ? 0 : (qi > 1023 ? 1023 : qi));
    }
    unsigned m = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    keys[t] = ((unsigned long long)m << 32) | (unsigned)t;
}

__device__ __forceinline__ int delta(const unsigned long long* keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(keys[i] ^ keys[j]);
}

// Internal node i of n - 1: children in child[2i], child[2i+1] (>= 0
// internal node, < 0 leaf ~k for sorted triangle k); parents recorded.
__global__ void k_lbvh_karras(const unsigned long long* keys, int n, int* child, int* parent_int, int* parent_leaf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0;
    int div = 2;
    for (;;) {
        int t = (l + div - 1) / div;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
        div <<= 1;
    }
    int gamma = i + s * d + (d < 0 ? -1 : 0);
    int lo = i < j ? i : j, hi = i < j ? j : i;
    int left = (lo == gamma) ? ~gamma : gamma;
    int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    child[2 * i] = left;
    child[2 * i + 1] = right;
    if (left < 0) parent_leaf[~left] = i; else parent_int[left] = i;
    if (right < 0) parent_leaf[~right] = i; else parent_int[right] = i;
}

__device__ __forceinline__ void load_box(const float* nbox, const float* tbox, const unsigned long long* keys, int c,
                                         float b[6]) {
    if (c < 0) {
        unsigned t = (unsigned)(keys[~c] & 0xffffffffu);
        for (int k = 0; k < 6; k++) b[k] = __ldcg(tbox + 6 * (size_t)t + k);
    } else {
        for (int k = 0; k < 6; k++) b[k] = __ldcg(nbox + 6 * (size_t)c + k);
    }
}

// Bottom-up pass, one thread per leaf: the second thread to reach an internal
// node writes the node (both children's boxes) and its union box, then climbs.
__global__ void k_lbvh_up(const unsigned long long* keys, int n, const int* child, const int* parent_int,
                          const int* parent_leaf, const float* tbox, float* nbox, int* arrivals, float* nodes) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int p = parent_leaf[k];
    while (p >= 0) {
        __threadfence();
        if (atomicAdd(&arrivals[p], 1) == 0) return;  // first arrival: the sibling finishes the node
        __threadfence();
        int c0 = child[2 * p], c1 = child[2 * p + 1];
        float a[6], b[6];
        load_box(nbox, tbox, keys, c0, a);
        load_box(nbox, tbox, keys, c1, b);
        float* dst = nodes + 16 * (size_t)p;
        dst[0] = a[0]; dst[1] = a[3]; dst[2] = a[1]; dst[3] = a[4];
        dst[4] = b[0]; dst[5] = b[3]; dst[6] = b[1]; dst[7] = b[4];
        dst[8] = a[2]; dst[9] = a[5]; dst[10] = b[2]; dst[11] = b[5];
        int code0 = c0 >= 0 ? c0 : ~(((~c0) << 3) | 0);
        int code1 = c1 >= 0 ? c1 : ~(((~c1) << 3) | 0);
        dst[12] = __int_as_float(code0);
        dst[13] = __int_as_float(code1);
        dst[14] = 0.0f;
        dst[15] = 0.0f;
        for (int q = 0; q < 3; q++) {
            nbox[6 * (size_t)p + q] = fminf(a[q], b[q]);
            nbox[6 * (size_t)p + 3 + q] = fmaxf(a[3 + q], b[3 + q]);
        }
        p = parent_int[p];
    }
}

__global__ void k_lbvh_tris(const unsigned long long* keys, int n, const float* pos, const int4* vidx, float* tris) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int t = (int)(keys[k] & 0xffffffffu);
    int4 f = vidx[t];
    const float* p0 = pos + 3 * (size_t)f.x;
    const float* p1 = pos + 3 * (size_t)f.y;
    const float* p2 = pos + 3 * (size_t)f.z;
    float* r = tris + 12 * (size_t)k;
    r[0] = p0[0]; r[1] = p0[1]; r[2] = p0[2];
    r[3] = __int_as_float(t);
    for (int q = 0; q < 3; q++) {
        r[4 + q] = p1[q] - p0[q];
        r[8 + q] = p2[q] - p0[q];
    }
    r[7] = 0.0f;
    r[11] = 0.0f;
}

// A one-triangle tree: a root whose two children are that leaf.
__global__ void k_lbvh_single(const float* tbox, float* nodes) {
    float a[6];
    for (int k = 0; k < 6; k++) a[k] = tbox[k];
    float vals[12] = {a[0], a[3], a[1], a[4], a[0], a[3], a[1], a[4], a[2], a[5], a[2], a[5]};
    for (int k = 0; k < 12; k++) nodes[k] = vals[k];
    int code = ~0;
    nodes[12] = __int_as_float(code);
    nodes[13] = __int_as_float(code);
    nodes[14] = 0.0f;
    nodes[15] = 0.0f;
}

}  // namespace

#define LCK(call)                                                       \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) {                                        \
            *err = cudaGetErrorString(e_);                              \
            goto done;                                                  \
        }                                                               \
    } while (0)

bool build_lbvh_device(const float* d_pos, const int4* d_vidx, int n, cudaStream_t st, float4** d_nodes,
                       float4** d_tris, int64_t* nnodes, int* depth, const char** err) {
    *d_nodes = nullptr;
    *d_tris = nullptr;
    *nnodes = 0;
    *depth = 0;
    if (n <= 0) return true;
    if (n >= (1 << 28)) {
        *err = "too many triangles for the 28-bit leaf encoding";
        return false;
    }
    bool ok = false;
    float *tbox = nullptr, *nbox = nullptr, *nodes = nullptr, *tris = nullptr;
    unsigned* cb = nullptr;
    unsigned long long *keys = nullptr, *keys_sorted = nullptr;
    int *child = nullptr, *pint = nullptr, *pleaf = nullptr, *arrivals = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    int ni = n > 1 ? n - 1 : 1;
    unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    LCK(cudaMallocAsync((void**)&tbox, 24 * (size_t)n, st));
    LCK(cudaMallocAsync((void**)&cb, 24, st));
    LCK(cudaMemcpyAsync(cb, init, 24, cudaMemcpyHostToDevice, st));
    k_lbvh_boxes<<<(n + 255) / 256, 256, 0, st>>>(d_pos, d_vidx, n, tbox, cb);
    LCK(cudaGetLastError());
    LCK(cudaMalloc((void**)&nodes, 64 * (size_t)ni));
    LCK(cudaMalloc((void**)&tris, 48 * (size_t)n));
    if (n == 1) {
        LCK(cudaMallocAsync((void**)&keys_sorted, 8, st));
        LCK(cudaMemsetAsync(keys_sorted, 0, 8, st));
        k_lbvh_single<<<1, 1, 0, st>>>(tbox, nodes);
        LCK(cudaGetLastError());
        k_lbvh_tris<<<1, 32, 0, st>>>(keys_sorted, 1, d_pos, d_vidx, tris);
        LCK(cudaGetLastError());
        LCK(cudaStreamSynchronize(st));
        *nnodes = 1;
        *depth = 1;
        ok = true;
        goto done;
    }
    LCK(cudaMallocAsync((void**)&keys, 8 * (size_t)n, st));
    LCK(cudaMallocAsync((void**)&keys_sorted, 8 * (size_t)n, st));
    k_lbvh_morton<<<(n + 255) / 256, 256, 0, st>>>(tbox, cb, n, keys);
    LCK(cudaGetLastError());
    LCK(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, keys, keys_sorted, n, 0, 64, st));
    LCK(cudaMallocAsync(&temp, temp_bytes, st));
    LCK(cub::DeviceRadixSort::SortKeys(temp, temp_bytes, keys, keys_sorted, n, 0, 64, st));
    LCK(cudaMallocAsync((void**)&child, 8 * (size_t)ni, st));
    LCK(cudaMallocAsync((void**)&pint, 4 * (size_t)ni, st));
    LCK(cudaMallocAsync((void**)&pleaf, 4 * (size_t)n, st));
    LCK(cudaMallocAsync((void**)&arrivals, 4 * (size_t)ni, st));
    LCK(cudaMallocAsync((void**)&nbox, 24 * (size_t)ni, st));
    LCK(cudaMemsetAsync(arrivals, 0, 4 * (size_t)ni, st));
    LCK(cudaMemsetAsync(pint, 0xff, 4 * (size_t)ni, st));  // the root's parent stays -1
    k_lbvh_karras<<<(ni + 255) / 256, 256, 0, st>>>(keys_sorted, n, child, pint, pleaf);
    LCK(cudaGetLastError());
    k_lbvh_up<<<(n + 255) / 256, 256, 0, st>>>(keys_sorted, n, child, pint, pleaf, tbox, nbox, arrivals, nodes);
    LCK(cudaGetLastError());
    k_lbvh_tris<<<(n + 255) / 256, 256, 0, st>>>(keys_sorted, n, d_pos, d_vidx, tris);
    LCK(cudaGetLastError());
    {
        // depth, for the traversal stack bound: walk parents on the host
        int* hp = new int[ni];
        int* hl = new int[n];
        cudaError_t e1 = cudaMemcpyAsync(hp, pint, 4 * (size_t)ni, cudaMemcpyDeviceToHost, st);
        cudaError_t e2 = cudaMemcpyAsync(hl, pleaf, 4 * (size_t)n, cudaMemcpyDeviceToHost, st);
        cudaError_t e3 = cudaStreamSynchronize(st);
        int dmax = 0;
        if (e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess) {
            for (int k = 0; k < n; k++) {
                int d = 1, p = hl[k];
                while (p >= 0 && d < 4096) { d++; p = hp[p]; }
                if (d > dmax) dmax = d;
            }
        }
        delete[] hp;
        delete[] hl;
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
            *err = "LBVH read-back failed";
            goto done;
        }
        *depth = dmax;
    }
    *nnodes = ni;
    ok = true;
done:
    cudaFreeAsync(tbox, st);
    cudaFreeAsync(cb, st);
    cudaFreeAsync(keys, st);
    cudaFreeAsync(keys_sorted, st);
    cudaFreeAsync(temp, st);
    cudaFreeAsync(child, st);
    cudaFreeAsync(pint, st);
    cudaFreeAsync(pleaf, st);
    cudaFreeAsync(arrivals, st);
    cudaFreeAsync(nbox, st);
    if (!ok) {
        cudaFree(nodes);
        cudaFree(tris);
        return false;
    }
    *d_nodes = (float4*)nodes;
    *d_tris = (float4*)tris;
    return true;
}

}  // namespace rl
