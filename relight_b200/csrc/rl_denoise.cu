// Lightmap denoiser: a 4-level convolutional encoder-decoder over BF16
// activations, trained and run with hand-written sm_100a tensor-core
// kernels (tcgen05.mma, FP32 accumulation in tensor memory, operands staged
// by TMA).
//
// Layout.  Activations are NHWC BF16 with the channel count padded to a
// multiple of 16.  A 3x3 "same" convolution is an implicit GEMM:
//   M = 128 output pixels (a 16 x 8 spatial tile), N = output channels,
//   K = 9 taps x input channels in blocks of 64.
// For each (tap, channel block) the A tile is one TMA box of the input at
// the tap's offset; pixels outside the image come back as zeros, which is
// the convolution's zero padding.  Weights are BF16 [Co][9][Ci_pad64] (the
// forward pass) or, for the data gradient, [Ci][9][Co_pad64] with the taps
// flipped; both are K-major B tiles of one box per (tap, block).  The weight
// gradient is a second GEMM with K = pixels: the gradient and the shifted
// input are the same TMA boxes, read by the tensor core as MN-major
// operands.
//
// Every wait on an mbarrier is bounded; a wait that runs out sets an error
// flag that the host reads back, and the kernel still releases its tensor
// memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/relight_b200.h"
#include "rl_device.cuh"

int rl_internal_fail(int code, const char* msg);
const rl::DevMap* rl_internal_map(const rl_map* m);
const rl::DevScene* rl_internal_scene(const rl_scene* s);

namespace {

using bf16 = __nv_bfloat16;

int dn_fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return rl_internal_fail(code, buf);
}

#define DN_CK(call)                                                                                 \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return dn_fail(RL_CUDA_ERROR, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------ PTX helpers

constexpr uint32_t kSpinLimit = 1u << 22;  // bounded mbarrier waits (about a second)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of parity `parity`; false (and err |= code) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
    for (uint32_t i = 0; i < kSpinLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, code);
    return false;
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6}], [%2];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, uint64_t* bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
        "%5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, BF16 inputs, FP32 accumulate.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on `bar` once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns of tensor memory.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor, 128-byte swizzle (the layout TMA writes
// with CU_TENSOR_MAP_SWIZZLE_128B): start address, leading / stride byte
// offsets (16-byte units), descriptor version 1, layout type 2.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool a_mn_major, bool b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((b_mn_major ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
    uint32_t a = smem_u32(p);
    return p + ((1024 - (a & 1023)) & 1023);
}

// ------------------------------------------------------- the conv kernel

constexpr int kTileW = 16, kTileH = 8;   // 128 output pixels per tile
constexpr uint32_t kABytes = 128 * 128;   // 128 pixels x 64 channels x 2 bytes

struct ConvArgs {
    int W, H;              // spatial size (input = output)
    int nblk[2];           // 64-channel blocks per input segment
    int ncols;             // MMA N = output channels (multiple of 16, <= 256)
    int tmem_cols;         // power of two >= max(32, ncols)
    int stages;
    const float* bias;     // [ncols] or null
    int relu;
    // output segments: accumulator columns [c0, c0 + cn) -> tensor out (cstride channels)
    bf16* out[2];
    int out_c0[2], out_cn[2], out_cs[2];
    const bf16* mask[2];   // optional: out *= (mask > 0), same layout as out
    int nout;
    int* err;
};

// Implicit-GEMM 3x3 convolution (forward, or data gradient with flipped
// transposed weights).  Warp 0 lane 0 issues TMA, warp 1 lane 0 issues the
// MMAs, all four warps run the epilogue (warp w reads TMEM lanes 32w..32w+31,
// i.e. output pixels 32w..32w+31 of the tile).
__global__ void __launch_bounds__(128, 2) k_conv3x3(const __grid_constant__ CUtensorMap tmA0,
                                                   const __grid_constant__ CUtensorMap tmA1,
                                                   const __grid_constant__ CUtensorMap tmB, const ConvArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align1024(smem_raw);
    const int S = a.stages;
    const uint32_t b_bytes = (uint32_t)a.ncols * 128;
    uint8_t* sa = smem;
    uint8_t* sb = smem + S * kABytes;
    uint64_t* full = (uint64_t*)(sb + S * b_bytes);
    uint64_t* empty = full + S;
    uint64_t* done = empty + S;
    uint32_t* tmem_slot = (uint32_t*)(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH, img = blockIdx.z;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        mbar_init(done, 1);
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, a.tmem_cols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int per_tap = a.nblk[0] + a.nblk[1];
    const int total = 9 * per_tap;

    if (warp == 0 && lane == 0) {
        int issued = 0;
        for (int kb = 0; kb < total; kb++) {
            const int s = kb % S, round = kb / S;
            if (!mbar_wait(empty + s, (round & 1) ^ 1, a.err, 1)) break;
            const int tap = kb / per_tap, j = kb % per_tap;
            const int seg = j < a.nblk[0] ? 0 : 1, cb = seg ? j - a.nblk[0] : j;
            mbar_expect_tx(full + s, kABytes + b_bytes);
            tma_load_4d(sa + s * kABytes, seg ? &tmA1 : &tmA0, full + s, cb * 64, x0 + tap % 3 - 1, y0 + tap / 3 - 1,
                        img);
            tma_load_3d(sb + s * b_bytes, &tmB, full + s, j * 64, tap, 0);
            issued = kb + 1;
        }
        // no copy may still be landing when the block exits
        for (int kb = issued > S ? issued - S : 0; kb < issued; kb++) mbar_wait(full + kb % S, (kb / S) & 1, a.err, 64);
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = idesc_bf16(a.ncols, false, false);
        for (int kb = 0; kb < total; kb++) {
            const int s = kb % S, round = kb / S;
            if (!mbar_wait(full + s, round & 1, a.err, 2)) break;
            tc_fence_after();
            const uint64_t ad = desc_sw128(smem_u32(sa + s * kABytes), 16, 1024);
            const uint64_t bd = desc_sw128(smem_u32(sb + s * b_bytes), 16, 1024);
#pragma unroll
            for (int kk = 0; kk < 4; kk++)  // K = 16 per MMA: 32 bytes along the swizzled row
                umma_bf16(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0);
            umma_commit(empty + s);
        }
        umma_commit(done);  // also on a timeout: tensor memory is freed only after the issued MMAs
    }
    __syncwarp();

    // epilogue
    const bool finished = mbar_wait(done, 0, a.err, 4);
    tc_fence_after();
    const int row = warp * 32 + lane;
    const int px = x0 + (row % kTileW), py = y0 + (row / kTileW);
    const bool inb = finished && px < a.W && py < a.H;
    const long long pix = ((long long)img * a.H + py) * a.W + px;
    for (int c = 0; c < a.ncols; c += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, r);
        if (!inb) continue;
        for (int o = 0; o < a.nout; o++) {
            if (c < a.out_c0[o] || c >= a.out_c0[o] + a.out_cn[o]) continue;
            const int oc = c - a.out_c0[o];
            float v[16];
#pragma unroll
            for (int i = 0; i < 16; i++) {
                float x = __uint_as_float(r[i]);
                if (a.bias) x += a.bias[c + i];
                if (a.relu) x = fmaxf(x, 0.0f);
                v[i] = x;
            }
            const long long off = pix * a.out_cs[o] + oc;
            if (a.mask[o]) {
                const uint4* mp = reinterpret_cast<const uint4*>(a.mask[o] + off);
                uint4 m0 = mp[0], m1 = mp[1];
                const bf16* mb0 = reinterpret_cast<const bf16*>(&m0);
                const bf16* mb1 = reinterpret_cast<const bf16*>(&m1);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    if (!(__bfloat162float(mb0[i]) > 0.0f)) v[i] = 0.0f;
                    if (!(__bfloat162float(mb1[i]) > 0.0f)) v[8 + i] = 0.0f;
                }
            }
            uint4 w0, w1;
            __nv_bfloat162* p0 = reinterpret_cast<__nv_bfloat162*>(&w0);
            __nv_bfloat162* p1 = reinterpret_cast<__nv_bfloat162*>(&w1);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                p0[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                p1[i] = __floats2bfloat162_rn(v[8 + 2 * i], v[8 + 2 * i + 1]);
            }
            uint4* dst = reinterpret_cast<uint4*>(a.out[o] + off);
            dst[0] = w0;
            dst[1] = w1;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, a.tmem_cols);
}

// ------------------------------------------------- the weight gradient

struct WgradArgs {
    int W, H, N;           // spatial size, images
    int tiles_x, tiles_y;  // pixel tiles per image
    int splits;            // CTAs sharing the pixel range of one (tap, chunk)
    int nb;                // 64-channel input blocks in this launch (N = 64 nb)
    int c_base;            // first input channel of this launch
    int cin;               // input channels of the segment (columns written: c_base + c < cin)
    int cout;              // gradient channels (rows written)
    int ci_off;            // column offset of the segment in dW
    int ci_total;          // dW row length per tap
    int stages;
    float* dw;             // [cout][9][ci_total], accumulated with atomics
    int* err;
};

// dW[co][tap][ci] += sum over pixels p of G[p][co] * X[p + off(tap)][ci].
// GEMM with M = 128 gradient channels (the second 64 read as zeros when
// absent), N = 64 nb input channels, K = pixels; both operands are the
// NHWC boxes as stored, i.e. MN-major.  grid = (9 taps, 1, splits); one
// launch covers input channels [c_base, c_base + 64 nb).
__global__ void __launch_bounds__(128, 1) k_conv3x3_wgrad(const __grid_constant__ CUtensorMap tmG,
                                                         const __grid_constant__ CUtensorMap tmX, const WgradArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align1024(smem_raw);
    const int S = a.stages;
    const uint32_t a_bytes = 2 * kABytes;
    const uint32_t b_bytes = (uint32_t)a.nb * kABytes;
    uint8_t* sa = smem;
    uint8_t* sb = smem + S * a_bytes;
    uint64_t* full = (uint64_t*)(sb + S * b_bytes);
    uint64_t* empty = full + S;
    uint64_t* done = empty + S;
    uint32_t* tmem_slot = (uint32_t*)(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tap = blockIdx.x, split = blockIdx.z;
    const int n = a.nb * 64;
    const uint32_t tcols = n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        mbar_init(done, 1);
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, tcols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const long long tiles = (long long)a.tiles_x * a.tiles_y * a.N;
    const long long mine = tiles > split ? (tiles - split + a.splits - 1) / a.splits : 0;
    const int dx = tap % 3 - 1, dy = tap / 3 - 1;

    if (warp == 0 && lane == 0) {
        long long issued = 0;
        for (long long kb = 0; kb < mine; kb++) {
            const int s = (int)(kb % S);
            const long long round = kb / S;
            if (!mbar_wait(empty + s, (uint32_t)((round & 1) ^ 1), a.err, 8)) break;
            issued = kb + 1;
            const long long t = split + kb * a.splits;
            const int tx = (int)(t % a.tiles_x), ty = (int)((t / a.tiles_x) % a.tiles_y), img = (int)(t / ((long long)a.tiles_x * a.tiles_y));
            const int x0 = tx * kTileW, y0 = ty * kTileH;
            mbar_expect_tx(full + s, a_bytes + b_bytes);
            tma_load_4d(sa + s * a_bytes, &tmG, full + s, 0, x0, y0, img);
            tma_load_4d(sa + s * a_bytes + kABytes, &tmG, full + s, 64, x0, y0, img);
            for (int j = 0; j < a.nb; j++)
                tma_load_4d(sb + s * b_bytes + j * kABytes, &tmX, full + s, a.c_base + j * 64, x0 + dx, y0 + dy, img);
        }
        for (long long kb = issued > S ? issued - S : 0; kb < issued; kb++)
            mbar_wait(full + kb % S, (uint32_t)((kb / S) & 1), a.err, 64);
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = idesc_bf16(n, true, true);
        for (long long kb = 0; kb < mine; kb++) {
            const int s = (int)(kb % S);
            const long long round = kb / S;
            if (!mbar_wait(full + s, (uint32_t)(round & 1), a.err, 16)) break;
            tc_fence_after();
            // MN-major: 64-element blocks along M / N are 16 KB apart (LBO),
            // groups of 8 pixel rows 1 KB apart (SBO); K = 16 pixels per MMA.
            const uint32_t abase = smem_u32(sa + s * a_bytes), bbase = smem_u32(sb + s * b_bytes);
#pragma unroll
            for (int kk = 0; kk < 8; kk++)
                umma_bf16(tmem, desc_sw128(abase + kk * 2048, kABytes, 1024), desc_sw128(bbase + kk * 2048, kABytes, 1024),
                          idesc, (kb | kk) != 0);
            umma_commit(empty + s);
        }
        umma_commit(done);
    }
    __syncwarp();

    const bool finished = mbar_wait(done, 0, a.err, 32) && mine > 0;
    tc_fence_after();
    const int co = warp * 32 + lane;
    for (int c = 0; c < n; c += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, r);
        if (!finished || co >= a.cout) continue;
        const int ci0 = a.c_base + c;
        float* dst = a.dw + ((long long)co * 9 + tap) * a.ci_total + a.ci_off;
#pragma unroll
        for (int i = 0; i < 16; i++)
            if (ci0 + i < a.cin) atomicAdd(dst + ci0 + i, __uint_as_float(r[i]));
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, tcols);
}

// ------------------------------------------------------ tensor maps (host)

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

// NHWC BF16 activations [n][h][w][c] (c a multiple of 8), boxes of 64
// channels x 16 x 8 pixels, 128-byte swizzle, zero fill outside.
int act_map(CUtensorMap* tm, const void* base, int c, int w, int h, int n) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return dn_fail(RL_CUDA_ERROR, "cuTensorMapEncodeTiled unavailable");
    if (c % 8 || ((uintptr_t)base & 15)) return dn_fail(RL_INVALID_CALL, "activation layout: %d channels", c);
    cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * w, (cuuint64_t)c * 2 * w * h};
    cuuint32_t box[4] = {64, kTileW, kTileH, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return dn_fail(RL_CUDA_ERROR, "tensor map (activation) error %d", (int)r);
    return RL_OK;
}

// Weights [rows][9][k] (k a multiple of 64), boxes of 64 x 1 x rows.
int weight_map(CUtensorMap* tm, const void* base, int k, int rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return dn_fail(RL_CUDA_ERROR, "cuTensorMapEncodeTiled unavailable");
    if (k % 64 || rows > 256 || rows % 16) return dn_fail(RL_INVALID_CALL, "weight layout %d x %d", rows, k);
    cuuint64_t dims[3] = {(cuuint64_t)k, 9, (cuuint64_t)rows};
    cuuint64_t strides[2] = {(cuuint64_t)k * 2, (cuuint64_t)k * 2 * 9};
    cuuint32_t box[3] = {64, 1, (cuuint32_t)rows};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return dn_fail(RL_CUDA_ERROR, "tensor map (weights) error %d", (int)r);
    return RL_OK;
}

int pow2_cols(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256; }

int conv_smem(int ncols, int stages) { return stages * (int)(kABytes + ncols * 128) + 2 * stages * 8 + 16 + 1024; }

}  // namespace

// ---------------------------------------------------------------- C ABI

// One 3x3 "same" convolution over NHWC BF16 tensors (see the header).
extern "C" int rl_dn_conv3x3(const void* in0, int c0, const void* in1, int c1, int width, int height, int images,
                             const void* weights, int ncols, const float* bias, int relu, void* out0, int out0_c0,
                             int out0_cn, int out0_cs, const void* mask0, void* out1, int out1_c0, int out1_cn,
                             int out1_cs, const void* mask1, int* d_err, void* stream) {
    if (!in0 || !weights || !out0 || width <= 0 || height <= 0 || images <= 0)
        return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: bad arguments");
    if (ncols < 16 || ncols > 256 || ncols % 16) return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: ncols %d", ncols);
    const int nb0 = (c0 + 63) / 64, nb1 = in1 ? (c1 + 63) / 64 : 0;
    const int nout = out1 ? 2 : 1;
    const int oc0[2] = {out0_c0, out1_c0}, ocn[2] = {out0_cn, out1_cn}, ocs[2] = {out0_cs, out1_cs};
    for (int o = 0; o < nout; o++)
        if (ocn[o] % 16 || ocs[o] % 16 || oc0[o] % 16 || ocn[o] > ocs[o] || oc0[o] + ocn[o] > ncols)
            return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: output segment %d", o);
    CUtensorMap tA0, tA1, tB;
    if (int rc = act_map(&tA0, in0, c0, width, height, images)) return rc;
    if (int rc = act_map(&tA1, in1 ? in1 : in0, in1 ? c1 : c0, width, height, images)) return rc;
    if (int rc = weight_map(&tB, weights, 64 * (nb0 + nb1), ncols)) return rc;
    ConvArgs a;
    memset(&a, 0, sizeof a);
    a.W = width;
    a.H = height;
    a.nblk[0] = nb0;
    a.nblk[1] = nb1;
    a.ncols = ncols;
    a.tmem_cols = pow2_cols(ncols);
    a.stages = ncols > 128 ? 2 : 3;  // two CTAs per SM
    a.bias = bias;
    a.relu = relu;
    a.nout = nout;
    a.out[0] = (bf16*)out0;
    a.out[1] = (bf16*)out1;
    for (int o = 0; o < 2; o++) {
        a.out_c0[o] = oc0[o];
        a.out_cn[o] = ocn[o];
        a.out_cs[o] = ocs[o];
    }
    a.mask[0] = (const bf16*)mask0;
    a.mask[1] = (const bf16*)mask1;
    a.err = d_err;
    const int smem = conv_smem(ncols, a.stages);
    static std::once_flag attr;
    cudaError_t ae = cudaSuccess;
    std::call_once(attr, [&] { ae = cudaFuncSetAttribute(k_conv3x3, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024); });
    if (ae != cudaSuccess) return dn_fail(RL_CUDA_ERROR, "conv smem attribute: %s", cudaGetErrorString(ae));
    dim3 grid((width + kTileW - 1) / kTileW, (height + kTileH - 1) / kTileH, images);
    k_conv3x3<<<grid, 128, smem, (cudaStream_t)stream>>>(tA0, tA1, tB, a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dn_fail(RL_CUDA_ERROR, "k_conv3x3: %s", cudaGetErrorString(e));
    return RL_OK;
}

extern "C" int rl_dn_conv3x3_wgrad(const void* grad, int cout, int grad_cs, const void* in, int cin, int in_cs,
                                   int width, int height, int images, float* dw, int ci_off, int ci_total, int* d_err,
                                   void* stream) {
    if (!grad || !in || !dw || cout <= 0 || cout > 128 || cin <= 0 || width <= 0 || height <= 0 || images <= 0)
        return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3_wgrad: bad arguments");
    CUtensorMap tG, tX;
    if (int rc = act_map(&tG, grad, grad_cs, width, height, images)) return rc;
    if (int rc = act_map(&tX, in, in_cs, width, height, images)) return rc;
    const int blocks = (cin + 63) / 64, chunks = (blocks + 3) / 4;
    WgradArgs a;
    memset(&a, 0, sizeof a);
    a.W = width;
    a.H = height;
    a.N = images;
    a.tiles_x = (width + kTileW - 1) / kTileW;
    a.tiles_y = (height + kTileH - 1) / kTileH;
    a.cin = cin;
    a.cout = cout;
    a.ci_off = ci_off;
    a.ci_total = ci_total;
    a.dw = dw;
    a.err = d_err;
    static std::once_flag attr;
    cudaError_t ae = cudaSuccess;
    std::call_once(attr, [&] {
        ae = cudaFuncSetAttribute(k_conv3x3_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    if (ae != cudaSuccess) return dn_fail(RL_CUDA_ERROR, "wgrad smem attribute: %s", cudaGetErrorString(ae));
    const long long tiles = (long long)a.tiles_x * a.tiles_y * images;
    const int splits = (int)std::min<long long>(tiles, 32);
    for (int ch = 0; ch < chunks; ch++) {
        WgradArgs b = a;
        b.nb = std::min(4, blocks - ch * 4);
        b.c_base = ch * 256;
        b.stages = b.nb > 2 ? 2 : 3;
        b.splits = splits;
        const int smem = b.stages * (int)(2 * kABytes + b.nb * kABytes) + 2 * b.stages * 8 + 16 + 1024;
        k_conv3x3_wgrad<<<dim3(9, 1, splits), 128, smem, (cudaStream_t)stream>>>(tG, tX, b);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return dn_fail(RL_CUDA_ERROR, "k_conv3x3_wgrad: %s", cudaGetErrorString(e));
    }
    return RL_OK;
}
