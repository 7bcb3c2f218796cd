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

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while its predecessor in the stream is finishing;
// pdl_wait() blocks until the predecessor has completed and its writes are
// visible (at once when launched normally), so everything before it must
// touch no global memory the predecessor may write.  pdl_trigger() lets the
// successor launch as soon as this grid's CTAs are all running.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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
//
// Implicit-GEMM 3x3 convolution over a halo tile.  A tile is 16 rows of 8
// pixels (one half, M = 128: TMEM lane m = pixel (m % 8, m / 8)) or of 16
// pixels (two halves side by side, one accumulator each).  Its input halo,
// 18 rows of halo_w = 8 halves + 2 pixels, is staged once per tile in shared
// memory by TMA as one plane per 8 input channels (one 5-D box of 8 channels
// x halo_w x 18 pixels, zero fill outside the image): pixel-major, 16 bytes
// per pixel, which is the tensor core's unswizzled K-major layout (core
// matrices of 8 pixels x 8 channels, 128 contiguous bytes).  The nine taps
// (and the two halves) are descriptor views of the same halo, started
// (ky * halo_w + kx + 8 h) pixels in, with rows of 8 pixels halo_w x 16 bytes
// apart: a tap reads no global memory.  Weights
// are packed BF16 [9][K/8][ncols][8] in the same layout (core matrices of 8
// output x 8 input channels), resident in shared memory when all nine taps
// fit beside two halo stages, else streamed through a ring of units (a run
// of one tap's 16-channel K-steps).
//
// One tcgen05.mma occupies its issuing thread for about 150 cycles whatever
// its N, so at these channel counts (N = 16-128) a single issuing thread
// keeps the tensor pipe mostly idle, while issuers on different SM
// sub-partitions run concurrently.  Each tile's MMAs (9 taps x K/16) are
// therefore split among `issuers` threads, one per sub-partition (contiguous
// runs with resident weights, streamed units round-robin), each accumulating
// a partial sum in its own TMEM columns; the epilogue adds the partials.
//
// Roles (one CTA per SM walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...):
//   warp 0    tensor memory; the halo loads (HS-stage ring);
//   warp 1    the weight copies (nine bulk copies once, or one per unit);
//   warps 2-5 the epilogue (warp w owns TMEM lanes 32 (w % 4) .. +31), which
//             drains accumulator set i % nbuf while the issuers fill the others;
//   warps 6-9 the MMA issuers (lane 0 of each; warp 6 + k is issuer k);
//   warps 10-13 a second epilogue group when there are two or more
//             accumulator sets: groups 0 and 1 take the even and odd tiles.

constexpr int kTileW = 16, kTileH = 8;    // the weight gradient's pixel tile: 128 pixels
constexpr uint32_t kABytes = 128 * 128;   // 128 pixels x 64 channels x 2 bytes
constexpr int kHTileH = 16;               // the convolution's tile: 16 rows of 8 pixels per half
constexpr int kHaloH = kHTileH + 2;
constexpr int kMaxIssuers = 4;
constexpr int kConvThreads = (10 + kMaxIssuers) * 32;

struct ConvArgs {
    int W, H;              // spatial size (input = output)
    int nkc[2];            // 8-channel planes of each input segment (even: segments padded to 16 channels)
    int nkc_total;
    int ncols;             // MMA N = output channels (multiple of 16, <= 256)
    int tmem_cols;         // power of two >= max(32, ncols): one partial accumulator
    int halves;            // 8-pixel-wide halves per tile (1 or 2): a tile is 16 rows x 8 halves pixels
    int halo_w;            // halo width: 8 halves + 2 pixels
    uint32_t plane_box;    // bytes TMA writes per plane: halo_w x 18 x 16
    uint32_t plane_bytes;  // plane stride: plane_box rounded up to 128
    int issuers;           // MMA-issuing threads (partial accumulators per tile)
    int nbuf;              // accumulator sets (1 to 4): nbuf x halves x tmem_cols <= 512 / issuers
    int pstride;           // TMEM columns between issuers' partials: 512 / issuers
    int hstages;           // halo ring depth
    int resident;          // 1: all nine taps of weights loaded once per CTA
    int bslots;            // streamed weights: ring slots of one unit each
    int kgroup, ngroups;   // K-steps (16 channels) per unit, units per tap
    uint32_t unit_bytes;   // one slot: kgroup x ncols x 32
    uint32_t halo_bytes;   // one halo stage: nkc_total planes
    uint32_t tap_bytes;    // one tap of packed weights: ncols x K x 2
    const bf16* wpk;       // packed weights [9][K/8][ncols][8]
    const float* bias;     // [ncols] or null
    int relu;              // leaky ReLU with negative slope `slope` (0: ReLU)
    float slope;
    // output segments: accumulator columns [c0, c0 + cn) -> tensor out (cstride channels)
    bf16* out[2];
    int out_c0[2], out_cn[2], out_cs[2];
    const bf16* mask[2];   // optional: out *= (mask > 0 ? 1 : slope), same layout as out
    int nout;
    int* err;
};

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* tm, uint64_t* bar, int c0, int c1, int c2,
                                            int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6, %7}], [%2];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
}

// Contiguous global -> shared copy of `bytes` (a multiple of 16, both ends
// 16-byte aligned), completing on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// D[tmem] (+)= A * B^T with both shared-memory descriptors given as 32-bit
// halves: lo = start address (16-byte units, bits 0-13) | leading byte
// offset (bits 16-29); hi = stride byte offset (bits 0-13) | version (bit
// 14); layout type 0 (no swizzle).
__device__ __forceinline__ void umma_lh(uint32_t d, uint32_t alo, uint32_t ahi, uint32_t blo, uint32_t bhi,
                                        uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t.reg .b64 da, db;\n\t"
        "setp.ne.b32 p, %5, 0;\n\t"
        "mov.b64 da, {%1, %2};\n\t"
        "mov.b64 db, {%3, %4};\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], da, db, %6, p;\n\t}" ::"r"(d),
        "r"(alo), "r"(ahi), "r"(blo), "r"(bhi), "r"(accumulate), "r"(idesc)
        : "memory");
}

// 32 lanes x 16 columns of tensor memory, without waiting (tmem_wait_ld).
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Orders uses of registers filled by tmem_ld16_async after tmem_wait_ld.
__device__ __forceinline__ void tmem_regs_ready(uint32_t (&r)[16]) {
    asm volatile(""
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]));
}

// One 16-column chunk of an output row: the summed accumulator values x[16]
// of columns [c, c + 16) -> bias, activation (in place), mask -> BF16 stores
// into the output segments that hold those columns.
__device__ __forceinline__ void conv_store_chunk(const ConvArgs& a, int c, float (&x)[16], long long pix) {
#pragma unroll
    for (int i = 0; i < 16; i++) {
        float t = x[i];
        if (a.bias) t += a.bias[c + i];
        if (a.relu && !(t > 0.0f)) t *= a.slope;
        x[i] = t;
    }
    for (int o = 0; o < a.nout; o++) {
        if (c < a.out_c0[o] || c >= a.out_c0[o] + a.out_cn[o]) continue;
        const long long off = pix * a.out_cs[o] + (c - a.out_c0[o]);
        uint4 m0 = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u), m1 = m0;  // BF16 1.0
        if (a.mask[o]) {
            const uint4* mp = reinterpret_cast<const uint4*>(a.mask[o] + off);
            m0 = mp[0];
            m1 = mp[1];
        }
        const bf16* mb0 = reinterpret_cast<const bf16*>(&m0);
        const bf16* mb1 = reinterpret_cast<const bf16*>(&m1);
        uint4 w0, w1;
        __nv_bfloat162* p0 = reinterpret_cast<__nv_bfloat162*>(&w0);
        __nv_bfloat162* p1 = reinterpret_cast<__nv_bfloat162*>(&w1);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float f0 = __bfloat162float(mb0[2 * i]) > 0.0f ? 1.0f : a.slope;
            const float f1 = __bfloat162float(mb0[2 * i + 1]) > 0.0f ? 1.0f : a.slope;
            const float f2 = __bfloat162float(mb1[2 * i]) > 0.0f ? 1.0f : a.slope;
            const float f3 = __bfloat162float(mb1[2 * i + 1]) > 0.0f ? 1.0f : a.slope;
            p0[i] = __floats2bfloat162_rn(x[2 * i] * f0, x[2 * i + 1] * f1);
            p1[i] = __floats2bfloat162_rn(x[8 + 2 * i] * f2, x[8 + 2 * i + 1] * f3);
        }
        uint4* dst = reinterpret_cast<uint4*>(a.out[o] + off);
        dst[0] = w0;
        dst[1] = w1;
    }
}

// The partial accumulators' 16 columns at `col` of this thread's TMEM lane
// (taddr = lane, column 0 of the tile's first partial; partial k starts k x
// pstride columns further), summed; two partials per load round keep the
// registers in use at 32.
__device__ __forceinline__ void conv_sum_chunk(const ConvArgs& a, uint32_t taddr, int col, float (&x)[16]) {
#pragma unroll
    for (int k0 = 0; k0 < kMaxIssuers; k0 += 2) {
        if (k0 >= a.issuers) break;
        uint32_t r0[16], r1[16];
        tmem_ld16_async(taddr + (uint32_t)(k0 * a.pstride + col), r0);
        if (k0 + 1 < a.issuers) tmem_ld16_async(taddr + (uint32_t)((k0 + 1) * a.pstride + col), r1);
        tmem_wait_ld();
        tmem_regs_ready(r0);
        if (k0 + 1 < a.issuers) tmem_regs_ready(r1);
#pragma unroll
        for (int i = 0; i < 16; i++) {
            float t = __uint_as_float(r0[i]);
            if (k0 + 1 < a.issuers) t += __uint_as_float(r1[i]);
            x[i] = k0 == 0 ? t : x[i] + t;
        }
    }
}

struct TileXY {
    int x0, y0, img;
};
__device__ __forceinline__ TileXY tile_xy(int tile, int tiles_x, int tiles_y, int tile_w) {
    TileXY t;
    t.x0 = (tile % tiles_x) * tile_w;
    t.y0 = ((tile / tiles_x) % tiles_y) * kHTileH;
    t.img = tile / (tiles_x * tiles_y);
    return t;
}

// Epilogue of one tile for this thread's TMEM lane (pixel row % 8, row / 8 of
// each 8-pixel half; half h's accumulator starts h x tmem_cols columns on),
// then the accumulator set's release (`drained`).  When the tile has at most
// 64 columns in all (halves x ncols) and no mask, the finished BF16 values
// are held in registers and the set is released before the global stores, so
// the release (which orders this thread's earlier memory operations) does not
// wait for them; otherwise the row is stored chunk by chunk and released
// after.
template <int kHalves>
__device__ __forceinline__ void conv_epilogue_tile(const ConvArgs& a, uint32_t taddr, const TileXY& tx, int row,
                                                   bool ready, uint64_t* drained) {
    const int cpc = a.ncols / 16;  // 16-column chunks per half
    auto pixel = [&](int h, long long& pix) {
        const int px = tx.x0 + 8 * h + (row & 7), py = tx.y0 + (row >> 3);
        pix = ((long long)tx.img * a.H + py) * a.W + px;
        return ready && px < a.W && py < a.H;
    };
    if (kHalves * a.ncols <= 64 && !a.mask[0] && !a.mask[1]) {
        // finished BF16 values, 16 bytes per 8 columns
        uint4 q[4][2];
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (j < kHalves * cpc) {
                const int h = j / cpc, c = 16 * (j - h * cpc);
                float x[16];
                conv_sum_chunk(a, taddr + (uint32_t)(h * a.tmem_cols), c, x);
                __nv_bfloat162* p0 = reinterpret_cast<__nv_bfloat162*>(&q[j][0]);
                __nv_bfloat162* p1 = reinterpret_cast<__nv_bfloat162*>(&q[j][1]);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    float t = x[i];
                    if (a.bias) t += a.bias[c + i];
                    if (a.relu && !(t > 0.0f)) t *= a.slope;
                    x[i] = t;
                }
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    p0[i] = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
                    p1[i] = __floats2bfloat162_rn(x[8 + 2 * i], x[8 + 2 * i + 1]);
                }
            }
        tc_fence_before();
        mbar_arrive(drained);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (j < kHalves * cpc) {
                const int h = j / cpc, c = 16 * (j - h * cpc);
                long long pix;
                if (!pixel(h, pix)) continue;
                for (int o = 0; o < a.nout; o++) {
                    if (c < a.out_c0[o] || c >= a.out_c0[o] + a.out_cn[o]) continue;
                    uint4* dst = reinterpret_cast<uint4*>(a.out[o] + pix * a.out_cs[o] + (c - a.out_c0[o]));
                    dst[0] = q[j][0];
                    dst[1] = q[j][1];
                }
            }
        return;
    }
    for (int h = 0; h < kHalves; h++) {
        long long pix;
        const bool inb = pixel(h, pix);
        for (int c = 0; c < a.ncols; c += 16) {
            float x[16];
            conv_sum_chunk(a, taddr + (uint32_t)(h * a.tmem_cols), c, x);
            if (inb) conv_store_chunk(a, c, x, pix);
        }
    }
    tc_fence_before();
    mbar_arrive(drained);
}

template <int kHalves>
__global__ void __launch_bounds__(kConvThreads, 1)
    k_conv3x3_h(const __grid_constant__ CUtensorMap tmA0, const __grid_constant__ CUtensorMap tmA1, const ConvArgs a,
                int tiles_x, int tiles_y, int ntiles) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align1024(smem_raw);
    const int HS = a.hstages, BS = a.bslots, NI = a.issuers, NB = a.nbuf;
    uint8_t* sw = smem;                                                        // weights
    uint8_t* sh = smem + (a.resident ? 9 * a.tap_bytes : BS * a.unit_bytes);  // halo stages
    uint64_t* hfull = (uint64_t*)(sh + HS * a.halo_bytes);
    uint64_t* hempty = hfull + HS;
    uint64_t* bfull = hempty + HS;
    uint64_t* bempty = bfull + BS;
    uint64_t* accf = bempty + BS;  // accumulator set k ready for the epilogue (one commit per issuer)
    uint64_t* acce = accf + 4;     // accumulator set k drained (128 epilogue threads)
    uint32_t* tmem_slot = (uint32_t*)(acce + 4);
    const uint32_t tmem_total = 512;  // the issuers' column ranges, 512 / issuers apart
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    pdl_trigger();
    if (threadIdx.x == 0) {
        for (int s = 0; s < HS; s++) {
            mbar_init(hfull + s, 1);
            mbar_init(hempty + s, (uint32_t)NI);
        }
        for (int s = 0; s < BS; s++) {
            mbar_init(bfull + s, 1);
            mbar_init(bempty + s, 1);
        }
        for (int k = 0; k < 4; k++) {
            mbar_init(accf + k, (uint32_t)NI);
            mbar_init(acce + k, 128);
        }
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, tmem_total);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // set-up above overlaps the predecessor's tail; inputs, weights and
    // outputs are touched only after it has completed
    pdl_wait();
    const uint32_t tmem = *tmem_slot;
    const int nk16 = a.nkc_total / 2;
    const int nunits = 9 * a.ngroups;  // a tile's MMA units, in (tap, group) order

    if (warp == 0) {
        if (lane == 0) {
            int i = 0;
            for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, i++) {
                const int s = i % HS;
                if (!mbar_wait(hempty + s, (uint32_t)((i / HS) & 1) ^ 1, a.err, 1)) break;
                const TileXY tx = tile_xy(tile, tiles_x, tiles_y, 8 * kHalves);
                uint8_t* dst = sh + s * a.halo_bytes;
                mbar_expect_tx(hfull + s, (uint32_t)a.nkc_total * a.plane_box);
                for (int c = 0; c < a.nkc[0]; c++)
                    tma_load_5d(dst + c * a.plane_bytes, &tmA0, hfull + s, 0, c, tx.x0 - 1, tx.y0 - 1, tx.img);
                for (int c = 0; c < a.nkc[1]; c++)
                    tma_load_5d(dst + (a.nkc[0] + c) * a.plane_bytes, &tmA1, hfull + s, 0, c, tx.x0 - 1, tx.y0 - 1,
                                tx.img);
            }
            // no copy may still be landing when the CTA exits
            for (int k = i > HS ? i - HS : 0; k < i; k++)
                mbar_wait(hfull + k % HS, (uint32_t)((k / HS) & 1), a.err, 64);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint8_t* wsrc = reinterpret_cast<const uint8_t*>(a.wpk);
            if (a.resident) {
                mbar_expect_tx(bfull, 9 * a.tap_bytes);
                for (int tap = 0; tap < 9; tap++)
                    bulk_load(sw + tap * a.tap_bytes, wsrc + (size_t)tap * a.tap_bytes, a.tap_bytes, bfull);
                mbar_wait(bfull, 0, a.err, 64);
            } else {
                const uint32_t step = (uint32_t)a.ncols * 32;  // one K-step of one tap
                long long g = 0;
                bool ok = true;
                for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x)
                    for (int u = 0; u < nunits; u++, g++) {
                        const int bs = (int)(g % BS);
                        if (!mbar_wait(bempty + bs, (uint32_t)((g / BS) & 1) ^ 1, a.err, 1)) {
                            ok = false;
                            break;
                        }
                        const int tap = u / a.ngroups, k0 = (u - tap * a.ngroups) * a.kgroup;
                        const uint32_t bytes = (uint32_t)(min(nk16, k0 + a.kgroup) - k0) * step;
                        mbar_expect_tx(bfull + bs, bytes);
                        bulk_load(sw + bs * a.unit_bytes, wsrc + (size_t)tap * a.tap_bytes + (size_t)k0 * step, bytes,
                                  bfull + bs);
                    }
                for (long long k = g > BS ? g - BS : 0; k < g; k++)
                    mbar_wait(bfull + k % BS, (uint32_t)((k / BS) & 1), a.err, 64);
            }
        }
    } else if (warp <= 5 || (warp >= 6 + kMaxIssuers && NB >= 2)) {
        // epilogue group 0 (warps 2-5) takes every tile when there is one
        // accumulator set; with two, group 1 (warps 10-13) takes the odd tiles
        const int group = warp <= 5 ? 0 : 1, ngroup = NB >= 2 ? 2 : 1;
        const uint32_t quarter = (uint32_t)(warp & 3);
        const int row = (int)quarter * 32 + lane;
        int i = group;
        for (int tile = blockIdx.x + group * gridDim.x; tile < ntiles; tile += ngroup * gridDim.x, i += ngroup) {
            const int buf = i % NB;
            const bool ready = mbar_wait(accf + buf, (uint32_t)((i / NB) & 1), a.err, 4);
            tc_fence_after();
            const TileXY tx = tile_xy(tile, tiles_x, tiles_y, 8 * kHalves);
            conv_epilogue_tile<kHalves>(a, tmem + (quarter * 32u << 16) + (uint32_t)(buf * kHalves * a.tmem_cols), tx,
                                        row, ready, acce + buf);
            if (!ready) break;
        }
    } else if (warp >= 6 && warp - 6 < NI) {
        if (lane == 0) {
            const int w = warp - 6;
            const uint32_t idesc = idesc_bf16(a.ncols, false, false);
            const uint32_t lbo_b = (uint32_t)a.ncols * 16;
            // descriptor halves (umma_lh): A rows of 8 pixels halo_w x 16 bytes
            // apart, planes plane_bytes apart; B rows of 8 channels 128 bytes
            // apart, K-chunks ncols x 16 bytes apart
            const uint32_t ahi = (uint32_t)a.halo_w | (1u << 14), bhi = (128u >> 4) | (1u << 14);
            const uint32_t alead = (a.plane_bytes >> 4) << 16, blead = (lbo_b >> 4) << 16;
            const uint32_t astep = (2 * a.plane_bytes) >> 4, bstep = (2 * lbo_b) >> 4;
            const uint32_t wbase = smem_u32(sw) >> 4, tapb = a.tap_bytes >> 4;
            const uint32_t hcol = (uint32_t)a.tmem_cols;  // the second half's accumulator, 8 pixels on
            constexpr bool two = kHalves == 2;
            // tap (ky, kx) starts ky * halo_w + kx pixels into the halo; ky = tap / 3 = (11 tap) >> 5
            const int hw = a.halo_w;
            auto toff = [hw](int t) { return (uint32_t)(t + (hw - 3) * ((t * 11) >> 5)); };
            // resident weights: this issuer's run of the tile's 9 x nk16 K-steps
            const int u0 = w * 9 * nk16 / NI, u1 = (w + 1) * 9 * nk16 / NI;
            const int tap0 = u0 / nk16, k0s = u0 - tap0 * nk16;
            bool ok = !a.resident || mbar_wait(bfull, 0, a.err, 2);
            int i = 0;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, i++) {
                const int buf = i % NB, s = i % HS;
                if (!mbar_wait(acce + buf, (uint32_t)((i / NB) & 1) ^ 1, a.err, 128)) break;
                if (!mbar_wait(hfull + s, (uint32_t)((i / HS) & 1), a.err, 2)) ok = false;
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(w * a.pstride + buf * kHalves * a.tmem_cols);
                const uint32_t abase = smem_u32(sh + s * a.halo_bytes) >> 4;
                uint32_t acc = 0;
                if (a.resident) {
                    // a contiguous run of the tile's K-steps in (tap, step)
                    // order, [u0, u1): between two MMAs only two adds, and a
                    // descriptor reload where the run crosses into the next tap
                    // (a thread's instructions between MMAs add to its issue
                    // time)
                    int tap = tap0, k = k0s;
                    uint32_t alo = (abase + toff(tap) + (uint32_t)k * astep) | alead;
                    uint32_t blo = (wbase + (uint32_t)tap * tapb + (uint32_t)k * bstep) | blead;
                    for (int u = u0; u < u1; u++) {
                        umma_lh(d, alo, ahi, blo, bhi, idesc, acc);
                        if (two) umma_lh(d + hcol, alo + 8, ahi, blo, bhi, idesc, acc);
                        acc = 1;
                        if (++k == nk16) {
                            k = 0;
                            tap++;
                            alo = (abase + toff(tap)) | alead;
                            blo = (wbase + (uint32_t)tap * tapb) | blead;
                        } else {
                            alo += astep;
                            blo += bstep;
                        }
                    }
                } else {
                    // streamed units u = w, w + NI, ...: each waits for its
                    // ring slot; (tap, group) as running counters
                    int tap = 0, grp = w;
                    while (grp >= a.ngroups) {
                        grp -= a.ngroups;
                        tap++;
                    }
                    uint32_t g = (uint32_t)i * (uint32_t)nunits + (uint32_t)w;  // ring position
                    for (int u = w; u < nunits && ok; u += NI) {
                        const int kb = grp * a.kgroup, ke = min(nk16, kb + a.kgroup);
                        const int bs = (int)(g % (uint32_t)BS);
                        if (!mbar_wait(bfull + bs, (g / (uint32_t)BS) & 1, a.err, 2)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        uint32_t blo = (smem_u32(sw + bs * a.unit_bytes) >> 4) | blead;
                        uint32_t alo = (abase + toff(tap) + (uint32_t)kb * astep) | alead;
                        for (int k = kb; k < ke; k++) {
                            umma_lh(d, alo, ahi, blo, bhi, idesc, acc);
                            if (two) umma_lh(d + hcol, alo + 8, ahi, blo, bhi, idesc, acc);
                            acc = 1;
                            alo += astep;
                            blo += bstep;
                        }
                        umma_commit(bempty + bs);
                        grp += NI;
                        while (grp >= a.ngroups) {
                            grp -= a.ngroups;
                            tap++;
                        }
                        g += (uint32_t)NI;
                    }
                }
                umma_commit(hempty + s);
                umma_commit(accf + buf);  // also after a timeout: the epilogue then waits for the issued MMAs
            }
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, tmem_total);
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

// Launch with programmatic stream serialisation (see pdl_wait).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
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

// The convolution's halo planes: NHWC BF16 [n][h][w][c] (c a multiple of 8)
// seen as [n][h][w][c / 8][8]; a box is one plane of 8 channels x halo_w x
// 18 pixels, unswizzled (16 bytes per pixel), zero fill outside.
int halo_map(CUtensorMap* tm, const void* base, int c, int w, int h, int n, int halo_w) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return dn_fail(RL_CUDA_ERROR, "cuTensorMapEncodeTiled unavailable");
    if (c <= 0 || c % 8 || ((uintptr_t)base & 15)) return dn_fail(RL_INVALID_CALL, "activation layout: %d channels", c);
    cuuint64_t dims[5] = {8, (cuuint64_t)(c / 8), (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    cuuint64_t strides[4] = {16, (cuuint64_t)c * 2, (cuuint64_t)c * 2 * w, (cuuint64_t)c * 2 * w * h};
    cuuint32_t box[5] = {8, 1, (cuuint32_t)halo_w, kHaloH, 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return dn_fail(RL_CUDA_ERROR, "tensor map (halo) error %d", (int)r);
    return RL_OK;
}

int pow2_cols(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256; }

}  // namespace

// ---------------------------------------------------------------- C ABI

// One 3x3 "same" convolution over NHWC BF16 tensors (see the header).
extern "C" int rl_dn_conv3x3(const void* in0, int c0, const void* in1, int c1, int width, int height, int images,
                             const void* weights, int ncols, const float* bias, int relu, float slope, void* out0,
                             int out0_c0,
                             int out0_cn, int out0_cs, const void* mask0, void* out1, int out1_c0, int out1_cn,
                             int out1_cs, const void* mask1, int* d_err, void* stream) {
    if (!in0 || !weights || !out0 || width <= 0 || height <= 0 || images <= 0 || c0 <= 0 || (in1 && c1 <= 0))
        return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: bad arguments");
    if (ncols < 16 || ncols > 256 || ncols % 16) return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: ncols %d", ncols);
    if ((uintptr_t)weights & 15) return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: weights not 16-byte aligned");
    const int nout = out1 ? 2 : 1;
    const int oc0[2] = {out0_c0, out1_c0}, ocn[2] = {out0_cn, out1_cn}, ocs[2] = {out0_cs, out1_cs};
    for (int o = 0; o < nout; o++)
        if (ocn[o] % 16 || ocs[o] % 16 || oc0[o] % 16 || ocn[o] > ocs[o] || oc0[o] + ocn[o] > ncols)
            return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: output segment %d", o);
    ConvArgs a;
    memset(&a, 0, sizeof a);
    a.W = width;
    a.H = height;
    a.nkc[0] = (c0 + 15) / 16 * 2;
    a.nkc[1] = in1 ? (c1 + 15) / 16 * 2 : 0;
    a.nkc_total = a.nkc[0] + a.nkc[1];
    a.ncols = ncols;
    a.tmem_cols = pow2_cols(ncols);
    a.tap_bytes = (uint32_t)a.nkc_total * (uint32_t)ncols * 16;
    a.wpk = (const bf16*)weights;
    // partial accumulators: four issuers, each in its own 128-column quarter
    // of tensor memory; two issuers 256 columns apart for 256 columns
    a.issuers = a.tmem_cols <= 128 ? 4 : 2;
    a.pstride = 512 / a.issuers;
    // shared memory: the nine taps of weights resident beside at least two
    // halo stages when they fit (units of one K-step, dealt to the issuers);
    // else two or three halo stages and a ring of at least four weight
    // units, each the widest run of a tap's K-steps that allows it.  Tiles
    // are 16 x 16 pixels (two halves: twice the MMAs per barrier wait and
    // commit) for layers of at most 32 input channels whose weights are
    // resident and whose two halves still leave each issuer two accumulator
    // sets (measured at 1024^2: 16 -> 32 channels 69 -> 63 us, 32 -> 3
    // channels 70 -> 54 us; with more input channels, or with one accumulator
    // set, the wider tile was slower); otherwise 16 x 8.
    const long long budget = 225 * 1024;
    const long long tap = a.tap_bytes, step = (long long)ncols * 32;
    const int nk16 = a.nkc_total / 2;
    auto plane_of = [](int halo_w) { return (uint32_t)((halo_w * kHaloH * 16 + 127) / 128 * 128); };
    a.halves = (nk16 <= 2 && 4 * a.tmem_cols <= a.pstride && 9 * tap + 2LL * a.nkc_total * plane_of(18) <= budget)
                   ? 2
                   : 1;
    a.halo_w = 8 * a.halves + 2;
    a.plane_box = (uint32_t)(a.halo_w * kHaloH * 16);
    a.plane_bytes = plane_of(a.halo_w);
    a.halo_bytes = (uint32_t)a.nkc_total * a.plane_bytes;
    a.nbuf = std::min(4, a.pstride / (a.halves * a.tmem_cols));
    const long long halo = a.halo_bytes;
    CUtensorMap tA0, tA1;
    if (int rc = halo_map(&tA0, in0, c0, width, height, images, a.halo_w)) return rc;
    if (int rc = halo_map(&tA1, in1 ? in1 : in0, in1 ? c1 : c0, width, height, images, a.halo_w)) return rc;
    if (9 * tap + 2 * halo <= budget) {
        a.resident = 1;
        a.bslots = 1;
        a.kgroup = 1;
        a.ngroups = nk16;
        a.hstages = (int)std::min<long long>(8, (budget - 9 * tap) / halo);
    } else {
        a.resident = 0;
        // with at most four tiles per SM there is little halo load to hide:
        // one halo stage leaves room for twice the weight bytes in flight,
        // which is what bounds these layers (measured on the 128 + 96 -> 96
        // layer at 256^2: 77 -> 52 us)
        const long long tiles = (long long)((width + 7) / 8) * ((height + 15) / 16) * images;
        const bool few = tiles <= 4LL * 148;
        a.hstages = few ? 1 : (budget - 3 * halo >= 3 * tap ? 3 : 2);
        const long long rem = budget - a.hstages * halo;
        a.kgroup = nk16;
        while (a.kgroup > 1 && rem / (a.kgroup * step) < 4) a.kgroup = (a.kgroup + 1) / 2;
        a.ngroups = (nk16 + a.kgroup - 1) / a.kgroup;
        a.bslots = (int)std::min<long long>(few ? 16 : 8, rem / (a.kgroup * step));
        if (a.bslots < 2)
            return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: %d input and %d output channels exceed shared memory",
                           c0 + (in1 ? c1 : 0), ncols);
    }
    a.unit_bytes = (uint32_t)(a.kgroup * step);
    a.bias = bias;
    a.relu = relu;
    a.slope = slope;
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
    // one CTA per SM: at least 116 KB of shared memory each, so two CTAs
    // never contend for tensor memory
    const long long need = (a.resident ? 9 * tap : (long long)a.bslots * a.unit_bytes) + (long long)a.hstages * halo +
                           (2LL * a.hstages + 2LL * a.bslots + 8) * 8 + 16 + 1024;
    const int smem = (int)std::max<long long>(need, 116 * 1024);
    static int sms = 0;
    static std::once_flag attr;
    cudaError_t ae = cudaSuccess;
    std::call_once(attr, [&] {
        ae = cudaFuncSetAttribute(k_conv3x3_h<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (ae == cudaSuccess)
            ae = cudaFuncSetAttribute(k_conv3x3_h<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        int dev = 0;
        if (ae == cudaSuccess) ae = cudaGetDevice(&dev);
        if (ae == cudaSuccess) ae = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    });
    if (ae != cudaSuccess) return dn_fail(RL_CUDA_ERROR, "conv set-up: %s", cudaGetErrorString(ae));
    const int tile_w = 8 * a.halves;
    const int tiles_x = (width + tile_w - 1) / tile_w, tiles_y = (height + kHTileH - 1) / kHTileH;
    const long long ntiles = (long long)tiles_x * tiles_y * images;
    if (ntiles > INT32_MAX) return dn_fail(RL_INVALID_CALL, "rl_dn_conv3x3: too many tiles");
    const int grid = (int)std::min<long long>(ntiles, std::max(sms, 1));
    cudaError_t e = launch_pdl(a.halves == 2 ? k_conv3x3_h<2> : k_conv3x3_h<1>, dim3(grid), dim3(kConvThreads),
                               (size_t)smem, (cudaStream_t)stream, tA0, tA1, a, tiles_x, tiles_y, (int)ntiles);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return dn_fail(RL_CUDA_ERROR, "k_conv3x3_h: %s", cudaGetErrorString(e));
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

// ================================================================ network
//
// (relu = leaky ReLU, negative slope 0.1)
//   x (16: log1p noisy rgb, normal, albedo, valid)
//   e0 = relu(c0(x))            32  full       p0 = pool(e0)
//   e1 = relu(c1(p0))           64  1/2        p1 = pool(e1)
//   e2 = relu(c2(p1))           96  1/4        p2 = pool(e2)
//   e3 = relu(c3(p2))          128  1/8
//   d2 = relu(c4(up(e3), e2))   96  1/4
//   d1 = relu(c5(up(d2), e1))   64  1/2
//   d0 = relu(c6(up(d1), e0))   32  full
//   y  = c7(d0)                  3  full;   prediction = y + log1p(noisy)
//
// Loss: mean |prediction - log1p(clean)| over valid texels (L1 in log space).

namespace {

constexpr int kFeat = 16;
constexpr float kLeak = 0.1f;  // leaky ReLU slope: no unit can die

__device__ __forceinline__ float bf(bf16 v) { return __bfloat162float(v); }

// The resampling kernels move 8 channels (16 bytes) per thread: C is a
// multiple of 8, and each thread decodes its pixel once.
union Pack8 {
    uint4 u;
    bf16 h[8];
};

// 2x2 average pooling; odd edges average the children that exist.
__global__ void k_dn_pool(const bf16* in, bf16* out, int C, int W, int H, int N) {
    pdl_trigger();
    pdl_wait();
    // one thread per output pixel and 8-channel group; 32-bit index arithmetic
    // (the host launches this only below 2^31 elements)
    const int W2 = (W + 1) / 2, H2 = (H + 1) / 2, G = C / 8;
    const unsigned total = (unsigned)N * H2 * W2 * G;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned g = i % G, p = i / G;
        const unsigned x = p % W2, q = p / W2;
        const unsigned y = q % H2, n = q / H2;
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int cnt = 0;
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                const unsigned xx = 2 * x + dx, yy = 2 * y + dy;
                if (xx < (unsigned)W && yy < (unsigned)H) {
                    Pack8 v;
                    v.u = reinterpret_cast<const uint4*>(in + (((size_t)n * H + yy) * W + xx) * C)[g];
#pragma unroll
                    for (int k = 0; k < 8; k++) s[k] += bf(v.h[k]);
                    cnt++;
                }
            }
        Pack8 o;
#pragma unroll
        for (int k = 0; k < 8; k++) o.h[k] = __float2bfloat16(s[k] / cnt);
        reinterpret_cast<uint4*>(out)[i] = o.u;
    }
}

__global__ void k_dn_pool_bwd(const bf16* gout, const bf16* mask, bf16* gin, int C, int W, int H, int N, float slope) {
    const int W2 = (W + 1) / 2, H2 = (H + 1) / 2, G = C / 8;
    const long long total = (long long)N * H * W * G;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        int g = (int)(i % G);
        long long p = i / G;
        int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((long long)W * H));
        int x2 = x / 2, y2 = y / 2;
        float inv = 1.0f / ((2 * x2 + 1 < W ? 2 : 1) * (2 * y2 + 1 < H ? 2 : 1));
        Pack8 go, m, gi;
        go.u = reinterpret_cast<const uint4*>(gout + (((long long)n * H2 + y2) * W2 + x2) * C)[g];
        m.u = reinterpret_cast<const uint4*>(mask)[i];
        gi.u = reinterpret_cast<const uint4*>(gin)[i];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            float v = bf(go.h[k]) * inv;
            if (!(bf(m.h[k]) > 0.f)) v *= slope;
            gi.h[k] = __float2bfloat16(bf(gi.h[k]) + v);
        }
        reinterpret_cast<uint4*>(gin)[i] = gi.u;
    }
}

// Nearest 2x upsampling to W x H.
__global__ void k_dn_up(const bf16* in, bf16* out, int C, int W, int H, int N) {
    pdl_trigger();
    pdl_wait();
    // one thread per source pixel and 8-channel group: one 16-byte read, up
    // to four 16-byte writes; 32-bit index arithmetic (launched only below
    // 2^31 source elements)
    const int W2 = (W + 1) / 2, H2 = (H + 1) / 2, G = C / 8;
    const unsigned total = (unsigned)N * H2 * W2 * G;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const unsigned g = i % G, p = i / G;
        const unsigned x = p % W2, q = p / W2;
        const unsigned y = q % H2, n = q / H2;
        const uint4 v = reinterpret_cast<const uint4*>(in)[i];
        for (int dy = 0; dy < 2; dy++) {
            const unsigned yy = 2 * y + dy;
            if (yy >= (unsigned)H) break;
            uint4* row = reinterpret_cast<uint4*>(out + (((size_t)n * H + yy) * W + 2 * x) * C) + g;
            row[0] = v;
            if (2 * x + 1 < (unsigned)W) row[G] = v;
        }
    }
}

__global__ void k_dn_up_bwd(const bf16* gout, bf16* gin, int C, int W, int H, int N) {
    const int W2 = (W + 1) / 2, H2 = (H + 1) / 2, G = C / 8;
    const long long total = (long long)N * H2 * W2 * G;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        int g = (int)(i % G);
        long long p = i / G;
        int x = (int)(p % W2), y = (int)((p / W2) % H2), n = (int)(p / ((long long)W2 * H2));
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                int xx = 2 * x + dx, yy = 2 * y + dy;
                if (xx < W && yy < H) {
                    Pack8 v;
                    v.u = reinterpret_cast<const uint4*>(gout + (((long long)n * H + yy) * W + xx) * C)[g];
#pragma unroll
                    for (int k = 0; k < 8; k++) s[k] += bf(v.h[k]);
                }
            }
        Pack8 o;
#pragma unroll
        for (int k = 0; k < 8; k++) o.h[k] = __float2bfloat16(s[k]);
        reinterpret_cast<uint4*>(gin)[i] = o.u;
    }
}

// db[c] += sum over pixels of g[p][c], c < cout (blockDim.x = channel stride).
__global__ void k_dn_bias_grad(const bf16* g, int cs, int cout, long long P, float* db) {
    const int c = threadIdx.x;
    float s = 0.f;
    for (long long p = blockIdx.x; p < P; p += gridDim.x) s += bf(g[p * cs + c]);
    if (c < cout) atomicAdd(db + c, s);
}

// L1 loss on log1p colours: pred = y[:3] + x[:3]; gy = sign(pred - t) * valid * scale.
__global__ void k_dn_loss(const bf16* y, const bf16* x, const float4* t, long long P, float scale, bf16* gy,
                          float* loss) {
    float acc = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        float4 tt = t[p];
        float tv[3] = {tt.x, tt.y, tt.z};
        for (int c = 0; c < kFeat; c++) {
            float g = 0.f;
            if (c < 3 && tt.w > 0.f) {
                float d = bf(y[p * kFeat + c]) + bf(x[p * kFeat + c]) - tv[c];
                acc += fabsf(d);
                g = (d > 0.f ? 1.f : d < 0.f ? -1.f : 0.f) * scale;
            }
            gy[p * kFeat + c] = __float2bfloat16(g);
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, acc * scale);
}

__global__ void k_dn_adam(float* p, float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                          float bc1, float bc2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.f - b1) * gi;
        float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        g[i] = 0.f;
    }
}

// Master weights [cout][9][kpad] (each input segment's columns from a
// multiple of 64) -> the convolution's packed BF16 operands, [9][K/8][rows][8]:
//   forward:       rows = ncols, K = pad16(seg0) + pad16(seg1); K column kk is
//                  master column kk (segment 0) or pad64(seg0) + kk - pad16(seg0);
//   data gradient: rows = kpad (the forward's input columns), K = ncols (the
//                  forward's output channels), taps flipped.
__global__ void k_dn_pack(const float* w, int cout, int ncols, int seg0, int seg1, int kpad, bf16* wp, bf16* wt) {
    const int k0 = (seg0 + 15) / 16 * 16, K = k0 + (seg1 + 15) / 16 * 16, s1 = (seg0 + 63) / 64 * 64;
    const long long nf = 9LL * K * ncols, nt = 9LL * ncols * kpad;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nf + nt; i += (long long)gridDim.x * blockDim.x) {
        if (i < nf) {
            const int e = (int)(i & 7);
            const long long q = i >> 3;
            const int r = (int)(q % ncols), kc = (int)((q / ncols) % (K / 8)), t = (int)(q / ((long long)ncols * (K / 8)));
            const int kk = kc * 8 + e;
            const int col = kk < k0 ? (kk < seg0 ? kk : -1) : (kk - k0 < seg1 ? s1 + kk - k0 : -1);
            wp[i] = __float2bfloat16(r < cout && col >= 0 ? w[((long long)r * 9 + t) * kpad + col] : 0.f);
        } else {
            const long long j = i - nf;
            const int e = (int)(j & 7);
            const long long q = j >> 3;
            const int r = (int)(q % kpad), kc = (int)((q / kpad) % (ncols / 8)), t = (int)(q / ((long long)kpad * (ncols / 8)));
            const int co = kc * 8 + e;
            wt[j] = __float2bfloat16(co < cout ? w[((long long)co * 9 + (8 - t)) * kpad + r] : 0.f);
        }
    }
}

// Face::colorAt at each valid lumel's texel centre (the surface albedo).
__device__ __forceinline__ bool uv_bary(float2 a, float2 b, float2 c, float2 uv, float& bu, float& bv) {
    float v0x = c.x - a.x, v0y = c.y - a.y, v1x = b.x - a.x, v1y = b.y - a.y, v2x = uv.x - a.x, v2y = uv.y - a.y;
    float d00 = v0x * v0x + v0y * v0y, d01 = v0x * v1x + v0y * v1y, d02 = v0x * v2x + v0y * v2y;
    float d11 = v1x * v1x + v1y * v1y, d12 = v1x * v2x + v1y * v2y;
    float inv = 1.0f / (d00 * d11 - d01 * d01);
    bu = (d11 * d02 - d01 * d12) * inv;
    bv = (d00 * d12 - d01 * d02) * inv;
    return true;
}

// Features of one lightmap: [h][w][16] = log1p(max(colour, 0)), normal,
// albedo, valid, zeros.
__global__ void k_dn_features(rl::DevScene s, rl::DevMap m, bf16* x) {
    const long long n = (long long)m.width * m.height;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float f[kFeat];
        for (int c = 0; c < kFeat; c++) f[c] = 0.f;
        if (m.flags[i] & 1) {
            for (int c = 0; c < 3; c++) {
                f[c] = log1pf(fmaxf(m.color[3 * i + c], 0.f));
                f[3 + c] = m.normal[3 * i + c];
            }
            int mesh = m.mesh[i], face = m.face[i];
            float4 alb = make_float4(1.f, 1.f, 1.f, 1.f);
            if (mesh >= 0 && mesh < s.nmeshes) {
                int tri = s.mesh_first_tri[mesh] + face;
                int4 fv = s.tri_vidx[tri];
                float2 a = make_float2(s.uv1[2 * fv.x], s.uv1[2 * fv.x + 1]);
                float2 b = make_float2(s.uv1[2 * fv.y], s.uv1[2 * fv.y + 1]);
                float2 c = make_float2(s.uv1[2 * fv.z], s.uv1[2 * fv.z + 1]);
                int u = (int)(i % m.width), v = (int)(i / m.width);
                float2 uv = make_float2((u + 0.5f) / (float)m.width, (v + 0.5f) / (float)m.height);
                float bu, bv;
                uv_bary(a, b, c, uv, bu, bv);
                alb = rl::face_color(s, fv, bu, bv);
            }
            f[6] = alb.x;
            f[7] = alb.y;
            f[8] = alb.z;
            f[9] = 1.f;
        }
        for (int c = 0; c < kFeat; c++) x[i * kFeat + c] = __float2bfloat16(f[c]);
    }
}

// Targets of one lightmap: (log1p(max(colour, 0)), valid).
__global__ void k_dn_targets(rl::DevMap m, float4* t) {
    const long long n = (long long)m.width * m.height;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        bool v = m.flags[i] & 1;
        t[i] = v ? make_float4(log1pf(fmaxf(m.color[3 * i], 0.f)), log1pf(fmaxf(m.color[3 * i + 1], 0.f)),
                               log1pf(fmaxf(m.color[3 * i + 2], 0.f)), 1.f)
                 : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// colour = base + expm1(prediction) on valid lumels (base may be null = 0).
__global__ void k_dn_apply(const bf16* y, const bf16* x, rl::DevMap m, const float* base) {
    const long long n = (long long)m.width * m.height;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (!(m.flags[i] & 1)) continue;
        for (int c = 0; c < 3; c++) {
            float v = expm1f(bf(y[i * kFeat + c]) + bf(x[i * kFeat + c]));
            m.color[3 * i + c] = (base ? base[3 * i + c] : 0.f) + fmaxf(v, 0.f);
        }
    }
}

int grid_of(long long n, int block) {
    long long g = (n + block - 1) / block;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 16));
}

struct Conv {
    int cout, ncols, segs[2], kpad, copad;
    float *w, *b, *gw, *gb, *mw, *vw, *mb, *vb;
    bf16 *wp, *wt;
    float* bias;  // [ncols]
    long long nw() const { return (long long)cout * 9 * kpad; }
};

struct Level {
    int w, h;
};

}  // namespace

struct rl_denoiser {
    Conv conv[8];
    float* params = nullptr;  // one block: every layer's w, b, gw, gb, mw, vw, mb, vb, bias
    bf16* packed = nullptr;
    long long nparam = 0;      // weights + biases
    int* d_err = nullptr;
    long long step = 0;
    // activation / gradient buffers for the current shape
    int bn = 0, bh = 0, bw = 0, btrain = 0;
    bf16* act = nullptr;
    size_t act_bytes = 0;
    bf16 *x, *e0, *p0, *e1, *p1, *e2, *p2, *e3, *u2, *d2, *u1, *d1, *u0, *d0, *y;
    bf16 *gy, *gd0, *gu0, *ge0, *gd1, *gu1, *ge1, *gd2, *gu2, *ge2, *ge3, *gp2, *gp1, *gp0;
    float4* tgt = nullptr;
    ~rl_denoiser() {
        cudaFree(params);
        cudaFree(packed);
        cudaFree(d_err);
        cudaFree(act);
    }
};

namespace {

const int kCout[8] = {32, 64, 96, 128, 96, 64, 32, 3};
const int kSeg0[8] = {16, 32, 64, 96, 128, 96, 64, 32};
const int kSeg1[8] = {0, 0, 0, 0, 96, 64, 32, 0};

int pad64(int c) { return (c + 63) / 64 * 64; }
int pad16(int c) { return (c + 15) / 16 * 16; }

// Deterministic He-uniform initialisation from a 64-bit seed.
void init_weights(std::vector<float>& w, int fan_in, uint64_t seed) {
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
    float lim = sqrtf(6.0f / (float)fan_in);
    for (float& v : w) {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        v = ((float)((s >> 11) & 0xFFFFFF) / 16777216.0f * 2.0f - 1.0f) * lim;
    }
}

// Carve the activation (and, for training, gradient) buffers of an n x h x
// w batch from one allocation that only grows.  Every buffer is fully
// written before it is read, so reuse needs no clearing.
int alloc_shapes(rl_denoiser* d, int n, int h, int w, bool train, cudaStream_t st) {
    if (d->bn == n && d->bh == h && d->bw == w && (d->btrain || !train) && d->act) return RL_OK;
    (void)st;
    Level L[4];
    L[0] = {w, h};
    for (int k = 1; k < 4; k++) L[k] = {(L[k - 1].w + 1) / 2, (L[k - 1].h + 1) / 2};
    auto sz = [&](int lvl, int c) { return (size_t)n * L[lvl].w * L[lvl].h * c * sizeof(bf16); };
    struct Buf { bf16** p; int lvl, c; bool grad; };
    Buf bufs[] = {{&d->x, 0, 16, 0},   {&d->e0, 0, 32, 0},  {&d->p0, 1, 32, 0},  {&d->e1, 1, 64, 0},
                  {&d->p1, 2, 64, 0},  {&d->e2, 2, 96, 0},  {&d->p2, 3, 96, 0},  {&d->e3, 3, 128, 0},
                  {&d->u2, 2, 128, 0}, {&d->d2, 2, 96, 0},  {&d->u1, 1, 96, 0},  {&d->d1, 1, 64, 0},
                  {&d->u0, 0, 64, 0},  {&d->d0, 0, 32, 0},  {&d->y, 0, 16, 0},   {&d->gy, 0, 16, 1},
                  {&d->gd0, 0, 32, 1}, {&d->gu0, 0, 64, 1}, {&d->ge0, 0, 32, 1}, {&d->gd1, 1, 64, 1},
                  {&d->gu1, 1, 96, 1}, {&d->ge1, 1, 64, 1}, {&d->gd2, 2, 96, 1}, {&d->gu2, 2, 128, 1},
                  {&d->ge2, 2, 96, 1}, {&d->ge3, 3, 128, 1}, {&d->gp2, 3, 96, 1}, {&d->gp1, 2, 64, 1},
                  {&d->gp0, 1, 32, 1}};
    size_t total = 0;
    for (const Buf& b : bufs)
        if (train || !b.grad) total += (sz(b.lvl, b.c) + 255) / 256 * 256;
    size_t tbytes = train ? (size_t)n * h * w * sizeof(float4) : 0;
    total += tbytes + 256;
    if (total > d->act_bytes) {
        DN_CK(cudaDeviceSynchronize());
        cudaFree(d->act);
        d->act = nullptr;
        d->act_bytes = 0;
        DN_CK(cudaMalloc(&d->act, total));
        d->act_bytes = total;
    }
    char* p = (char*)d->act;
    for (const Buf& b : bufs) {
        if (!train && b.grad) {
            *b.p = nullptr;
            continue;
        }
        *b.p = (bf16*)p;
        p += (sz(b.lvl, b.c) + 255) / 256 * 256;
    }
    d->tgt = train ? (float4*)p : nullptr;
    d->bn = n;
    d->bh = h;
    d->bw = w;
    d->btrain = train;
    return RL_OK;
}

int conv_fwd(rl_denoiser* d, int l, const bf16* in0, const bf16* in1, int w, int h, int n, bf16* out, bool relu,
             cudaStream_t st) {
    Conv& c = d->conv[l];
    return rl_dn_conv3x3(in0, c.segs[0], in1, c.segs[1], w, h, n, c.wp, c.ncols, c.bias, relu ? 1 : 0, kLeak, out, 0,
                         c.ncols, c.ncols, nullptr, nullptr, 0, 0, 0, nullptr, d->d_err, st);
}

// Data gradient of layer l: gout (ncols stored) -> g0 (segment 0) / g1,
// each scaled by the leaky-ReLU derivative of the matching forward input
// (the activation keeps the sign; upsampled inputs carry their source's).
int conv_dgrad(rl_denoiser* d, int l, const bf16* gout, int w, int h, int n, bf16* g0, const bf16* m0, bf16* g1,
               const bf16* m1, cudaStream_t st) {
    Conv& c = d->conv[l];
    return rl_dn_conv3x3(gout, c.ncols, nullptr, 0, w, h, n, c.wt, c.kpad, nullptr, 0, kLeak, g0, 0, c.segs[0],
                         c.segs[0], m0, g1, pad64(c.segs[0]), g1 ? c.segs[1] : 0, g1 ? c.segs[1] : 0, m1, d->d_err, st);
}

int conv_wgrad(rl_denoiser* d, int l, const bf16* gout, const bf16* in0, const bf16* in1, int w, int h, int n,
               cudaStream_t st) {
    Conv& c = d->conv[l];
    if (int rc = rl_dn_conv3x3_wgrad(gout, c.cout, c.ncols, in0, c.segs[0], c.segs[0], w, h, n, c.gw, 0, c.kpad,
                                     d->d_err, st))
        return rc;
    if (in1)
        if (int rc = rl_dn_conv3x3_wgrad(gout, c.cout, c.ncols, in1, c.segs[1], c.segs[1], w, h, n, c.gw,
                                         pad64(c.segs[0]), c.kpad, d->d_err, st))
            return rc;
    const long long P = (long long)n * w * h;
    k_dn_bias_grad<<<(int)std::min<long long>(P, 2048), c.ncols, 0, st>>>(gout, c.ncols, c.cout, P, c.gb);
    return RL_OK;
}

int forward(rl_denoiser* d, int n, int h, int w, cudaStream_t st) {
    // the resampling kernels index 16-byte elements in 32 bits
    if ((long long)n * h * w * 16 > INT32_MAX) return dn_fail(RL_INVALID_CALL, "denoiser: %d x %d x %d too large", n, h, w);
    Level L[4];
    L[0] = {w, h};
    for (int k = 1; k < 4; k++) L[k] = {(L[k - 1].w + 1) / 2, (L[k - 1].h + 1) / 2};
    auto pool = [&](const bf16* in, bf16* out, int c, int lvl) {
        long long tot = (long long)n * L[lvl + 1].w * L[lvl + 1].h * (c / 8);
        launch_pdl(k_dn_pool, dim3(grid_of(tot, 256)), dim3(256), 0, st, in, out, c, L[lvl].w, L[lvl].h, n);
    };
    auto up = [&](const bf16* in, bf16* out, int c, int lvl) {
        long long tot = (long long)n * L[lvl + 1].w * L[lvl + 1].h * (c / 8);
        launch_pdl(k_dn_up, dim3(grid_of(tot, 256)), dim3(256), 0, st, in, out, c, L[lvl].w, L[lvl].h, n);
    };
    int rc;
    if ((rc = conv_fwd(d, 0, d->x, nullptr, L[0].w, L[0].h, n, d->e0, true, st))) return rc;
    pool(d->e0, d->p0, 32, 0);
    if ((rc = conv_fwd(d, 1, d->p0, nullptr, L[1].w, L[1].h, n, d->e1, true, st))) return rc;
    pool(d->e1, d->p1, 64, 1);
    if ((rc = conv_fwd(d, 2, d->p1, nullptr, L[2].w, L[2].h, n, d->e2, true, st))) return rc;
    pool(d->e2, d->p2, 96, 2);
    if ((rc = conv_fwd(d, 3, d->p2, nullptr, L[3].w, L[3].h, n, d->e3, true, st))) return rc;
    up(d->e3, d->u2, 128, 2);
    if ((rc = conv_fwd(d, 4, d->u2, d->e2, L[2].w, L[2].h, n, d->d2, true, st))) return rc;
    up(d->d2, d->u1, 96, 1);
    if ((rc = conv_fwd(d, 5, d->u1, d->e1, L[1].w, L[1].h, n, d->d1, true, st))) return rc;
    up(d->d1, d->u0, 64, 0);
    if ((rc = conv_fwd(d, 6, d->u0, d->e0, L[0].w, L[0].h, n, d->d0, true, st))) return rc;
    if ((rc = conv_fwd(d, 7, d->d0, nullptr, L[0].w, L[0].h, n, d->y, false, st))) return rc;
    DN_CK(cudaGetLastError());
    return RL_OK;
}

int backward(rl_denoiser* d, int n, int h, int w, cudaStream_t st) {
    Level L[4];
    L[0] = {w, h};
    for (int k = 1; k < 4; k++) L[k] = {(L[k - 1].w + 1) / 2, (L[k - 1].h + 1) / 2};
    auto up_bwd = [&](const bf16* gfine, bf16* gcoarse, int c, int lvl) {
        long long tot = (long long)n * L[lvl + 1].w * L[lvl + 1].h * (c / 8);
        k_dn_up_bwd<<<grid_of(tot, 256), 256, 0, st>>>(gfine, gcoarse, c, L[lvl].w, L[lvl].h, n);
    };
    auto pool_bwd = [&](const bf16* gcoarse, const bf16* mask, bf16* gfine, int c, int lvl) {
        long long tot = (long long)n * L[lvl].w * L[lvl].h * (c / 8);
        k_dn_pool_bwd<<<grid_of(tot, 256), 256, 0, st>>>(gcoarse, mask, gfine, c, L[lvl].w, L[lvl].h, n, kLeak);
    };
    int rc;
    const int W0 = L[0].w, H0 = L[0].h;
    // output layer
    if ((rc = conv_wgrad(d, 7, d->gy, d->d0, nullptr, W0, H0, n, st))) return rc;
    if ((rc = conv_dgrad(d, 7, d->gy, W0, H0, n, d->gd0, d->d0, nullptr, nullptr, st))) return rc;
    // level 0 decoder: d0 = c6(u0, e0)
    if ((rc = conv_wgrad(d, 6, d->gd0, d->u0, d->e0, W0, H0, n, st))) return rc;
    if ((rc = conv_dgrad(d, 6, d->gd0, W0, H0, n, d->gu0, d->u0, d->ge0, d->e0, st))) return rc;
    up_bwd(d->gu0, d->gd1, 64, 0);
    // level 1 decoder: d1 = c5(u1, e1)
    if ((rc = conv_wgrad(d, 5, d->gd1, d->u1, d->e1, L[1].w, L[1].h, n, st))) return rc;
    if ((rc = conv_dgrad(d, 5, d->gd1, L[1].w, L[1].h, n, d->gu1, d->u1, d->ge1, d->e1, st))) return rc;
    up_bwd(d->gu1, d->gd2, 96, 1);
    // level 2 decoder: d2 = c4(u2, e2)
    if ((rc = conv_wgrad(d, 4, d->gd2, d->u2, d->e2, L[2].w, L[2].h, n, st))) return rc;
    if ((rc = conv_dgrad(d, 4, d->gd2, L[2].w, L[2].h, n, d->gu2, d->u2, d->ge2, d->e2, st))) return rc;
    up_bwd(d->gu2, d->ge3, 128, 2);
    // bottleneck e3 = c3(p2)
    if ((rc = conv_wgrad(d, 3, d->ge3, d->p2, nullptr, L[3].w, L[3].h, n, st))) return rc;
    if ((rc = conv_dgrad(d, 3, d->ge3, L[3].w, L[3].h, n, d->gp2, nullptr, nullptr, nullptr, st))) return rc;
    pool_bwd(d->gp2, d->e2, d->ge2, 96, 2);
    // encoder e2 = c2(p1)
    if ((rc = conv_wgrad(d, 2, d->ge2, d->p1, nullptr, L[2].w, L[2].h, n, st))) return rc;
    if ((rc = conv_dgrad(d, 2, d->ge2, L[2].w, L[2].h, n, d->gp1, nullptr, nullptr, nullptr, st))) return rc;
    pool_bwd(d->gp1, d->e1, d->ge1, 64, 1);
    // encoder e1 = c1(p0)
    if ((rc = conv_wgrad(d, 1, d->ge1, d->p0, nullptr, L[1].w, L[1].h, n, st))) return rc;
    if ((rc = conv_dgrad(d, 1, d->ge1, L[1].w, L[1].h, n, d->gp0, nullptr, nullptr, nullptr, st))) return rc;
    pool_bwd(d->gp0, d->e0, d->ge0, 32, 0);
    // encoder e0 = c0(x)
    if ((rc = conv_wgrad(d, 0, d->ge0, d->x, nullptr, W0, H0, n, st))) return rc;
    DN_CK(cudaGetLastError());
    return RL_OK;
}

int pack_all(rl_denoiser* d, cudaStream_t st) {
    for (int l = 0; l < 8; l++) {
        Conv& c = d->conv[l];
        const long long K = pad16(c.segs[0]) + (c.segs[1] ? pad16(c.segs[1]) : 0);
        long long tot = 9LL * K * c.ncols + 9LL * c.ncols * c.kpad;
        k_dn_pack<<<grid_of(tot, 256), 256, 0, st>>>(c.w, c.cout, c.ncols, c.segs[0], c.segs[1], c.kpad, c.wp, c.wt);
        DN_CK(cudaMemcpyAsync(c.bias, c.b, c.cout * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    DN_CK(cudaGetLastError());
    return RL_OK;
}

}  // namespace

extern "C" int rl_denoiser_create(uint64_t seed, rl_denoiser** out) {
    if (!out) return dn_fail(RL_INVALID_CALL, "rl_denoiser_create: null argument");
    *out = nullptr;
    rl_denoiser* d = new (std::nothrow) rl_denoiser;
    if (!d) return dn_fail(RL_OUT_OF_MEMORY, "host allocation failed");
    long long floats = 0, halves = 0;
    for (int l = 0; l < 8; l++) {
        Conv& c = d->conv[l];
        c.cout = kCout[l];
        c.ncols = pad16(kCout[l]);
        c.segs[0] = kSeg0[l];
        c.segs[1] = kSeg1[l];
        c.kpad = pad64(c.segs[0]) + (c.segs[1] ? pad64(c.segs[1]) : 0);
        c.copad = pad64(c.ncols);
        floats += 4 * c.nw() + 4 * c.cout + c.ncols + 64;
        halves += (long long)c.ncols * 9 * c.kpad + (long long)c.kpad * 9 * c.copad + 128;
        d->nparam += c.nw() + c.cout;
    }
    cudaError_t e = cudaMalloc(&d->params, floats * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d->packed, halves * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&d->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d->params, 0, floats * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(d->d_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        delete d;
        return dn_fail(RL_OUT_OF_MEMORY, "denoiser parameters: %s", cudaGetErrorString(e));
    }
    float* p = d->params;
    bf16* q = d->packed;
    auto take = [&](long long n) { float* r = p; p += (n + 15) / 16 * 16; return r; };
    for (int l = 0; l < 8; l++) {
        Conv& c = d->conv[l];
        c.w = take(c.nw());
        c.b = take(c.cout);
        c.gw = take(c.nw());
        c.gb = take(c.cout);
        c.mw = take(c.nw());
        c.vw = take(c.nw());
        c.mb = take(c.cout);
        c.vb = take(c.cout);
        c.bias = take(c.ncols);
        c.wp = q;
        q += ((long long)c.ncols * 9 * c.kpad + 63) / 64 * 64;
        c.wt = q;
        q += ((long long)c.kpad * 9 * c.copad + 63) / 64 * 64;
    }
    // weights of the real input channels only; padding columns stay zero
    for (int l = 0; l < 8; l++) {
        Conv& c = d->conv[l];
        std::vector<float> w(c.nw(), 0.f);
        int real0 = l == 0 ? 10 : c.segs[0], real1 = c.segs[1];
        std::vector<float> r((size_t)c.cout * 9 * (real0 + real1));
        init_weights(r, 9 * (real0 + real1), seed + 7919 * (l + 1));
        if (l == 7)
            for (float& v : r) v *= 0.1f;  // start near the identity (prediction = noisy input)
        for (int co = 0; co < c.cout; co++)
            for (int t = 0; t < 9; t++) {
                for (int k = 0; k < real0; k++)
                    w[((size_t)co * 9 + t) * c.kpad + k] = r[((size_t)co * 9 + t) * (real0 + real1) + k];
                for (int k = 0; k < real1; k++)
                    w[((size_t)co * 9 + t) * c.kpad + pad64(c.segs[0]) + k] =
                        r[((size_t)co * 9 + t) * (real0 + real1) + real0 + k];
            }
        e = cudaMemcpy(c.w, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            delete d;
            return dn_fail(RL_CUDA_ERROR, "denoiser init: %s", cudaGetErrorString(e));
        }
    }
    if (int rc = pack_all(d, 0)) {
        delete d;
        return rc;
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        delete d;
        return dn_fail(RL_CUDA_ERROR, "denoiser init: %s", cudaGetErrorString(e));
    }
    *out = d;
    return RL_OK;
}

extern "C" int rl_denoiser_destroy(rl_denoiser* d) {
    if (!d) return dn_fail(RL_INVALID_CALL, "null denoiser");
    cudaDeviceSynchronize();
    delete d;
    return RL_OK;
}

extern "C" int rl_denoiser_param_count(const rl_denoiser* d, int64_t* n) {
    if (!d || !n) return dn_fail(RL_INVALID_CALL, "null argument");
    *n = d->nparam;
    return RL_OK;
}

// Parameters as one host array: per layer, weights [cout][9][kpad] then biases.
extern "C" int rl_denoiser_get_params(const rl_denoiser* d, float* host) {
    if (!d || !host) return dn_fail(RL_INVALID_CALL, "null argument");
    for (int l = 0; l < 8; l++) {
        const Conv& c = d->conv[l];
        DN_CK(cudaMemcpy(host, c.w, c.nw() * sizeof(float), cudaMemcpyDeviceToHost));
        host += c.nw();
        DN_CK(cudaMemcpy(host, c.b, c.cout * sizeof(float), cudaMemcpyDeviceToHost));
        host += c.cout;
    }
    return RL_OK;
}

extern "C" int rl_denoiser_set_params(rl_denoiser* d, const float* host) {
    if (!d || !host) return dn_fail(RL_INVALID_CALL, "null argument");
    for (int l = 0; l < 8; l++) {
        Conv& c = d->conv[l];
        DN_CK(cudaMemcpy(c.w, host, c.nw() * sizeof(float), cudaMemcpyHostToDevice));
        host += c.nw();
        DN_CK(cudaMemcpy(c.b, host, c.cout * sizeof(float), cudaMemcpyHostToDevice));
        host += c.cout;
    }
    if (int rc = pack_all(d, 0)) return rc;
    DN_CK(cudaDeviceSynchronize());
    return RL_OK;
}

// Accumulated gradients in the rl_denoiser_get_params layout; clears them.
extern "C" int rl_denoiser_get_grads(rl_denoiser* d, float* host) {
    if (!d || !host) return dn_fail(RL_INVALID_CALL, "null argument");
    DN_CK(cudaDeviceSynchronize());
    for (int l = 0; l < 8; l++) {
        Conv& c = d->conv[l];
        DN_CK(cudaMemcpy(host, c.gw, c.nw() * sizeof(float), cudaMemcpyDeviceToHost));
        host += c.nw();
        DN_CK(cudaMemcpy(host, c.gb, c.cout * sizeof(float), cudaMemcpyDeviceToHost));
        host += c.cout;
        DN_CK(cudaMemset(c.gw, 0, c.nw() * sizeof(float)));
        DN_CK(cudaMemset(c.gb, 0, c.cout * sizeof(float)));
    }
    return RL_OK;
}

extern "C" int rl_denoiser_features(const rl_scene* scene, const rl_map* map, void* d_x, void* stream) {
    const rl::DevMap* m = rl_internal_map(map);
    const rl::DevScene* s = rl_internal_scene(scene);
    if (!m || !s || !d_x) return dn_fail(RL_INVALID_CALL, "rl_denoiser_features: null argument");
    long long n = (long long)m->width * m->height;
    k_dn_features<<<grid_of(n, 256), 256, 0, (cudaStream_t)stream>>>(*s, *m, (bf16*)d_x);
    DN_CK(cudaGetLastError());
    return RL_OK;
}

extern "C" int rl_denoiser_targets(const rl_map* map, float* d_t, void* stream) {
    const rl::DevMap* m = rl_internal_map(map);
    if (!m || !d_t) return dn_fail(RL_INVALID_CALL, "rl_denoiser_targets: null argument");
    long long n = (long long)m->width * m->height;
    k_dn_targets<<<grid_of(n, 256), 256, 0, (cudaStream_t)stream>>>(*m, (float4*)d_t);
    DN_CK(cudaGetLastError());
    return RL_OK;
}

extern "C" int rl_denoiser_train_step(rl_denoiser* d, const void* d_x, const float* d_t, int batch, int patch,
                                      float lr, float* d_loss, void* stream) {
    if (!d || !d_x || !d_t || batch <= 0 || patch < 8) return dn_fail(RL_INVALID_CALL, "rl_denoiser_train_step: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    if (int rc = alloc_shapes(d, batch, patch, patch, true, st)) return rc;
    const long long P = (long long)batch * patch * patch;
    DN_CK(cudaMemcpyAsync(d->x, d_x, P * kFeat * sizeof(bf16), cudaMemcpyDeviceToDevice, st));
    DN_CK(cudaMemcpyAsync(d->tgt, d_t, P * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    // gradient buffers that are accumulated into start at zero
    if (int rc = forward(d, batch, patch, patch, st)) return rc;
    k_dn_loss<<<grid_of(P, 256), 256, 0, st>>>(d->y, d->x, d->tgt, P, 1.0f / (float)(P * 3), d->gy, d_loss);
    if (int rc = backward(d, batch, patch, patch, st)) return rc;
    if (lr < 0.f) return RL_OK;  // gradients only (rl_denoiser_get_grads)
    d->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - powf(b1, (float)d->step), bc2 = 1.f - powf(b2, (float)d->step);
    for (int l = 0; l < 8; l++) {
        Conv& c = d->conv[l];
        k_dn_adam<<<grid_of(c.nw(), 256), 256, 0, st>>>(c.w, c.gw, c.mw, c.vw, c.nw(), lr, b1, b2, 1e-8f, bc1, bc2);
        k_dn_adam<<<1, 128, 0, st>>>(c.b, c.gb, c.mb, c.vb, c.cout, lr, b1, b2, 1e-8f, bc1, bc2);
    }
    return pack_all(d, st);
}

extern "C" int rl_denoiser_apply(rl_denoiser* d, const rl_scene* scene, rl_map* map, const float* d_base,
                                 void* stream) {
    const rl::DevMap* m = rl_internal_map(map);
    const rl::DevScene* s = rl_internal_scene(scene);
    if (!d || !m || !s) return dn_fail(RL_INVALID_CALL, "rl_denoiser_apply: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (int rc = alloc_shapes(d, 1, m->height, m->width, false, st)) return rc;
    long long n = (long long)m->width * m->height;
    k_dn_features<<<grid_of(n, 256), 256, 0, st>>>(*s, *m, d->x);
    if (int rc = forward(d, 1, m->height, m->width, st)) return rc;
    k_dn_apply<<<grid_of(n, 256), 256, 0, st>>>(d->y, d->x, *m, d_base);
    DN_CK(cudaGetLastError());
    return RL_OK;
}

extern "C" int rl_denoiser_forward(rl_denoiser* d, const void* d_x, int images, int height, int width, void* d_y,
                                   void* stream) {
    if (!d || !d_x || !d_y) return dn_fail(RL_INVALID_CALL, "rl_denoiser_forward: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (int rc = alloc_shapes(d, images, height, width, d->btrain != 0, st)) return rc;
    const long long P = (long long)images * height * width;
    DN_CK(cudaMemcpyAsync(d->x, d_x, P * kFeat * sizeof(bf16), cudaMemcpyDeviceToDevice, st));
    if (int rc = forward(d, images, height, width, st)) return rc;
    DN_CK(cudaMemcpyAsync(d_y, d->y, P * kFeat * sizeof(bf16), cudaMemcpyDeviceToDevice, st));
    return RL_OK;
}

extern "C" int rl_denoiser_reserve(rl_denoiser* d, int images, int height, int width, int train) {
    if (!d || images <= 0 || height <= 0 || width <= 0) return dn_fail(RL_INVALID_CALL, "rl_denoiser_reserve: bad arguments");
    if (int rc = alloc_shapes(d, images, height, width, train != 0, 0)) return rc;
    DN_CK(cudaDeviceSynchronize());
    return RL_OK;
}

extern "C" int rl_denoiser_status(rl_denoiser* d, int* flags) {
    if (!d || !flags) return dn_fail(RL_INVALID_CALL, "null argument");
    DN_CK(cudaMemcpy(flags, d->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    return RL_OK;
}
