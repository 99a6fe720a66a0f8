// mlp.cu -- the importance-sampling proposal network (include/mcg_is.h).
//
// 16 features -> 64 -> 64 -> 1, ReLU, sigmoid; BF16 operands, FP32
// accumulation.  Every dense product -- the two hidden layers forward, the
// back-propagated hidden gradient, and the weight and bias gradients -- is a
// tcgen05.mma on the fifth-generation tensor cores with its accumulator in
// tensor memory (TMEM); the output layer (64 -> 1), the sigmoid and the loss
// are per-row work on the CUDA cores.
//
// A CTA of 128 threads works on tiles of 128 rows: TMEM lane r and thread r
// hold row r, so a tcgen05.ld of an accumulator gives each thread its own
// row and every row-wise step (bias, ReLU, output dot product, loss) stays
// in one thread.  Feature rows arrive by bulk copies (cp.async.bulk with an
// mbarrier transaction count), the next tile's while the current one is
// computed.  One elected thread issues the MMAs and commits them to an
// mbarrier the others wait on (bounded waits: a wait that runs out sets an
// error flag the host reads, and the CTA releases its TMEM and returns).
//
// Shared-memory operands use the tensor cores' no-swizzle canonical layout:
// a tile of rows x units (BF16) is stored as 8 x 8 blocks of 128 contiguous
// bytes, line i of a block holding row 8 rb + i's units 8 ub .. 8 ub + 7,
// blocks ordered row-block-major.  The same bytes serve as a K-major operand
// (rows as M, units as K) and as an MN-major one (units as M or N, rows as
// K); only the descriptor's two block strides differ.  The weight gradients
// reduce over rows, so they are products with K = rows whose accumulators
// stay in TMEM across all of a CTA's tiles:
//   G1 = [dH2 | H2]^T [H1 | 1 | dz]  ->  dW2^T, db2 (rows 0..63), dW3 (rows 64..127, column 65)
//   G2 = [dH1 | dH2]^T [X | 1]       ->  dW1^T, db1 (rows 0..63; rows 64..127 unused)
// Each CTA writes one partial gradient and a second kernel sums them in CTA
// order (the same rows give the same gradient bit for bit).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "error.hpp"
#include "mcg_is.h"

namespace {

#define MCG_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t err_ = (call);                                                              \
        if (err_ != cudaSuccess) {                                                              \
            return mcg::fail(err_ == cudaErrorMemoryAllocation ? MCG_ERR_OOM : MCG_ERR_CUDA,    \
                             std::string(#call) + ": " + cudaGetErrorString(err_));             \
        }                                                                                       \
    } while (0)

constexpr int kIn = MCG_MLP_IN;       // 16
constexpr int kHid = MCG_MLP_HIDDEN;  // 64
// parameter offsets (FP32 master layout)
constexpr int kOffW1 = 0;                  // [16][64]
constexpr int kOffB1 = kOffW1 + kIn * kHid;   // [64]
constexpr int kOffW2 = kOffB1 + kHid;         // [64][64]
constexpr int kOffB2 = kOffW2 + kHid * kHid;  // [64]
constexpr int kOffW3 = kOffB2 + kHid;         // [64]
constexpr int kOffB3 = kOffW3 + kHid;         // [1]
constexpr int kParams = kOffB3 + 1;
static_assert(kParams == MCG_MLP_PARAMS, "parameter layout");

typedef __nv_bfloat16 bf16;

// Packed BF16 operands: W1t[64][16] and W2t[64][64] (output-major), W3[64].
constexpr int kPackW1t = 0;
constexpr int kPackW2t = kPackW1t + kHid * kIn;
constexpr int kPackW3 = kPackW2t + kHid * kHid;
constexpr int kPackSize = kPackW3 + kHid;

constexpr int kTile = 128;     // rows per tile: the MMA's M, TMEM lanes, threads
constexpr int kThreads = 128;  // 4 warps; warp w reads TMEM lanes 32w .. 32w + 31
constexpr int kCtasPerSm = 2;  // two CTAs of 256 TMEM columns fill the SM's 512
constexpr uint32_t kTmemCols = 256;
// TMEM columns (FP32 accumulators, 128 lanes each)
constexpr uint32_t kColD1 = 0;    // X W1; later dH2 W2^T
constexpr uint32_t kColD2 = 64;   // H1 W2
constexpr uint32_t kColG1 = 128;  // 80 columns, accumulated over the CTA's tiles
constexpr uint32_t kColG2 = 208;  // 32 columns, accumulated over the CTA's tiles
// units per row of the shared-memory tiles
constexpr int kUnitsX = 32;   // X (16) | 1 | 0 ...            (B of G2, A of layer 1)
constexpr int kUnitsE = 80;   // H1 (64) | 1 | dz | 0 ...      (A of layer 2, B of G1)
constexpr int kUnitsC = 192;  // dH1 (64) | dH2 (64) | H2 (64) (A of dH2 W2^T, G1, G2)
constexpr uint32_t kRowBlockX = kUnitsX / 8 * 128;  // bytes between row blocks
constexpr uint32_t kRowBlockE = kUnitsE / 8 * 128;
constexpr uint32_t kRowBlockC = kUnitsC / 8 * 128;
constexpr uint64_t kWaitNs = 2000000000ull;  // bound of every mbarrier wait (2 s)

struct alignas(128) TcSmem {
    float stage[kTile * kIn];  // the next tile's feature rows as the bulk copy leaves them
    bf16 x[2][kTile * kUnitsX];  // two X tiles: a tile's G2 product may still read one while the next is filled
    bf16 e[kTile * kUnitsE];
    bf16 c[kTile * kUnitsC];
    bf16 w1[kHid * kIn];     // B of layer 1: N = hidden, K = feature (K-major)
    bf16 w2[kHid * kHid];    // B of layer 2: N = out, K = in (K-major); of dH2 W2^T: N = in, K = out (MN-major)
    float b1[kHid], b2[kHid], w3[kHid], w3b[kHid];
    float red[2][kThreads / 32];
    unsigned long long bar_mma, bar_end, bar_rows;
    uint32_t tmem;
};

// --- PTX wrappers --------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned long long *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase with the given parity to complete, for kWaitNs at most.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = now_ns();
    while (!mbar_try(bar, parity)) {
        if (now_ns() - t0 > kWaitNs) return false;
    }
    return true;
}

// Bulk copy of `bytes` (a multiple of 16, 16-byte aligned ends) into shared
// memory, completing a transaction on bar.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, unsigned long long *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Shared-memory matrix descriptor, no swizzle: lbo = bytes between core
// matrices along K, sbo = bytes between core matrices along M/N.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1 (sm_100)
}

// Instruction descriptor: BF16 A and B, FP32 accumulator, M = 128, N = n;
// a_mn / b_mn select the MN-major form of an operand.
__host__ __device__ constexpr uint32_t idesc(int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
}

// D (+)= A B, issued by one thread.
__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(id), "r"((uint32_t)accumulate)
        : "memory");
}

// Arrives on bar once every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(unsigned long long *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

#define MCG_R8(i) "=r"(r[i]), "=r"(r[i + 1]), "=r"(r[i + 2]), "=r"(r[i + 3]), "=r"(r[i + 4]), "=r"(r[i + 5]), \
                  "=r"(r[i + 6]), "=r"(r[i + 7])

// 32 or 16 consecutive FP32 columns of this thread's TMEM lane; the wait is
// in the same statement, so the registers are valid when it returns.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : MCG_R8(0), MCG_R8(8), MCG_R8(16), MCG_R8(24)
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : MCG_R8(0), MCG_R8(8)
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
#undef MCG_R8

// --- tile layout ---------------------------------------------------------

// The 16 bytes holding units 8 ub .. 8 ub + 7 of row r in a tile of `units` per row.
template <int Units>
__device__ __forceinline__ uint4 *chunk(bf16 *tile, int r, int ub) {
    return reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(tile) +
                                     ((uint32_t)((r >> 3) * (Units / 8) + ub) << 7) + ((uint32_t)(r & 7) << 4));
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a in the low half (lower unit)
    return *reinterpret_cast<const uint32_t *>(&h);
}

__device__ __forceinline__ void unpack8(const uint4 &q, float (&f)[8]) {
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        f[2 * i] = __uint_as_float(w[i] << 16);
        f[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
    }
}

__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
    return make_uint4(pack2(f[0], f[1]), pack2(f[2], f[3]), pack2(f[4], f[5]), pack2(f[6], f[7]));
}

__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// --- shared steps of the forward and gradient kernels ---------------------

// Weights into their operand layouts, biases and W3; the constant zero
// units of the X and E tiles.  Called by all threads before the first barrier.
__device__ void setup_operands(TcSmem &s, const bf16 *__restrict__ pack, const float *__restrict__ params) {
    const int tid = threadIdx.x;
    unsigned char *w1 = reinterpret_cast<unsigned char *>(s.w1);
    for (int i = tid; i < kHid * kIn; i += kThreads) {  // N = hidden h, K = feature f
        const int h = i / kIn, f = i % kIn;
        *reinterpret_cast<bf16 *>(w1 + (((h >> 3) * (kIn / 8) + (f >> 3)) << 7) + ((h & 7) << 4) + ((f & 7) << 1)) =
            pack[kPackW1t + i];
    }
    unsigned char *w2 = reinterpret_cast<unsigned char *>(s.w2);
    for (int i = tid; i < kHid * kHid; i += kThreads) {  // N = out o, K = in j
        const int o = i / kHid, j = i % kHid;
        *reinterpret_cast<bf16 *>(w2 + (((o >> 3) * (kHid / 8) + (j >> 3)) << 7) + ((o & 7) << 4) + ((j & 7) << 1)) =
            pack[kPackW2t + i];
    }
    for (int i = tid; i < kHid; i += kThreads) {
        s.b1[i] = params[kOffB1 + i];
        s.b2[i] = params[kOffB2 + i];
        s.w3[i] = params[kOffW3 + i];
        s.w3b[i] = __bfloat162float(pack[kPackW3 + i]);
    }
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
    *chunk<kUnitsX>(s.x[0], tid, 3) = zero;  // units 24..31
    *chunk<kUnitsX>(s.x[1], tid, 3) = zero;
    *chunk<kUnitsE>(s.e, tid, 9) = zero;  // units 72..79
}

// TMEM allocation (warp 0) and mbarriers (thread 0); returns after the
// barrier that publishes both.
__device__ uint32_t setup_tmem_and_barriers(TcSmem &s) {
    const int tid = threadIdx.x;
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s.tmem)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&s.bar_mma, 1);
        mbar_init(&s.bar_end, 1);
        mbar_init(&s.bar_rows, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    return s.tmem;
}

// Barrier that also agrees on ok across the CTA; a failure anywhere ends the
// tile loop in every thread with ok = false.
#define MCG_SYNC_OR_BREAK()                    \
    if (!__syncthreads_and(ok)) {              \
        ok = false;                            \
        break;                                 \
    }

__device__ void release_tmem(uint32_t tmem) {
    tc_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// Thread 0: the bulk copy of tile `tile`'s feature rows into the stage
// (the copy of the CTA's j-th tile completes phase j of bar_rows).
__device__ __forceinline__ void load_rows(TcSmem &s, const float *__restrict__ feat, uint32_t n, uint32_t tile) {
    const uint32_t row0 = tile * kTile;
    const uint32_t rows = min((uint32_t)kTile, n - row0);
    bulk_load(s.stage, feat + (uint64_t)row0 * kIn, rows * kIn * (uint32_t)sizeof(float), &s.bar_rows);
}

// Row r of the staged features (zero past n) into X tile xb, with the ones unit.
__device__ __forceinline__ void rows_to_x(TcSmem &s, int xb, bool valid) {
    const int r = threadIdx.x;
    const float4 *src = reinterpret_cast<const float4 *>(s.stage + r * kIn);
    float f[16];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float4 q = valid ? src[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        f[4 * i] = q.x;
        f[4 * i + 1] = q.y;
        f[4 * i + 2] = q.z;
        f[4 * i + 3] = q.w;
    }
    bf16 *x = s.x[xb];
    *chunk<kUnitsX>(x, r, 0) = make_uint4(pack2(f[0], f[1]), pack2(f[2], f[3]), pack2(f[4], f[5]), pack2(f[6], f[7]));
    *chunk<kUnitsX>(x, r, 1) =
        make_uint4(pack2(f[8], f[9]), pack2(f[10], f[11]), pack2(f[12], f[13]), pack2(f[14], f[15]));
    *chunk<kUnitsX>(x, r, 2) = make_uint4(valid ? 0x3F80u : 0u, 0u, 0u, 0u);  // unit 16 = 1.0 (BF16 0x3F80)
}

// Thread 0: D1 = X W1 (one K = 16 step) from X tile xb.
__device__ __forceinline__ void issue_layer1(TcSmem &s, uint32_t tmem, int xb) {
    umma(tmem + kColD1, sdesc(smem_addr(s.x[xb]), 128, kRowBlockX), sdesc(smem_addr(s.w1), 128, 2 * 128),
         idesc(kHid, false, false), false);
}

// Thread 0: G2 += [dH1 | dH2]^T [X | 1] for the tile whose X tile is xb and
// whose dH1, dH2 are in the C tile (K = rows, both operands MN-major).
__device__ __forceinline__ void issue_g2(TcSmem &s, uint32_t tmem, int xb, bool accumulate) {
    const uint32_t a_c = smem_addr(s.c), a_x = smem_addr(s.x[xb]);
#pragma unroll
    for (int k = 0; k < kTile / 16; ++k)
        umma(tmem + kColG2, sdesc(a_c + 2 * kRowBlockC * k, kRowBlockC, 128),
             sdesc(a_x + 2 * kRowBlockX * k, kRowBlockX, 128), idesc(32, true, true), accumulate || k > 0);
}

// Thread 0: D2 = H1 W2 (four K = 16 steps).
__device__ __forceinline__ void issue_layer2(TcSmem &s, uint32_t tmem) {
#pragma unroll
    for (int k = 0; k < kHid / 16; ++k)
        umma(tmem + kColD2, sdesc(smem_addr(s.e) + 256 * k, 128, kRowBlockE),
             sdesc(smem_addr(s.w2) + 256 * k, 128, (kHid / 8) * 128), idesc(kHid, false, false), k > 0);
}

// H1 = relu(D1 + b1) into units 0..63 of the E tile.
__device__ __forceinline__ void epilogue_h1(TcSmem &s, uint32_t t_row) {
    const int r = threadIdx.x;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        float v[32];
        tmem_ld32(t_row + kColD1 + 32 * half, v);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            float h[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) h[j] = fmaxf(v[8 * g + j] + s.b1[32 * half + 8 * g + j], 0.f);
            *chunk<kUnitsE>(s.e, r, 4 * half + g) = pack8(h);
        }
    }
}

// H2 = relu(D2 + b2) (BF16-rounded), optionally stored into units 128..191
// of the C tile; returns z = H2 . W3 + b3 with BF16 W3 and FP32 sums.
template <bool STORE>
__device__ __forceinline__ float epilogue_h2(TcSmem &s, uint32_t t_row, float b3) {
    const int r = threadIdx.x;
    float z = b3;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        float v[32];
        tmem_ld32(t_row + kColD2 + 32 * half, v);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            float h[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int u = 32 * half + 8 * g + j;
                h[j] = bf16_round(fmaxf(v[8 * g + j] + s.b2[u], 0.f));
                z = fmaf(h[j], s.w3b[u], z);
            }
            if constexpr (STORE) *chunk<kUnitsC>(s.c, r, 16 + 4 * half + g) = pack8(h);
        }
    }
    return z;
}

// Error exit (a wait ran out), thread 0: record it, let the bulk copies
// still in flight land (the CTA's tiles [waited, issued)) and let every MMA
// it issued finish (commits_end arrivals were committed to bar_end before),
// so that shared memory and TMEM are no longer in use when the CTA leaves.
__device__ void on_timeout(TcSmem &s, int *err, uint32_t waited, uint32_t issued, uint32_t commits_end) {
    atomicExch(err, 1);
    for (uint32_t j = waited; j < issued; ++j) mbar_wait(&s.bar_rows, j & 1);
    umma_commit(&s.bar_end);
    mbar_wait(&s.bar_end, commits_end & 1);
}

// q = sigmoid(network(features)) for rows [0, n): persistent CTAs over 128-row tiles.
__global__ void __launch_bounds__(kThreads, kCtasPerSm)
    k_mlp_forward(const bf16 *__restrict__ pack, const float *__restrict__ params, const float *__restrict__ feat,
                  uint32_t n, float *__restrict__ q, int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TcSmem &s = *reinterpret_cast<TcSmem *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t my_tiles = blockIdx.x < tiles ? (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
    setup_operands(s, pack, params);
    const uint32_t tmem = setup_tmem_and_barriers(s);
    const uint32_t t_row = tmem + ((uint32_t)(warp * 32) << 16);
    const float b3 = params[kOffB3];
    uint32_t issued = 0;  // bulk copies issued (thread 0)
    if (tid == 0 && my_tiles > 0) {
        load_rows(s, feat, n, blockIdx.x);
        issued = 1;
    }
    bool ok = true;
    uint32_t ph = 0, i = 0;
    for (; i < my_tiles; ++i) {
        const uint32_t tile = blockIdx.x + i * gridDim.x;
        const uint32_t row = tile * kTile + tid;
        ok = mbar_wait(&s.bar_rows, i & 1) && ok;
        rows_to_x(s, 0, row < n);
        fence_async_smem();
        tc_before_sync();
        MCG_SYNC_OR_BREAK();
        tc_after_sync();
        if (tid == 0) {
            if (i + 1 < my_tiles) {  // every thread has read the stage
                load_rows(s, feat, n, tile + gridDim.x);
                ++issued;
            }
            issue_layer1(s, tmem, 0);
            umma_commit(&s.bar_mma);
        }
        ok = mbar_wait(&s.bar_mma, ph) && ok;
        ph ^= 1;
        tc_after_sync();
        epilogue_h1(s, t_row);
        fence_async_smem();
        tc_before_sync();
        MCG_SYNC_OR_BREAK();
        tc_after_sync();
        if (tid == 0) {
            issue_layer2(s, tmem);
            umma_commit(&s.bar_mma);
        }
        ok = mbar_wait(&s.bar_mma, ph) && ok;
        ph ^= 1;
        tc_after_sync();
        const float z = epilogue_h2<false>(s, t_row, b3);
        if (ok && row < n) q[row] = 1.f / (1.f + __expf(-z));
        tc_before_sync();  // the next tile's layer 2 overwrites D2 after the next barrier
    }
    ok = __syncthreads_and(ok) != 0;
    if (!ok && tid == 0) on_timeout(s, err, i, issued, 0);
    release_tmem(tmem);
}

// Weighted BCE gradient of rows [0, n): persistent CTAs, CTA b taking tiles
// b, b + gridDim.x, ...; its gradient (kParams floats, then the loss) goes to
// partial[b * (kParams + 1) ..], every entry written once.  A tile's G2
// product is issued with the next tile's layer 1 (or after the last tile):
// it reads that tile's X tile (two alternate) and the dH1, dH2 units of the
// C tile, which the next tile overwrites only after layer 1's completion --
// and a commit covers every MMA issued before it.
__global__ void __launch_bounds__(kThreads, kCtasPerSm)
    k_mlp_grad(const bf16 *__restrict__ pack, const float *__restrict__ params, const float *__restrict__ feat,
               const float *__restrict__ tgt, const float *__restrict__ wts, float inv_wsum, uint32_t n,
               float *__restrict__ partial, int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TcSmem &s = *reinterpret_cast<TcSmem *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t my_tiles = blockIdx.x < tiles ? (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
    setup_operands(s, pack, params);
    const uint32_t tmem = setup_tmem_and_barriers(s);
    const uint32_t t_row = tmem + ((uint32_t)(warp * 32) << 16);
    const float b3 = params[kOffB3];
    const uint32_t a_e = smem_addr(s.e), a_c = smem_addr(s.c), a_w2 = smem_addr(s.w2);
    uint32_t issued = 0, commits_end = 0;  // thread 0's bulk copies and bar_end commits
    if (tid == 0 && my_tiles > 0) {
        load_rows(s, feat, n, blockIdx.x);
        issued = 1;
    }
    float loss = 0.f, gb3 = 0.f;
    bool ok = true;
    uint32_t ph = 0, i = 0;
    for (; i < my_tiles; ++i) {
        const uint32_t tile = blockIdx.x + i * gridDim.x;
        const int xb = (int)(i & 1);
        const uint32_t row = tile * kTile + tid;
        const bool valid = row < n;
        const float tv = valid ? tgt[row] : 0.f;
        const float wv = valid ? (wts ? wts[row] : 1.f) * inv_wsum : 0.f;
        ok = mbar_wait(&s.bar_rows, i & 1) && ok;
        rows_to_x(s, xb, valid);  // the X tile tile i - 2 used: its G2 completed before tile i - 1's layer 1 did
        fence_async_smem();
        tc_before_sync();
        MCG_SYNC_OR_BREAK();
        tc_after_sync();
        if (tid == 0) {
            if (i + 1 < my_tiles) {  // every thread has read the stage
                load_rows(s, feat, n, tile + gridDim.x);
                ++issued;
            }
            if (i > 0) issue_g2(s, tmem, xb ^ 1, i > 1);
            issue_layer1(s, tmem, xb);
            umma_commit(&s.bar_mma);  // also covers the previous tile's G1 and G2
        }
        ok = mbar_wait(&s.bar_mma, ph) && ok;
        ph ^= 1;
        tc_after_sync();
        epilogue_h1(s, t_row);
        fence_async_smem();
        tc_before_sync();
        MCG_SYNC_OR_BREAK();
        tc_after_sync();
        if (tid == 0) {
            issue_layer2(s, tmem);
            umma_commit(&s.bar_mma);
        }
        ok = mbar_wait(&s.bar_mma, ph) && ok;
        ph ^= 1;
        tc_after_sync();
        const float z = epilogue_h2<true>(s, t_row, b3);
        // dL/dz = w (q - t) / sum w
        float d = 0.f;
        if (valid) {
            const float qv = 1.f / (1.f + __expf(-z));
            d = wv * (qv - tv);
            const float qc = fminf(fmaxf(qv, 1e-7f), 1.f - 1e-7f);
            loss -= wv * (tv * __logf(qc) + (1.f - tv) * __logf(1.f - qc));
        }
        gb3 += d;
        // dH2 = d W3 where H2 > 0, into units 64..127 of C; [1, d] into units 64, 65 of E
#pragma unroll
        for (int g = 0; g < 8; ++g) {
            float h[8], dh[8];
            unpack8(*chunk<kUnitsC>(s.c, tid, 16 + g), h);
#pragma unroll
            for (int j = 0; j < 8; ++j) dh[j] = h[j] > 0.f ? d * s.w3[8 * g + j] : 0.f;
            *chunk<kUnitsC>(s.c, tid, 8 + g) = pack8(dh);
        }
        *chunk<kUnitsE>(s.e, tid, 8) = make_uint4(pack2(valid ? 1.f : 0.f, d), 0u, 0u, 0u);
        fence_async_smem();
        tc_before_sync();
        MCG_SYNC_OR_BREAK();
        tc_after_sync();
        if (tid == 0) {
            // dH2 W2^T into D1's columns: A = dH2 (K-major, K = out), B = W2 read as N = in, K = out (MN-major)
#pragma unroll
            for (int k = 0; k < kHid / 16; ++k)
                umma(tmem + kColD1, sdesc(a_c + 8 * 128 + 256 * k, 128, kRowBlockC),
                     sdesc(a_w2 + 2 * (kHid / 8) * 128 * k, (kHid / 8) * 128, 128), idesc(kHid, false, true), k > 0);
            umma_commit(&s.bar_mma);
            // G1 += [dH2 | H2]^T [H1 | 1 | d]: K = rows, both operands MN-major
#pragma unroll
            for (int k = 0; k < kTile / 16; ++k)
                umma(tmem + kColG1, sdesc(a_c + 8 * 128 + 2 * kRowBlockC * k, kRowBlockC, 128),
                     sdesc(a_e + 2 * kRowBlockE * k, kRowBlockE, 128), idesc(80, true, true), i > 0 || k > 0);
        }
        ok = mbar_wait(&s.bar_mma, ph) && ok;
        ph ^= 1;
        tc_after_sync();
        // dH1 = D1 where H1 > 0, into units 0..63 of C
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            float v[32];
            tmem_ld32(t_row + kColD1 + 32 * half, v);
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                float h[8], dh[8];
                unpack8(*chunk<kUnitsE>(s.e, tid, 4 * half + g), h);
#pragma unroll
                for (int j = 0; j < 8; ++j) dh[j] = h[j] > 0.f ? v[8 * g + j] : 0.f;
                *chunk<kUnitsC>(s.c, tid, 4 * half + g) = pack8(dh);
            }
        }
        fence_async_smem();  // published by the next barrier, before this tile's G2 is issued
        tc_before_sync();
    }
    ok = __syncthreads_and(ok) != 0;
    if (ok && i > 0) {
        tc_after_sync();
        if (tid == 0) {
            issue_g2(s, tmem, (int)((i - 1) & 1), i > 1);
            umma_commit(&s.bar_end);
            commits_end = 1;
            ok = mbar_wait(&s.bar_end, 0);
        }
        ok = __syncthreads_and(ok) != 0;
    }
    float *out = partial + (uint64_t)blockIdx.x * (kParams + 1);
    if (ok) {
        tc_after_sync();
        float g1[80], g2[32];
        {
            float v[32];
            tmem_ld32(t_row + kColG1, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) g1[j] = v[j];
            tmem_ld32(t_row + kColG1 + 32, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) g1[32 + j] = v[j];
            float w[16];
            tmem_ld16(t_row + kColG1 + 64, w);
#pragma unroll
            for (int j = 0; j < 16; ++j) g1[64 + j] = w[j];
            tmem_ld32(t_row + kColG2, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) g2[j] = v[j];
        }
        if (i == 0) {  // no tile: the accumulators were never written
#pragma unroll
            for (int j = 0; j < 80; ++j) g1[j] = 0.f;
#pragma unroll
            for (int j = 0; j < 32; ++j) g2[j] = 0.f;
        }
        if (tid < kHid) {  // row tid of G1: out unit tid of dW2^T; of G2: hidden unit tid of dW1^T
#pragma unroll
            for (int j = 0; j < kHid; ++j) out[kOffW2 + j * kHid + tid] = g1[j];
            out[kOffB2 + tid] = g1[64];
#pragma unroll
            for (int f = 0; f < kIn; ++f) out[kOffW1 + f * kHid + tid] = g2[f];
            out[kOffB1 + tid] = g2[16];
        } else {  // row tid of G1: H2 unit tid - 64 against d
            out[kOffW3 + tid - kHid] = g1[65];
        }
    } else if (tid == 0) {
        on_timeout(s, err, i, issued, commits_end);
    }
    // loss and db3: sums over the CTA's threads
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
        gb3 += __shfl_xor_sync(0xFFFFFFFFu, gb3, o);
    }
    if (lane == 0) {
        s.red[0][warp] = loss;
        s.red[1][warp] = gb3;
    }
    __syncthreads();
    if (tid == 0) {
        float l = 0.f, g = 0.f;
        for (int w = 0; w < kThreads / 32; ++w) {
            l += s.red[0][w];
            g += s.red[1][w];
        }
        out[kOffB3] = g;
        out[kParams] = l;
    }
    release_tmem(tmem);
}

// grad[i] = sum over the CTAs of partial[b][i] (i = kParams: the loss).  A
// block of 256 threads takes 32 entries: thread (g, p) sums the partials
// b = g, g + 8, ... of entry p, then the eight sums are added in g order --
// a fixed order, so the same partials give the same gradient bit for bit.
constexpr int kReduceCols = 32, kReduceGroups = 8;
__global__ void __launch_bounds__(kReduceCols * kReduceGroups)
    k_mlp_reduce(const float *__restrict__ partial, uint32_t blocks, float *__restrict__ grad,
                 float *__restrict__ loss) {
    __shared__ float part[kReduceGroups][kReduceCols];
    const int p = threadIdx.x % kReduceCols, g = threadIdx.x / kReduceCols;
    const int i = blockIdx.x * kReduceCols + p;
    float v = 0.f;
    if (i <= kParams)
        for (uint32_t b = g; b < blocks; b += kReduceGroups) v += partial[(uint64_t)b * (kParams + 1) + i];
    part[g][p] = v;
    __syncthreads();
    if (g == 0 && i <= kParams) {
        float t = 0.f;
#pragma unroll
        for (int k = 0; k < kReduceGroups; ++k) t += part[k][p];
        if (i < kParams) grad[i] = t;
        else *loss = t;
    }
}

// FP32 master weights -> BF16 operand copies.
__global__ void k_mlp_pack(const float *__restrict__ p, bf16 *__restrict__ pack) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kPackSize; i += gridDim.x * blockDim.x) {
        float v;
        if (i < kPackW2t) {  // W1t[h][f] = W1[f][h]
            const int h = i / kIn, f = i % kIn;
            v = p[kOffW1 + f * kHid + h];
        } else if (i < kPackW3) {  // W2t[o][in] = W2[in][o]
            const int j = i - kPackW2t, o = j / kHid, in = j % kHid;
            v = p[kOffW2 + in * kHid + o];
        } else {
            v = p[kOffW3 + (i - kPackW3)];
        }
        pack[i] = __float2bfloat16(v);
    }
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       float lr, float b1c, float b2c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / b1c) / (sqrtf(vi / b2c) + 1e-8f);
}

}  // namespace

struct mcg_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    float *d_params = nullptr, *d_grad = nullptr, *d_m = nullptr, *d_v = nullptr, *d_loss = nullptr;
    bf16 *d_pack = nullptr;
    float *d_feat = nullptr, *d_tgt = nullptr, *d_w = nullptr, *d_q = nullptr;
    float *d_partial = nullptr;  // [ctas][kParams + 1] per-CTA gradients and losses
    int *d_err = nullptr;        // set by a kernel whose tensor-core or copy wait ran out
    uint32_t ctas = 0;           // persistent CTAs of the forward and gradient kernels
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // around the steps of the last mcg_mlp_train
    double train_ms = 0.0;
    uint32_t cap = 0;
    uint64_t adam_t = 0;
};

namespace {

mcg_status ensure_rows(mcg_mlp *m, uint32_t n) {
    if (n <= m->cap) return MCG_OK;
    cudaFree(m->d_feat);
    cudaFree(m->d_tgt);
    cudaFree(m->d_w);
    cudaFree(m->d_q);
    m->d_feat = m->d_tgt = m->d_w = m->d_q = nullptr;
    m->cap = 0;
    MCG_CUDA(cudaMalloc((void **)&m->d_feat, (size_t)n * kIn * sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_tgt, (size_t)n * sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_w, (size_t)n * sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_q, (size_t)n * sizeof(float)));
    m->cap = n;
    return MCG_OK;
}

// After a synchronised call: did one of its kernels give up on a tensor-core or copy wait?
mcg_status check_waits(mcg_mlp *m) {
    int err = 0;
    MCG_CUDA(cudaMemcpy(&err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err)
        return mcg::fail(MCG_ERR_CUDA, "proposal network: a tensor-core or bulk-copy wait timed out (results invalid)");
    return MCG_OK;
}

mcg_status pack(mcg_mlp *m) {
    k_mlp_pack<<<(kPackSize + 255) / 256, 256, 0, m->stream>>>(m->d_params, m->d_pack);
    MCG_CUDA(cudaGetLastError());
    return MCG_OK;
}

// The gradient of the uploaded rows into d_grad and d_loss: the persistent
// gradient kernel, then the reduction of its partials.
mcg_status grad_pass(mcg_mlp *m, uint32_t n, float inv_wsum, bool has_w) {
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>(tiles, m->ctas));
    k_mlp_grad<<<blocks, kThreads, sizeof(TcSmem), m->stream>>>(m->d_pack, m->d_params, m->d_feat, m->d_tgt,
                                                               has_w ? m->d_w : nullptr, inv_wsum, n, m->d_partial,
                                                               m->d_err);
    MCG_CUDA(cudaGetLastError());
    k_mlp_reduce<<<(kParams + 1 + kReduceCols - 1) / kReduceCols, kReduceCols * kReduceGroups, 0, m->stream>>>(
        m->d_partial, blocks, m->d_grad, m->d_loss);
    MCG_CUDA(cudaGetLastError());
    return MCG_OK;
}

// The call's rows to the device; also clears the wait-timeout flag, so that
// check_waits reports this call's kernels only.
mcg_status upload_rows(mcg_mlp *m, const float *feat, const float *tgt, const float *w, uint32_t n, float &inv_wsum) {
    mcg_status st = ensure_rows(m, n);
    if (st != MCG_OK) return st;
    MCG_CUDA(cudaMemsetAsync(m->d_err, 0, sizeof(int), m->stream));
    MCG_CUDA(cudaMemcpyAsync(m->d_feat, feat, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    if (tgt) MCG_CUDA(cudaMemcpyAsync(m->d_tgt, tgt, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    double ws = 0.0;
    if (w) {
        for (uint32_t i = 0; i < n; ++i) ws += w[i];
        MCG_CUDA(cudaMemcpyAsync(m->d_w, w, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    } else {
        ws = n;
    }
    inv_wsum = ws > 0 ? (float)(1.0 / ws) : 0.f;
    return MCG_OK;
}

}  // namespace

extern "C" {

mcg_status mcg_mlp_create(int32_t device, uint64_t seed, mcg_mlp **out) {
    mcg::clear_error();
    if (!out) return mcg::fail(MCG_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
        cudaGetLastError();
        return mcg::fail(MCG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    auto m = std::make_unique<mcg_mlp>();
    m->device = device;
    MCG_CUDA(cudaSetDevice(device));
    MCG_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    MCG_CUDA(cudaMalloc((void **)&m->d_params, kParams * sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_grad, kParams * sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_m, kParams * sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_v, kParams * sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_loss, sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_pack, kPackSize * sizeof(bf16)));
    MCG_CUDA(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem)));
    MCG_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem)));
    // two CTAs per SM need the largest shared-memory carveout
    MCG_CUDA(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    MCG_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int sms = 0, smem_sm = 0, reserved = 0;
    MCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    MCG_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    MCG_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device));
    // CTAs that fit an SM's shared memory, at most two: each holds 256 of the
    // SM's 512 TMEM columns
    const int per_sm = smem_sm / (int)(sizeof(TcSmem) + reserved);
    m->ctas = (uint32_t)std::max(1, sms * std::min(std::max(per_sm, 1), kCtasPerSm));
    MCG_CUDA(cudaMalloc((void **)&m->d_partial, (size_t)m->ctas * (kParams + 1) * sizeof(float)));
    MCG_CUDA(cudaMalloc((void **)&m->d_err, sizeof(int)));
    MCG_CUDA(cudaMemset(m->d_err, 0, sizeof(int)));
    MCG_CUDA(cudaEventCreate(&m->ev0));
    MCG_CUDA(cudaEventCreate(&m->ev1));
    // He-style initialisation from a seeded host generator
    std::vector<float> p(kParams, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (int i = 0; i < kIn * kHid; ++i) p[kOffW1 + i] = nd(rng) * std::sqrt(2.f / kIn);
    for (int i = 0; i < kHid * kHid; ++i) p[kOffW2 + i] = nd(rng) * std::sqrt(2.f / kHid);
    for (int i = 0; i < kHid; ++i) p[kOffW3 + i] = nd(rng) * std::sqrt(1.f / kHid);
    MCG_CUDA(cudaMemcpy(m->d_params, p.data(), kParams * sizeof(float), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemset(m->d_m, 0, kParams * sizeof(float)));
    MCG_CUDA(cudaMemset(m->d_v, 0, kParams * sizeof(float)));
    mcg_status st = pack(m.get());
    if (st != MCG_OK) return st;
    MCG_CUDA(cudaStreamSynchronize(m->stream));
    *out = m.release();
    return MCG_OK;
}

mcg_status mcg_mlp_destroy(mcg_mlp *m) {
    mcg::clear_error();
    if (!m) return MCG_OK;
    cudaSetDevice(m->device);
    cudaStreamSynchronize(m->stream);
    cudaFree(m->d_params);
    cudaFree(m->d_grad);
    cudaFree(m->d_m);
    cudaFree(m->d_v);
    cudaFree(m->d_loss);
    cudaFree(m->d_pack);
    cudaFree(m->d_feat);
    cudaFree(m->d_tgt);
    cudaFree(m->d_w);
    cudaFree(m->d_q);
    cudaFree(m->d_partial);
    cudaFree(m->d_err);
    if (m->ev0) cudaEventDestroy(m->ev0);
    if (m->ev1) cudaEventDestroy(m->ev1);
    cudaStreamDestroy(m->stream);
    delete m;
    return MCG_OK;
}

mcg_status mcg_mlp_set_params(mcg_mlp *m, const float *params) {
    mcg::clear_error();
    if (!m || !params) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    MCG_CUDA(cudaSetDevice(m->device));
    MCG_CUDA(cudaMemcpyAsync(m->d_params, params, kParams * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MCG_CUDA(cudaMemsetAsync(m->d_m, 0, kParams * sizeof(float), m->stream));
    MCG_CUDA(cudaMemsetAsync(m->d_v, 0, kParams * sizeof(float), m->stream));
    m->adam_t = 0;
    mcg_status st = pack(m);
    if (st != MCG_OK) return st;
    MCG_CUDA(cudaStreamSynchronize(m->stream));
    return MCG_OK;
}

mcg_status mcg_mlp_get_params(mcg_mlp *m, float *params) {
    mcg::clear_error();
    if (!m || !params) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    MCG_CUDA(cudaSetDevice(m->device));
    MCG_CUDA(cudaMemcpyAsync(params, m->d_params, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCG_CUDA(cudaStreamSynchronize(m->stream));
    return MCG_OK;
}

mcg_status mcg_mlp_forward(mcg_mlp *m, const float *features, uint32_t n, float *q_out) {
    mcg::clear_error();
    if (!m || !features || !q_out) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (n == 0) return MCG_OK;
    MCG_CUDA(cudaSetDevice(m->device));
    float inv = 0.f;
    mcg_status st = upload_rows(m, features, nullptr, nullptr, n, inv);
    if (st != MCG_OK) return st;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    k_mlp_forward<<<std::min(tiles, m->ctas), kThreads, sizeof(TcSmem), m->stream>>>(m->d_pack, m->d_params,
                                                                                     m->d_feat, n, m->d_q, m->d_err);
    MCG_CUDA(cudaGetLastError());
    MCG_CUDA(cudaMemcpyAsync(q_out, m->d_q, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCG_CUDA(cudaStreamSynchronize(m->stream));
    return check_waits(m);
}

mcg_status mcg_mlp_grad(mcg_mlp *m, const float *features, const float *targets, const float *weights, uint32_t n,
                        float *grad_out, float *loss_out) {
    mcg::clear_error();
    if (!m || !features || !targets || !grad_out) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (n == 0) return mcg::fail(MCG_ERR_INVALID, "no rows");
    MCG_CUDA(cudaSetDevice(m->device));
    float inv = 0.f;
    mcg_status st = upload_rows(m, features, targets, weights, n, inv);
    if (st != MCG_OK) return st;
    st = grad_pass(m, n, inv, weights != nullptr);
    if (st != MCG_OK) return st;
    MCG_CUDA(cudaMemcpyAsync(grad_out, m->d_grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    float loss = 0.f;
    MCG_CUDA(cudaMemcpyAsync(&loss, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCG_CUDA(cudaStreamSynchronize(m->stream));
    st = check_waits(m);
    if (st != MCG_OK) return st;
    if (loss_out) *loss_out = loss;
    return MCG_OK;
}

mcg_status mcg_mlp_train(mcg_mlp *m, const float *features, const float *targets, const float *weights, uint32_t n,
                         uint32_t steps, float lr, float *loss_out) {
    mcg::clear_error();
    if (!m || !features || !targets) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (n == 0) return mcg::fail(MCG_ERR_INVALID, "no rows");
    MCG_CUDA(cudaSetDevice(m->device));
    float inv = 0.f;
    mcg_status st = upload_rows(m, features, targets, weights, n, inv);
    if (st != MCG_OK) return st;
    MCG_CUDA(cudaEventRecord(m->ev0, m->stream));
    for (uint32_t s = 0; s < steps; ++s) {
        st = grad_pass(m, n, inv, weights != nullptr);
        if (st != MCG_OK) return st;
        ++m->adam_t;
        const float b1c = 1.f - std::pow(0.9f, (float)m->adam_t);
        const float b2c = 1.f - std::pow(0.999f, (float)m->adam_t);
        k_adam<<<(kParams + 255) / 256, 256, 0, m->stream>>>(m->d_params, m->d_grad, m->d_m, m->d_v, lr, b1c, b2c);
        st = pack(m);
        if (st != MCG_OK) return st;
    }
    MCG_CUDA(cudaGetLastError());
    MCG_CUDA(cudaEventRecord(m->ev1, m->stream));
    float loss = 0.f;
    MCG_CUDA(cudaMemcpyAsync(&loss, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCG_CUDA(cudaStreamSynchronize(m->stream));
    float ms = 0.f;
    MCG_CUDA(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
    m->train_ms = ms;
    st = check_waits(m);
    if (st != MCG_OK) return st;
    if (loss_out) *loss_out = loss;
    return MCG_OK;
}

mcg_status mcg_mlp_train_time(mcg_mlp *m, double *ms) {
    mcg::clear_error();
    if (!m || !ms) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    *ms = m->train_ms;
    return MCG_OK;
}

}  // extern "C"
