// mlp.cu -- the importance-sampling proposal network (include/mcg_is.h).
//
// 16 features -> 64 -> 64 -> 1, ReLU, sigmoid.  Dense products run on the
// tensor cores with mma.sync.m16n8k16 (BF16 operands, FP32 accumulation);
// the rank-1 and elementwise steps on CUDA cores.  A CTA of 4 warps works on
// 64 rows at a time: warp w the rows 16w .. 16w+15 for the row-wise products,
// and an output-tile slice of the weight gradients (a reduction over the
// rows).  The gradient kernel is persistent: each CTA walks 64-row tiles
// with its gradient slices held in the MMA accumulators and registers,
// writes one partial gradient at the end, and a second kernel sums the
// partials in CTA order (deterministic, no atomics on global memory).
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
constexpr int kRows = 64;             // rows per CTA
constexpr int kThreads = 128;         // 4 warps
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

// Packed BF16 operands: W1t[64][16], W2t[64][64] (out-major), W2[64][64]
// (in-major), W3t[8][64] (row 0 = W3, rows 1..7 zero).
constexpr int kPackW1t = 0;
constexpr int kPackW2t = kPackW1t + kHid * kIn;
constexpr int kPackW2 = kPackW2t + kHid * kHid;
constexpr int kPackW3t = kPackW2 + kHid * kHid;
constexpr int kPackSize = kPackW3t + 8 * kHid;

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Row strides (in BF16 elements) of the shared-memory tiles: 16-wide rows
// padded to 24 (48 B) and 64-wide rows to 72 (144 B).  Rows stay 16-byte
// aligned for ldmatrix, and a fragment's eight rows start on eight
// different bank groups, so neither the fragment loads below nor ldmatrix
// conflict (with 64-element rows every row would start on the same bank).
constexpr int kLdX = 24;
constexpr int kLd = 72;

// A fragment of the 16x16 tile at rows m0.., cols k0.. of row-major A (lda).
__device__ __forceinline__ void frag_a(uint32_t a[4], const bf16 *A, int lda, int m0, int k0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    a[0] = *reinterpret_cast<const uint32_t *>(&A[(m0 + g) * lda + k0 + 2 * t]);
    a[1] = *reinterpret_cast<const uint32_t *>(&A[(m0 + g + 8) * lda + k0 + 2 * t]);
    a[2] = *reinterpret_cast<const uint32_t *>(&A[(m0 + g) * lda + k0 + 2 * t + 8]);
    a[3] = *reinterpret_cast<const uint32_t *>(&A[(m0 + g + 8) * lda + k0 + 2 * t + 8]);
}

// B fragment of the 16x8 tile (k0.., n0..) of B given as Bt[n][k] (ldb).
__device__ __forceinline__ void frag_b(uint32_t b[2], const bf16 *Bt, int ldb, int n0, int k0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    b[0] = *reinterpret_cast<const uint32_t *>(&Bt[(n0 + g) * ldb + k0 + 2 * t]);
    b[1] = *reinterpret_cast<const uint32_t *>(&Bt[(n0 + g) * ldb + k0 + 2 * t + 8]);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// ldmatrix with transposition: 8x8 BF16 tiles whose rows lanes 8j .. 8j + 7
// address (tile j); each lane receives the tiles' elements in the layout of
// the transposed tiles' mma fragments.
__device__ __forceinline__ void ldsm_x4_trans(uint32_t r[4], const bf16 *row) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(row)));
}

__device__ __forceinline__ void ldsm_x2_trans(uint32_t r[2], const bf16 *row) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_addr(row)));
}

// A fragment of the 16x16 tile (m0.., k0..) of A = M^T for M stored
// row-major as M[k][m] (ldm): the tiles (k0, m0), (k0, m0 + 8), (k0 + 8, m0),
// (k0 + 8, m0 + 8) of M, transposed, are a[0] .. a[3].
__device__ __forceinline__ void frag_a_t(uint32_t a[4], const bf16 *M, int ldm, int m0, int k0, int lane) {
    const int tile = lane >> 3, row = lane & 7;
    ldsm_x4_trans(a, M + (k0 + row + ((tile & 2) ? 8 : 0)) * ldm + m0 + ((tile & 1) ? 8 : 0));
}

// B fragment of the 16x8 tile (k0.., n0..) of B stored row-major as B[k][n]
// (ldb): the tiles (k0, n0) and (k0 + 8, n0) of B, transposed.
__device__ __forceinline__ void frag_b_t(uint32_t b[2], const bf16 *B, int ldb, int n0, int k0, int lane) {
    const int tile = (lane >> 3) & 1, row = lane & 7;
    ldsm_x2_trans(b, B + (k0 + row + 8 * tile) * ldb + n0);
}

// ReLU masks are read back from the BF16 activations (h > 0); a positive
// pre-activation rounds to a positive BF16 value unless it is below the
// smallest BF16 subnormal's half.
struct Smem {
    bf16 w1[kIn * kLd];       // W1[in][out]
    bf16 w2[kHid * kLd];      // W2[in][out]
    bf16 w3t[8 * kLd];        // row 0 = W3
    bf16 x[kRows * kLdX];     // the tile's features, row-major
    bf16 h1[kRows * kLd];     // post-ReLU activations, row-major
    bf16 h2[kRows * kLd];
    bf16 dh2[kRows * kLd];    // gradients of the pre-activations, row-major
    bf16 dh1[kRows * kLd];
    float b1[kHid], b2[kHid], w3[kHid];
    float dz[kRows];
    float loss;
};

__device__ __forceinline__ bool relu_on(bf16 h) { return __bfloat162float(h) > 0.f; }

// Forward for the CTA's rows; writes h1/h2 and the masks and returns z for
// row r (valid in lanes with (lane & 3) == 0: rows g and g + 8).
__device__ void forward_rows(Smem &s, int warp, int lane, float b3, float z_out[2]) {
    const int m0 = warp * 16;
    const int g = lane >> 2, t = lane & 3;
    // layer 1: [16 x 16] x [16 x 64]
    {
        uint32_t a[4];
        frag_a(a, s.x, kLdX, m0, 0, lane);
#pragma unroll
        for (int nt = 0; nt < kHid / 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            uint32_t b[2];
            frag_b_t(b, s.w1, kLd, nt * 8, 0, lane);
            mma16816(c, a, b);
            const int col = nt * 8 + 2 * t;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = m0 + g + (j >= 2 ? 8 : 0), cc = col + (j & 1);
                const float v = c[j] + s.b1[cc];
                s.h1[r * kLd + cc] = __float2bfloat16(v > 0.f ? v : 0.f);
            }
        }
    }
    __syncwarp();
    // layer 2: [16 x 64] x [64 x 64]
#pragma unroll
    for (int nt = 0; nt < kHid / 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < kHid / 16; ++kt) {
            uint32_t a[4], b[2];
            frag_a(a, s.h1, kLd, m0, kt * 16, lane);
            frag_b_t(b, s.w2, kLd, nt * 8, kt * 16, lane);
            mma16816(c, a, b);
        }
        const int col = nt * 8 + 2 * t;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = m0 + g + (j >= 2 ? 8 : 0), cc = col + (j & 1);
            const float v = c[j] + s.b2[cc];
            s.h2[r * kLd + cc] = __float2bfloat16(v > 0.f ? v : 0.f);
        }
    }
    __syncwarp();
    // output: [16 x 64] x [64 x 8] (column 0 is W3)
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kt = 0; kt < kHid / 16; ++kt) {
        uint32_t a[4], b[2];
        frag_a(a, s.h2, kLd, m0, kt * 16, lane);
        frag_b(b, s.w3t, kLd, 0, kt * 16, lane);
        mma16816(c, a, b);
    }
    z_out[0] = c[0] + b3;  // row m0 + g, column 0 when t == 0
    z_out[1] = c[2] + b3;  // row m0 + g + 8
}

__device__ void load_weights(Smem &s, const bf16 *__restrict__ pack, const float *__restrict__ params) {
    for (int i = threadIdx.x; i < kIn * kHid; i += kThreads) {  // W1[f][h] = W1t[h][f]
        const int f = i / kHid, h = i % kHid;
        s.w1[f * kLd + h] = pack[kPackW1t + h * kIn + f];
    }
    for (int i = threadIdx.x; i < kHid * kHid; i += kThreads) s.w2[(i / kHid) * kLd + i % kHid] = pack[kPackW2 + i];
    for (int i = threadIdx.x; i < 8 * kHid; i += kThreads) s.w3t[(i / kHid) * kLd + i % kHid] = pack[kPackW3t + i];
    for (int i = threadIdx.x; i < kHid; i += kThreads) {
        s.b1[i] = params[kOffB1 + i];
        s.b2[i] = params[kOffB2 + i];
        s.w3[i] = params[kOffW3 + i];
    }
}

// The tile's rows as BF16; rows past n are 0.
__device__ void load_rows(Smem &s, const float *__restrict__ feat, uint32_t n, uint32_t row0) {
    for (int i = threadIdx.x; i < kRows * kIn; i += kThreads) {
        const int r = i / kIn, f = i % kIn;
        const float v = (row0 + r < n) ? feat[(uint64_t)(row0 + r) * kIn + f] : 0.f;
        s.x[r * kLdX + f] = __float2bfloat16(v);
    }
}

__device__ void load_tile(Smem &s, const bf16 *__restrict__ pack, const float *__restrict__ params,
                          const float *__restrict__ feat, uint32_t n, uint32_t row0) {
    load_weights(s, pack, params);
    load_rows(s, feat, n, row0);
    if (threadIdx.x == 0) s.loss = 0.f;
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads) k_mlp_forward(const bf16 *__restrict__ pack, const float *__restrict__ params,
                                                          const float *__restrict__ feat, uint32_t n,
                                                          float *__restrict__ q) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem &s = *reinterpret_cast<Smem *>(smem_raw);
    const uint32_t row0 = blockIdx.x * kRows;
    load_tile(s, pack, params, feat, n, row0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float z[2];
    forward_rows(s, warp, lane, params[kOffB3], z);
    if ((lane & 3) == 0) {
        const int g = lane >> 2;
        const uint32_t r0 = row0 + warp * 16 + g, r1 = r0 + 8;
        if (r0 < n) q[r0] = 1.f / (1.f + __expf(-z[0]));
        if (r1 < n) q[r1] = 1.f / (1.f + __expf(-z[1]));
    }
}

// Weighted BCE gradient of the rows [0, n): persistent CTAs, CTA b taking
// tiles b, b + gridDim.x, ...; its gradient (kParams floats, then the loss)
// goes to partial[b * (kParams + 1) ..] (every entry written once).
__global__ void __launch_bounds__(kThreads) k_mlp_grad(const bf16 *__restrict__ pack, const float *__restrict__ params,
                                                       const float *__restrict__ feat, const float *__restrict__ tgt,
                                                       const float *__restrict__ wts, float inv_wsum, uint32_t n,
                                                       float *__restrict__ partial) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem &s = *reinterpret_cast<Smem *>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = warp * 16;
    load_weights(s, pack, params);
    if (threadIdx.x == 0) s.loss = 0.f;
    const float b3 = params[kOffB3];
    // this CTA's gradient: dW2 rows m0 .. m0 + 15 and dW1 n-tiles 2w, 2w + 1 in
    // MMA accumulators; W3, b2, b1 (threads c < 64) and b3 (thread 64) in registers
    float acc2[kHid / 8][4], acc1[2][4];
#pragma unroll
    for (int nt = 0; nt < kHid / 8; ++nt)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc2[nt][j] = 0.f;
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc1[q][j] = 0.f;
    float gw3 = 0.f, gb2 = 0.f, gb1 = 0.f, gb3 = 0.f;
    const uint32_t tiles = (n + kRows - 1) / kRows;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t row0 = tile * kRows;
        load_rows(s, feat, n, row0);
        __syncthreads();
        float z[2];
        forward_rows(s, warp, lane, b3, z);
        // dL/dz = w (q - t) / sum w for the tile's rows
        if (t == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int rl = m0 + g + 8 * h;
                const uint32_t r = row0 + rl;
                float d = 0.f;
                if (r < n) {
                    const float qv = 1.f / (1.f + __expf(-z[h]));
                    const float tv = tgt[r];
                    const float wv = (wts ? wts[r] : 1.f) * inv_wsum;
                    d = wv * (qv - tv);
                    const float qc = fminf(fmaxf(qv, 1e-7f), 1.f - 1e-7f);
                    atomicAdd(&s.loss, -wv * (tv * __logf(qc) + (1.f - tv) * __logf(1.f - qc)));
                }
                s.dz[rl] = d;
            }
        }
        __syncthreads();
        // dH2 = dz W3^T masked
        for (int i = threadIdx.x; i < kRows * kHid; i += kThreads) {
            const int r = i / kHid, c = i % kHid;
            s.dh2[r * kLd + c] = __float2bfloat16(relu_on(s.h2[r * kLd + c]) ? s.dz[r] * s.w3[c] : 0.f);
        }
        __syncthreads();
        if (threadIdx.x < kHid) {
            const int c = threadIdx.x;
            for (int r = 0; r < kRows; ++r) {
                gw3 += __bfloat162float(s.h2[r * kLd + c]) * s.dz[r];
                gb2 += relu_on(s.h2[r * kLd + c]) ? s.dz[r] * s.w3[c] : 0.f;
            }
        } else if (threadIdx.x == kHid) {
            for (int r = 0; r < kRows; ++r) gb3 += s.dz[r];
        }
        // dW2[in][out] += H1^T dH2: M = 64 (in), N = 64 (out), K = 64 rows; warp w: in rows 16w..
#pragma unroll
        for (int kt = 0; kt < kRows / 16; ++kt) {
            uint32_t a[4];
            frag_a_t(a, s.h1, kLd, m0, kt * 16, lane);
#pragma unroll
            for (int nt = 0; nt < kHid / 8; ++nt) {
                uint32_t b[2];
                frag_b_t(b, s.dh2, kLd, nt * 8, kt * 16, lane);
                mma16816(acc2[nt], a, b);
            }
        }
        // dH1 = dH2 W2^T masked: [16 rows x 64 out] x [64 out x 64 in]; B = W2 (in-major) as Bt[in][out]
#pragma unroll
        for (int nt = 0; nt < kHid / 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < kHid / 16; ++kt) {
                uint32_t a[4], b[2];
                frag_a(a, s.dh2, kLd, m0, kt * 16, lane);
                frag_b(b, s.w2, kLd, nt * 8, kt * 16, lane);
                mma16816(c, a, b);
            }
            const int col = nt * 8 + 2 * t;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int r = m0 + g + (j >= 2 ? 8 : 0), cc = col + (j & 1);
                s.dh1[r * kLd + cc] = __float2bfloat16(relu_on(s.h1[r * kLd + cc]) ? c[j] : 0.f);
            }
        }
        __syncthreads();
        // db1 and dW1[f][h] += X^T dH1: M = 16 (features), N = 64, K = 64 rows; warp w: n-tiles 2w, 2w+1
        if (threadIdx.x < kHid) {
            const int c = threadIdx.x;
            for (int r = 0; r < kRows; ++r) gb1 += __bfloat162float(s.dh1[r * kLd + c]);
        }
#pragma unroll
        for (int kt = 0; kt < kRows / 16; ++kt) {
            uint32_t a[4];
            frag_a_t(a, s.x, kLdX, 0, kt * 16, lane);
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                uint32_t b[2];
                frag_b_t(b, s.dh1, kLd, (warp * 2 + q) * 8, kt * 16, lane);
                mma16816(acc1[q], a, b);
            }
        }
        __syncthreads();  // the next tile overwrites the rows and activations
    }
    float *out = partial + (uint64_t)blockIdx.x * (kParams + 1);
#pragma unroll
    for (int nt = 0; nt < kHid / 8; ++nt) {
        const int col = nt * 8 + 2 * t;
        out[kOffW2 + (m0 + g) * kHid + col] = acc2[nt][0];
        out[kOffW2 + (m0 + g) * kHid + col + 1] = acc2[nt][1];
        out[kOffW2 + (m0 + g + 8) * kHid + col] = acc2[nt][2];
        out[kOffW2 + (m0 + g + 8) * kHid + col + 1] = acc2[nt][3];
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int col = (warp * 2 + q) * 8 + 2 * t;
        out[kOffW1 + g * kHid + col] = acc1[q][0];
        out[kOffW1 + g * kHid + col + 1] = acc1[q][1];
        out[kOffW1 + (g + 8) * kHid + col] = acc1[q][2];
        out[kOffW1 + (g + 8) * kHid + col + 1] = acc1[q][3];
    }
    if (threadIdx.x < kHid) {
        out[kOffW3 + threadIdx.x] = gw3;
        out[kOffB2 + threadIdx.x] = gb2;
        out[kOffB1 + threadIdx.x] = gb1;
    } else if (threadIdx.x == kHid) {
        out[kOffB3] = gb3;
        out[kParams] = s.loss;
    }
}

// grad[i] = sum over the CTAs of partial[b][i] in CTA order (i = kParams: the loss).
__global__ void k_mlp_reduce(const float *__restrict__ partial, uint32_t blocks, float *__restrict__ grad,
                             float *__restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > kParams) return;
    float v = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) v += partial[(uint64_t)b * (kParams + 1) + i];
    if (i < kParams) grad[i] = v;
    else *loss = v;
}

// FP32 master weights -> BF16 operand copies.
__global__ void k_mlp_pack(const float *__restrict__ p, bf16 *__restrict__ pack) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kPackSize; i += gridDim.x * blockDim.x) {
        float v = 0.f;
        if (i < kPackW2t) {  // W1t[h][f] = W1[f][h]
            const int h = i / kIn, f = i % kIn;
            v = p[kOffW1 + f * kHid + h];
        } else if (i < kPackW2) {  // W2t[o][in] = W2[in][o]
            const int j = i - kPackW2t, o = j / kHid, in = j % kHid;
            v = p[kOffW2 + in * kHid + o];
        } else if (i < kPackW3t) {  // W2[in][o]
            v = p[kOffW2 + (i - kPackW2)];
        } else {
            const int j = i - kPackW3t, row = j / kHid, col = j % kHid;
            v = row == 0 ? p[kOffW3 + col] : 0.f;
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
    float *d_partial = nullptr;  // [grad_ctas][kParams + 1] per-CTA gradients and losses
    uint32_t grad_ctas = 0;      // persistent CTAs of the gradient kernel
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

mcg_status pack(mcg_mlp *m) {
    k_mlp_pack<<<(kPackSize + 255) / 256, 256, 0, m->stream>>>(m->d_params, m->d_pack);
    MCG_CUDA(cudaGetLastError());
    return MCG_OK;
}

// The gradient of the uploaded rows into d_grad and d_loss: the persistent
// gradient kernel, then the reduction of its partials.
mcg_status grad_pass(mcg_mlp *m, uint32_t n, float inv_wsum, bool has_w) {
    const uint32_t tiles = (n + kRows - 1) / kRows;
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>(tiles, m->grad_ctas));
    k_mlp_grad<<<blocks, kThreads, sizeof(Smem), m->stream>>>(m->d_pack, m->d_params, m->d_feat, m->d_tgt,
                                                             has_w ? m->d_w : nullptr, inv_wsum, n, m->d_partial);
    MCG_CUDA(cudaGetLastError());
    k_mlp_reduce<<<(kParams + 1 + 255) / 256, 256, 0, m->stream>>>(m->d_partial, blocks, m->d_grad, m->d_loss);
    MCG_CUDA(cudaGetLastError());
    return MCG_OK;
}

mcg_status upload_rows(mcg_mlp *m, const float *feat, const float *tgt, const float *w, uint32_t n, float &inv_wsum) {
    mcg_status st = ensure_rows(m, n);
    if (st != MCG_OK) return st;
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
    MCG_CUDA(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)));
    MCG_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem)));
    int sms = 0, per_sm = 0;
    MCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    MCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mlp_grad, kThreads, sizeof(Smem)));
    m->grad_ctas = (uint32_t)std::max(1, sms * std::max(per_sm, 1));
    MCG_CUDA(cudaMalloc((void **)&m->d_partial, (size_t)m->grad_ctas * (kParams + 1) * sizeof(float)));
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
    k_mlp_forward<<<(n + kRows - 1) / kRows, kThreads, sizeof(Smem), m->stream>>>(m->d_pack, m->d_params, m->d_feat,
                                                                                 n, m->d_q);
    MCG_CUDA(cudaGetLastError());
    MCG_CUDA(cudaMemcpyAsync(q_out, m->d_q, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCG_CUDA(cudaStreamSynchronize(m->stream));
    return MCG_OK;
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
