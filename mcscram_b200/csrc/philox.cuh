// philox.cuh -- Philox4x32-10 Bernoulli word sampler for sm_100a.
//
// Bit-exact with the reference sampler (mcSCRAM src/mc/prng/philox128.h:8-88,
// counter layout src/mc/kernel/basic_event.h:112-122):
//   counter = {pdag_idx+1, event_idx+1, sample_idx+1, ((iteration+1) << 6) + g},
//   key     = {382307844, 293830103} (fixed, bumped by {0x9E3779B9, 0xBB67AE85}),
//   bit (4g + j) of the word = (uint64)out_j < threshold, g = 0..15.
//
// The 16 Philox calls of one word differ only in counter word 3 (by g), so
// part of the first three rounds is common to all 16 calls and is computed
// once per word here:
//   round 1: both products (M0*x0 depends on the event, M1*x2 on the word),
//   round 2: the M0 product (its operand x0' does not depend on g),
//   round 3: the M1 product (its operand x2'' does not depend on g).
// That leaves 16*16 + 3 = 259 32x32->64 multiplies per word instead of 320,
// with identical results.  The key schedule is folded into immediates.
#pragma once
#include <cstdint>

namespace mcg {
namespace dev {

constexpr uint32_t kM0 = 0xD2511F53u;
constexpr uint32_t kM1 = 0xCD9E8D57u;
constexpr uint32_t kW0 = 0x9E3779B9u;
constexpr uint32_t kW1 = 0xBB67AE85u;
constexpr uint32_t kKey0 = 382307844u;
constexpr uint32_t kKey1 = 293830103u;

template <int R>
struct RoundKey {
    static constexpr uint32_t k0 = kKey0 + (uint32_t)R * kW0;
    static constexpr uint32_t k1 = kKey1 + (uint32_t)R * kW1;
};

// 32x32 -> 64-bit product split into halves.
template <int MulForm>
__device__ __forceinline__ void mul_hilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
    if constexpr (MulForm == 0) {
        const uint64_t p = (uint64_t)a * (uint64_t)b;
        hi = (uint32_t)(p >> 32);
        lo = (uint32_t)p;
    } else {
        hi = __umulhi(a, b);
        lo = a * b;
    }
}

// Standard round r on the full state (rounds 4..10 of every call).
template <int R, int MulForm>
__device__ __forceinline__ void philox_round(uint32_t &x0, uint32_t &x1, uint32_t &x2, uint32_t &x3) {
    uint32_t ha, la, hb, lb;
    mul_hilo<MulForm>(kM0, x0, ha, la);
    mul_hilo<MulForm>(kM1, x2, hb, lb);
    x0 = hb ^ x1 ^ RoundKey<R>::k0;
    x1 = lb;
    x2 = ha ^ x3 ^ RoundKey<R>::k1;
    x3 = la;
}

// Per-word constant: product of M1 with counter word 2 = sample_idx + 1.
struct WordCtx {
    uint32_t hb, lb;
};

template <int MulForm>
__device__ __forceinline__ WordCtx make_word_ctx(uint32_t sample_idx) {
    WordCtx c;
    mul_hilo<MulForm>(kM1, sample_idx + 1u, c.hb, c.lb);
    return c;
}

// Packs the comparison of four outputs against thr into a nibble.
__device__ __forceinline__ uint32_t nibble_lt(uint32_t o0, uint32_t o1, uint32_t o2, uint32_t o3,
                                              uint32_t thr) {
    return (uint32_t)(o0 < thr) | ((uint32_t)(o1 < thr) << 1) | ((uint32_t)(o2 < thr) << 2) |
           ((uint32_t)(o3 < thr) << 3);
}

// Shifts the "out >= thr" flag into acc from the right: acc = 2*acc + (o >= thr).
// The carry of (o - thr) is exactly that flag; both instructions sit in one
// asm block so the carry does not have to survive between statements.
__device__ __forceinline__ uint32_t shift_in_ge(uint32_t acc, uint32_t o, uint32_t thr) {
    asm("{\n\t.reg .u32 t;\n\tsub.cc.u32 t, %1, %2;\n\taddc.u32 %0, %0, %0;\n\t}" : "+r"(acc) : "r"(o), "r"(thr));
    return acc;
}

// One 64-bit word of Bernoulli draws.
//   x0 = pdag_idx + 1, x1 = event_idx + 1, ctx from sample_idx,
//   t3 = (iteration + 1) << 6, thr = threshold in [1, 2^32 - 1]
//   (thresholds 0 and 2^32 give constant words and are handled by callers).
// PackForm 0: compare-and-or nibbles; PackForm 1: carry-chain shift-in.
// be_words gives K such words from one set of Philox outputs: word k
// compares every output with thr[k] (each in [1, 2^32 - 1]), so out[k] is
// the word be_word gives for that threshold.  Instances that share a counter
// stream but not their thresholds (draws of one tree) pay for the 16 Philox
// calls once.
template <int MulForm, int PackForm, int K>
__device__ __forceinline__ void be_words(uint32_t x0, uint32_t x1, const WordCtx &ctx, uint32_t t3,
                                         const uint32_t (&thr)[K], uint64_t (&out)[K]) {
    // Round 1, shared by the 16 calls.
    uint32_t ha, la;
    mul_hilo<MulForm>(kM0, x0, ha, la);
    const uint32_t a0 = ctx.hb ^ x1 ^ RoundKey<0>::k0;
    const uint32_t a1 = ctx.lb;
    const uint32_t a2base = ha ^ t3 ^ RoundKey<0>::k1;  // x3 = t3 + g == t3 ^ g (g < 64)
    const uint32_t a3 = la;
    // Round 2: the M0 product is shared.
    uint32_t hc, lc;
    mul_hilo<MulForm>(kM0, a0, hc, lc);
    const uint32_t b2 = hc ^ a3 ^ RoundKey<1>::k1;
    const uint32_t b3 = lc;
    // Round 3: the M1 product is shared.
    uint32_t hf, lf;
    mul_hilo<MulForm>(kM1, b2, hf, lf);
    const uint32_t c1 = lf;

    uint32_t lo[K], hi[K];
#pragma unroll
    for (int k = 0; k < K; ++k) lo[k] = hi[k] = 0;
#pragma unroll
    for (int g = 0; g < 16; ++g) {
        // Round 2, per call.
        uint32_t hd, ld;
        mul_hilo<MulForm>(kM1, a2base ^ (uint32_t)g, hd, ld);
        const uint32_t b0 = hd ^ a1 ^ RoundKey<1>::k0;
        const uint32_t b1 = ld;
        // Round 3, per call.
        uint32_t he, le;
        mul_hilo<MulForm>(kM0, b0, he, le);
        uint32_t x0r = hf ^ b1 ^ RoundKey<2>::k0;
        uint32_t x1r = c1;
        uint32_t x2r = he ^ b3 ^ RoundKey<2>::k1;
        uint32_t x3r = le;
        philox_round<3, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<4, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<5, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<6, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<7, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<8, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<9, MulForm>(x0r, x1r, x2r, x3r);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if constexpr (PackForm == 0) {
                const uint32_t nib = nibble_lt(x0r, x1r, x2r, x3r, thr[k]);
                if (g < 8) lo[k] |= nib << (4 * g);
                else hi[k] |= nib << (4 * (g - 8));
            } else {
                // Each generation shifts four ">=" flags in from the right (x3
                // first), so generation g ends up at nibble 7 - (g % 8) of its half.
                if (g < 8) {
                    lo[k] = shift_in_ge(lo[k], x3r, thr[k]);
                    lo[k] = shift_in_ge(lo[k], x2r, thr[k]);
                    lo[k] = shift_in_ge(lo[k], x1r, thr[k]);
                    lo[k] = shift_in_ge(lo[k], x0r, thr[k]);
                } else {
                    hi[k] = shift_in_ge(hi[k], x3r, thr[k]);
                    hi[k] = shift_in_ge(hi[k], x2r, thr[k]);
                    hi[k] = shift_in_ge(hi[k], x1r, thr[k]);
                    hi[k] = shift_in_ge(hi[k], x0r, thr[k]);
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if constexpr (PackForm == 0) {
            out[k] = ((uint64_t)hi[k] << 32) | (uint64_t)lo[k];
        } else {
            // The shift-in order put generation g at nibble (7 - g) of its half
            // and stored ">=": reverse nibble order and complement.
            auto rev_nibbles = [](uint32_t v) -> uint32_t {
                v = ((v & 0x0F0F0F0Fu) << 4) | ((v >> 4) & 0x0F0F0F0Fu);
                return __byte_perm(v, 0, 0x0123);
            };
            out[k] = ((uint64_t)(~rev_nibbles(hi[k])) << 32) | (uint64_t)(~rev_nibbles(lo[k]));
        }
    }
}

template <int MulForm, int PackForm>
__device__ __forceinline__ uint64_t be_word(uint32_t x0, uint32_t x1, const WordCtx &ctx, uint32_t t3,
                                            uint32_t thr) {
    const uint32_t t[1] = {thr};
    uint64_t w[1];
    be_words<MulForm, PackForm, 1>(x0, x1, ctx, t3, t, w);
    return w[0];
}

// ---------------------------------------------------------------------------
// Per-pass event table.  For a fixed event and pass, the round-2 product
// M1 * x2' (x2' = hi(M0 * x0) ^ ((iteration + 1) << 6 | g) ^ key1) depends on
// the generation g but not on the sample word, and lo(M0 * x0) is a per-event
// constant; tabulating them once per pass removes 17 of the 259 multiplies of
// every word.  Layout: 17 uint2 per event, [g] = {hi, lo} of M1 * x2'_g for
// g = 0..15, [16] = {lo(M0 * x0), hi(M0 * x0)}.
constexpr int kEventTableStride = 17;

template <int MulForm>
__device__ __forceinline__ void event_table_entry(uint32_t x0, uint32_t t3, int g, uint2 &out) {
    uint32_t ha, la;
    mul_hilo<MulForm>(kM0, x0, ha, la);
    if (g < 16) {
        const uint32_t a2 = ha ^ t3 ^ RoundKey<0>::k1 ^ (uint32_t)g;
        uint32_t hd, ld;
        mul_hilo<MulForm>(kM1, a2, hd, ld);
        out = make_uint2(hd, ld);
    } else {
        out = make_uint2(la, ha);
    }
}

// be_word with the per-pass event table (same result as be_word).
template <int MulForm, int PackForm>
__device__ __forceinline__ uint64_t be_word_tab(uint32_t x1, const WordCtx &ctx, const uint2 *__restrict__ tab,
                                                uint32_t thr) {
    const uint32_t a0 = ctx.hb ^ x1 ^ RoundKey<0>::k0;
    const uint32_t a1 = ctx.lb;
    const uint32_t a3 = __ldg(&tab[16].x);
    uint32_t hc, lc;
    mul_hilo<MulForm>(kM0, a0, hc, lc);
    const uint32_t b2 = hc ^ a3 ^ RoundKey<1>::k1;
    const uint32_t b3 = lc;
    uint32_t hf, lf;
    mul_hilo<MulForm>(kM1, b2, hf, lf);
    const uint32_t c1 = lf;
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int g = 0; g < 16; ++g) {
        const uint2 d = __ldg(&tab[g]);
        const uint32_t b0 = d.x ^ a1 ^ RoundKey<1>::k0;
        const uint32_t b1 = d.y;
        uint32_t he, le;
        mul_hilo<MulForm>(kM0, b0, he, le);
        uint32_t x0r = hf ^ b1 ^ RoundKey<2>::k0;
        uint32_t x1r = c1;
        uint32_t x2r = he ^ b3 ^ RoundKey<2>::k1;
        uint32_t x3r = le;
        philox_round<3, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<4, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<5, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<6, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<7, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<8, MulForm>(x0r, x1r, x2r, x3r);
        philox_round<9, MulForm>(x0r, x1r, x2r, x3r);
        if constexpr (PackForm == 0) {
            const uint32_t nib = nibble_lt(x0r, x1r, x2r, x3r, thr);
            if (g < 8) lo |= nib << (4 * g);
            else hi |= nib << (4 * (g - 8));
        } else {
            if (g < 8) {
                lo = shift_in_ge(lo, x3r, thr);
                lo = shift_in_ge(lo, x2r, thr);
                lo = shift_in_ge(lo, x1r, thr);
                lo = shift_in_ge(lo, x0r, thr);
            } else {
                hi = shift_in_ge(hi, x3r, thr);
                hi = shift_in_ge(hi, x2r, thr);
                hi = shift_in_ge(hi, x1r, thr);
                hi = shift_in_ge(hi, x0r, thr);
            }
        }
    }
    if constexpr (PackForm == 0) {
        return ((uint64_t)hi << 32) | (uint64_t)lo;
    } else {
        auto rev_nibbles = [](uint32_t v) -> uint32_t {
            v = ((v & 0x0F0F0F0Fu) << 4) | ((v >> 4) & 0x0F0F0F0Fu);
            return __byte_perm(v, 0, 0x0123);
        };
        return ((uint64_t)(~rev_nibbles(hi)) << 32) | (uint64_t)(~rev_nibbles(lo));
    }
}

}  // namespace dev
}  // namespace mcg
