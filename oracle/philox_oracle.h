/*
 * oracle/philox_oracle.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Plain-C restatement of the reference's Philox4x32-10 Bernoulli sampler.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this; the product path (mcscram_b200) never includes or links it.
 *
 * Followed reference lines (paths inside the mcSCRAM project):
 *   src/mc/prng/state128.h:21-26   mulhilo: 32x32 -> 64-bit product split
 *   src/mc/prng/philox128.h:8-35   one round: M = {0xD2511F53, 0xCD9E8D57},
 *                                  W = {0x9E3779B9, 0xBB67AE85}
 *   src/mc/prng/philox128.h:37-54  generate: fixed key {382307844, 293830103},
 *                                  x3 += generation (uint8), 10 rounds
 *   src/mc/prng/philox128.h:59-74  sample: bit (4g+j) = (uint64)x_j < threshold
 *   src/mc/prng/philox128.h:76-88  pack_bernoulli_draws: 16 generations per word
 *   src/mc/kernel/basic_event.h:112-122  counter = {pdag_idx+1, event_idx+1,
 *                                  sample_idx+1, (iteration+1) << 6}
 *   src/mc/event/node.h:372-376    threshold = (uint64)(p * 2^32), truncated
 */
#ifndef MCG_ORACLE_PHILOX_H
#define MCG_ORACLE_PHILOX_H

#include <stdint.h>

#define ORC_KEY0 382307844u
#define ORC_KEY1 293830103u

static inline void orc_philox4x32_10(uint32_t x[4]) {
    uint32_t k0 = ORC_KEY0, k1 = ORC_KEY1;
    for (int r = 0; r < 10; ++r) {
        const uint64_t pa = (uint64_t)0xD2511F53u * (uint64_t)x[0];
        const uint64_t pb = (uint64_t)0xCD9E8D57u * (uint64_t)x[2];
        const uint32_t hi_a = (uint32_t)(pa >> 32), lo_a = (uint32_t)pa;
        const uint32_t hi_b = (uint32_t)(pb >> 32), lo_b = (uint32_t)pb;
        const uint32_t n0 = hi_b ^ x[1] ^ k0;
        const uint32_t n2 = hi_a ^ x[3] ^ k1;
        x[0] = n0;
        x[1] = lo_b;
        x[2] = n2;
        x[3] = lo_a;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

/* One 64-bit word of Bernoulli draws for counter base {c0, c1, c2, c3}. */
static inline uint64_t orc_pack_word(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                     uint64_t threshold) {
    uint64_t word = 0;
    for (uint32_t g = 0; g < 16; ++g) {
        uint32_t x[4] = {c0, c1, c2, c3 + (uint32_t)(uint8_t)g};
        orc_philox4x32_10(x);
        for (uint32_t j = 0; j < 4; ++j) {
            if ((uint64_t)x[j] < threshold) word |= (uint64_t)1 << (4u * g + j);
        }
    }
    return word;
}

/* Basic-event word: counter from (pdag_idx, event_idx, sample_idx, iteration). */
static inline uint64_t orc_be_word(uint32_t pdag_idx, uint32_t event_idx, uint32_t sample_idx,
                                   uint32_t iteration, uint64_t threshold) {
    return orc_pack_word(pdag_idx + 1u, event_idx + 1u, sample_idx + 1u,
                         (iteration + 1u) << 6, threshold);
}

/* threshold = (uint64)(p * 2^32), truncated toward zero. */
static inline uint64_t orc_threshold(double p) {
    return (uint64_t)(p * 4294967296.0);
}

#endif
