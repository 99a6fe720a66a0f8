// oracle/ref_philox_shim.cc -- TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own Philox sampler, compiled from its source tree
// (src/mc/prng/philox128.h, src/mc/prng/state128.h of mcSCRAM), behind one
// C symbol.  oracle/Makefile builds this into oracle/_ref/ only when the
// reference sources are present; nothing here is copied from them.
#include <cstdint>

#include "mc/prng/philox128.h"

extern "C" std::uint64_t ref_pack_word(std::uint32_t c0, std::uint32_t c1, std::uint32_t c2,
                                       std::uint32_t c3, std::uint64_t threshold) {
    const scram::mc::prng::state128 base = {{c0, c1, c2, c3}};
    return scram::mc::prng::philox::pack_bernoulli_draws<std::uint64_t>(base, threshold);
}
