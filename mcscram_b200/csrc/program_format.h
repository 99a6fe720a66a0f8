// program_format.h -- encoding of the fused kernel's node program.
//
// The host compiles a flattened PDAG into a linear program of 16-byte ops
// that every thread of the fused kernel interprets for its own sample word.
// All threads walk the same ops, so every branch on an op is warp-uniform.
//
// A gate is evaluated as BEGIN, one IN_* per input, END: an accumulator
// machine.  Basic events with a single consumer are sampled straight into the
// consumer's accumulator (IN_BE) and never stored; other values live in
// "slots": per-thread shared-memory cells, or per-thread columns of a global
// scratch array when shared memory runs out (a slot reference with
// kSlotGlobal set).
//
//   op        w0                                         w1          w2        w3
//   HALT      0
//   IN_BE     1 | neg<<7                                 pdag_idx+1  thr32     event_idx+1
//   BE_DEF    2 | slot_ref<<8                            pdag_idx+1  thr32     event_idx+1
//   BEGIN     3 | conn<<8 | k<<16 | nbits<<24
//   IN_SLOT   4 | neg<<7                                 slot_ref
//   IN_CONST  5 | neg<<7                                 lo          hi
//   END       6                                          slot_ref|kNoSlot
//   CONST_DEF 7 | slot_ref<<8                            lo          hi
//   TALLY     8                                          tally index
//
// BE_DEF / END / CONST_DEF leave their value in the interpreter's "last"
// register; a following TALLY counts its ones.  thr32 is the threshold for
// thresholds in [1, 2^32 - 1]; thresholds 0 and 2^32 give constant words
// (all zeros / all ones) and are compiled to IN_CONST / CONST_DEF.
#pragma once
#include <cstdint>

namespace mcg {

enum OpCode : uint32_t {
    kOpHalt = 0,
    kOpInBe = 1,
    kOpBeDef = 2,
    kOpBegin = 3,
    kOpInSlot = 4,
    kOpInConst = 5,
    kOpEnd = 6,
    kOpConstDef = 7,
    kOpTally = 8,
};

constexpr uint32_t kOpMask = 0xFu;
constexpr uint32_t kNegBit = 1u << 7;
constexpr uint32_t kSlotGlobal = 1u << 23;  // slot refs are 24-bit
constexpr uint32_t kSlotIndexMask = kSlotGlobal - 1u;
constexpr uint32_t kNoSlot = 0xFFFFFFu;

struct alignas(16) Op {
    uint32_t w[4];
};

}  // namespace mcg
