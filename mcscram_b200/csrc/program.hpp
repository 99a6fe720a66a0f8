// program.hpp -- compiles a flattened PDAG into the fused kernel's program.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "graph.hpp"
#include "program_format.h"

namespace mcg {

struct Program {
    std::vector<Op> ops;         // ends with kOpHalt plus one padding op
    uint32_t smem_slots = 0;     // shared-memory slots actually used
    uint32_t global_slots = 0;   // global scratch slots actually used
    uint32_t max_live = 0;       // peak number of simultaneously live slot values
    uint32_t n_inline_be = 0;    // basic events sampled straight into their consumer
    uint32_t n_def_be = 0;       // basic events stored to a slot (shared or tallied)
    uint64_t n_be_sampled = 0;   // Philox words per sample column
    uint32_t n_gate_evals = 0;   // gates evaluated per sample column
};

// Builds the program.  Only nodes that some tallied node depends on are
// evaluated.  smem_slot_budget bounds the shared-memory slots; values that do
// not fit go to global scratch slots (linear-scan allocation that spills the
// live value with the furthest last use).
//
// With variable_thresholds the basic-event ops carry the event's node id in
// place of its threshold (w2), for kernels that read thresholds from a
// per-instance table, and no event is treated as a constant word.
std::string compile_program(const Graph &g, uint32_t smem_slot_budget, Program &out,
                            bool variable_thresholds = false);

}  // namespace mcg
