// compile_api.cpp -- host-only program compilation entry (mcg_compile).
#include <algorithm>
#include <cstring>

#include "error.hpp"
#include "graph.hpp"
#include "mcg.h"
#include "program.hpp"

extern "C" mcg_status mcg_compile(const mcg_graph_desc *graph, uint32_t smem_slot_budget, uint32_t flags,
                                  mcg_program_info *info, uint32_t *ops, uint64_t ops_capacity) {
    mcg::clear_error();
    if (!graph || !info) return mcg::fail(MCG_ERR_INVALID, "graph and info must not be NULL");
    mcg::Graph g;
    std::string err = mcg::Graph::from_desc(*graph, g);
    if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, err);
    mcg::Program prog;
    err = mcg::compile_program(g, smem_slot_budget, prog, (flags & MCG_COMPILE_VARIABLE_THRESHOLDS) != 0);
    if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, err);
    std::memset(info, 0, sizeof(*info));
    info->n_ops = prog.ops.size();
    info->smem_slots = prog.smem_slots;
    info->global_slots = prog.global_slots;
    info->max_live = prog.max_live;
    info->n_inline_be = prog.n_inline_be;
    if (ops) {
        const uint64_t n = std::min<uint64_t>(prog.ops.size(), ops_capacity);
        std::memcpy(ops, prog.ops.data(), n * sizeof(mcg::Op));
    }
    return MCG_OK;
}
