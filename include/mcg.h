/*
 * mcg.h -- C ABI of the B200 Monte Carlo fault-tree engine (libmcg.so).
 *
 * The engine replaces the device half of mcSCRAM's Monte Carlo probability
 * path: scram::mc::queue::layer_manager<uint64_t> (src/mc/queue/layer_manager.h:98-402)
 * with its kernels src/mc/kernel/{basic_event,gate,tally}.h and the Philox
 * sampler src/mc/prng/philox128.h.  Paths are inside the mcSCRAM project.
 *
 * Plain C types only: pointers, sizes, status codes.  Every function returns
 * an mcg_status; on failure mcg_last_error() returns a message for the
 * calling thread.  No function calls exit().  A handle is not thread safe:
 * one host thread drives one engine, on one CUDA stream.
 *
 * Graph layout ("flattened PDAG"):
 *   node ids [0, n_be) are basic events, [n_be, n_be + n_gates) are gates
 *   in a topological order: every input id of gate g is < n_be + g.
 *   Gate g reads inputs[in_begin[g] .. in_begin[g] + in_count[g]); the last
 *   neg_count[g] of those are complemented (the reference stores negated
 *   inputs after the positive ones, src/mc/event/node.h:655-662).
 */
#ifndef MCG_H
#define MCG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int mcg_status;
#define MCG_OK 0
#define MCG_ERR_INVALID 1   /* malformed arguments or graph (reference: std::exit / runtime_error) */
#define MCG_ERR_CUDA 2      /* CUDA runtime failure (reference: sycl::exception via wait_and_throw) */
#define MCG_ERR_OOM 3       /* device allocation failed */
#define MCG_ERR_TIMEOUT 4   /* a bounded device wait gave up */
#define MCG_ERR_STATE 5     /* call not valid in the handle's current state */
#define MCG_ERR_NO_DEVICE 6 /* no CUDA device visible */

/* Gate connectives, numbered like core::Connective (src/pdag.h:265-276). */
enum mcg_connective {
    MCG_AND = 0, MCG_OR = 1, MCG_ATLEAST = 2, MCG_XOR = 3,
    MCG_NOT = 4, MCG_NAND = 5, MCG_NOR = 6, MCG_NULL = 7
};

/* Evaluation strategies for mcg_run. */
enum mcg_mode {
    MCG_MODE_AUTO = 0,    /* the launch shape mcg_tune picks for the tree's shape and the device
                             (include/mcg_tune.h): strip, staged or fused, with its CTAs per SM */
    MCG_MODE_LAYERED = 1, /* reference dataflow: materialised node words, one launch per layer */
    MCG_MODE_STAGED = 2,  /* two-phase pipeline: a pure sampler kernel writes basic-event words to
                             HBM, per-layer gate kernels with fused tallies read them; chunks are
                             double buffered on two streams so the phases overlap */
    MCG_MODE_STRIP = 3,   /* one persistent kernel per pass: each block takes 256-word strips, its
                             threads sample every event of their word and then evaluate every gate
                             for it from scratch rows of their own (n_nodes x 32 words per warp);
                             sampling and gate work of different blocks overlap on every SM */
    MCG_MODE_FUSED = 4    /* one persistent kernel per launch chunk: sample, gates, tallies fused */
};

/* Flattened PDAG handed to the engine.  All arrays are host memory, copied
 * at mcg_create.  Replaces the per-layer device blocks the reference builds
 * in src/mc/queue/kernel_builder.h:156-220 (basic events), 298-426 (gates)
 * and 694-770 (tallies). */
typedef struct mcg_graph_desc {
    uint32_t n_be;
    uint32_t n_gates;
    const int32_t *be_pdag_idx;   /* Variable::index() (>= 2); counter word 0 is pdag_idx + 1 */
    const uint32_t *be_event_idx; /* position in the basic-event block; counter word 1 is event_idx + 1 */
    const uint64_t *be_threshold; /* (uint64)(p * 2^32) in [0, 2^32] (src/mc/event/node.h:372-376) */
    const int32_t *gate_pdag_idx; /* may be NULL; informative only */
    const uint8_t *gate_op;       /* enum mcg_connective */
    const uint32_t *gate_k;       /* ATLEAST threshold, taken as uint8 like atleast_gate::at_least */
    const uint32_t *gate_in_begin;
    const uint32_t *gate_in_count;
    const uint32_t *gate_neg_count;
    const uint32_t *inputs;
    uint64_t n_inputs;
    uint32_t n_tally;             /* nodes whose ones are counted (the reference's tally block) */
    const uint32_t *tally_nodes;
} mcg_graph_desc;

#define MCG_SMEM_SLOTS_NONE 0xFFFFFFFFu

/* Engine options; zero-initialise and set what you need. */
typedef struct mcg_run_desc {
    uint32_t mode;            /* enum mcg_mode */
    int32_t device;           /* CUDA device ordinal */
    void *stream;             /* cudaStream_t to launch on; NULL = engine-owned stream */
    uint32_t block_threads;   /* fused kernel CTA size; 0 = tuned default */
    uint32_t smem_slots;      /* fused kernel shared-memory value slots per thread; 0 = auto,
                                 MCG_SMEM_SLOTS_NONE = keep every value in global scratch */
    uint32_t ctas_per_sm;     /* fused kernel persistent CTAs per SM (1..4); strip kernel resident
                                 blocks per SM (4..6, fewer = more registers per thread); 0 = auto */
    uint64_t chunk_words;     /* words per launch in one mcg_run; 0 = auto */
    uint64_t layered_max_words; /* layered/staged modes: words materialised per chunk; 0 = auto */
    uint32_t sampler_blocks_per_sm; /* staged mode: cap on sampler blocks per SM, to leave room for
                                       gate-phase blocks; 0 or 8 = no cap (measured best) */
    uint64_t tune_pass_words; /* MCG_MODE_AUTO: expected words per mcg_run call, the pass length the
                                 launch shape is tuned for; 0 = 2^24 */
} mcg_run_desc;

typedef struct mcg_engine mcg_engine;

/* Statistics of the fused program the engine compiled from the graph. */
typedef struct mcg_program_info {
    uint64_t n_ops;
    uint32_t smem_slots;      /* value slots resident in shared memory */
    uint32_t global_slots;    /* value slots spilled to the engine's global scratch */
    uint32_t max_live;        /* largest number of simultaneously live values */
    uint32_t block_threads;
    uint32_t grid_ctas;
    uint64_t scratch_bytes;   /* global scratch the fused kernel uses */
    uint32_t smem_bytes;      /* dynamic shared memory per CTA */
    uint32_t n_inline_be;     /* basic events generated straight into their one consumer */
} mcg_program_info;

/* Builds an engine: validates and copies the graph, compiles the fused
 * program, allocates device tables, tallies and scratch.
 * Replaces layer_manager::layer_manager (src/mc/queue/layer_manager.tpp:345-375). */
mcg_status mcg_create(const mcg_graph_desc *graph, const mcg_run_desc *run, mcg_engine **out);

/* Frees every device allocation of the engine.  The large work buffers
 * (strip and fused scratch, staged chunk buffers) are kept for the next
 * engine on the device, which takes the smallest kept one that fits instead
 * of allocating (at most 2 buffers, 32 GB per device; an allocation that
 * fails frees them first); mcg_trim_memory frees them.
 * Replaces layer_manager::~layer_manager (src/mc/queue/layer_manager.tpp:282-301). */
mcg_status mcg_destroy(mcg_engine *engine);

/* Frees the work buffers kept on `device` (none when no engine was
 * destroyed there).  No engine may be mid-destruction on that device. */
mcg_status mcg_trim_memory(int device);

/* Enqueues n_iterations passes, numbered iteration_first, iteration_first+1, ...
 * (the reference numbers passes from 1, src/mc/queue/queueable.h:725-731),
 * each over sample words [word_begin, word_begin + word_count).  Every tallied
 * node's ones grow by its popcount; total_bits grows by
 * n_iterations * word_count * 64.  Asynchronous on the engine's stream.
 * Replaces layer_manager::single_pass / pass (src/mc/queue/layer_manager.tpp:203-216).
 * Requires word_begin + word_count <= 2^32 (sample_idx is a uint32 counter word). */
mcg_status mcg_run(mcg_engine *engine, uint32_t iteration_first, uint32_t n_iterations,
                   uint64_t word_begin, uint64_t word_count);

/* Waits for all enqueued work (wait_and_throw, src/mc/queue/layer_manager.tpp:259). */
mcg_status mcg_synchronize(mcg_engine *engine);

/* Copies the tallies to host arrays of n_tally entries (either may be NULL);
 * synchronises first.  ones[i] belongs to tally_nodes[i].
 * Replaces collect_tallies / fetch_tally_for_event_with_index
 * (src/mc/queue/layer_manager.tpp:176-194, 271-279). */
mcg_status mcg_read_tallies(mcg_engine *engine, uint64_t *ones, uint64_t *total_bits);

/* Device address of the n_tally uint64 ones counters (for device-side
 * consumers such as a tally all-reduce).  Valid until mcg_destroy. */
mcg_status mcg_tally_device_ptr(mcg_engine *engine, uint64_t **ones_dev);

/* Overwrites the tallies with host-side counts (e.g. after a cross-rank reduction). */
mcg_status mcg_set_tallies(mcg_engine *engine, const uint64_t *ones, uint64_t total_bits);

/* Zeroes ones and total_bits. */
mcg_status mcg_reset_tallies(mcg_engine *engine);

/* Asynchronous snapshot of the tallies: enqueues on the engine's stream,
 * behind every pass submitted so far, a device-side copy of the counters
 * into the engine's snapshot slot `slot` (0 or 1) together with the total
 * bits those passes cover, and returns at once.  mcg_snapshot_read waits for
 * that copy only -- passes submitted after it keep running -- and returns
 * it.  Lets a caller decide on pass k while pass k + 1 runs (the pipelined
 * convergence loop of mcg_run_to_convergence).  No reference counterpart;
 * the reference waits for its queue before every harvest
 * (layer_manager.tpp:259). */
mcg_status mcg_snapshot_tallies(mcg_engine *engine, uint32_t slot);
mcg_status mcg_snapshot_read(mcg_engine *engine, uint32_t slot, uint64_t *ones, uint64_t *total_bits);

/* Materialised words of every node (n_be + n_gates rows of n_words) for pass
 * `iteration` over words [word_begin, word_begin + n_words), copied to host
 * memory out[node * n_words + w].  Uses the layered kernels; for parity
 * checks of individual words. */
mcg_status mcg_dump_words(mcg_engine *engine, uint32_t iteration, uint64_t word_begin,
                          uint64_t n_words, uint64_t *out);

mcg_status mcg_program_info_get(mcg_engine *engine, mcg_program_info *info);

/* Compiles the fused program of `graph` on the host only (no device needed)
 * with at most smem_slot_budget shared-memory slots.  Fills *info (the launch
 * fields stay 0) and, when ops is non-NULL, copies min(n_ops, ops_capacity)
 * ops of 4 uint32 words each.  For inspection and verification of the
 * program format; mcg_create compiles its own program. */
#define MCG_COMPILE_VARIABLE_THRESHOLDS 1u /* basic-event ops index a per-instance threshold table */
mcg_status mcg_compile(const mcg_graph_desc *graph, uint32_t smem_slot_budget, uint32_t flags,
                       mcg_program_info *info, uint32_t *ops, uint64_t ops_capacity);

/* Number of fused/layered kernel launches the engine has issued so far. */
mcg_status mcg_launch_count(mcg_engine *engine, uint64_t *launches);

/* Times `repeats` calls of mcg_run(engine, iteration_first, 1, word_begin, word_count)
 * with CUDA events on the engine's stream; *ms_per_run is the mean.  Tallies
 * are left accumulated. */
mcg_status mcg_time_runs(mcg_engine *engine, uint32_t iteration_first, uint64_t word_begin,
                         uint64_t word_count, uint32_t repeats, double *ms_per_run);

/* Staged mode: when enabled, every sampler-phase (k_stage_be) launch is
 * bracketed by CUDA events on its stream; mcg_profile_sampler_read returns
 * the number of timed launches since enabling and their summed duration.
 * For measurement only (adds two event records per launch). */
mcg_status mcg_profile_sampler(mcg_engine *engine, int32_t enable);
mcg_status mcg_profile_sampler_read(mcg_engine *engine, uint64_t *launches, double *total_ms);

/* Fused Monte Carlo pass that allocates no device memory.  No counterpart in
 * the reference, whose engine allocates every buffer it uses.
 *
 * For callers that cannot call cudaMalloc: work enqueued while a CUDA graph
 * is being captured, processes whose device memory comes from their own
 * pool or a fixed budget, and services that cannot afford the implicit
 * synchronisation of cudaMalloc/cudaFree.  The caller compiles the program
 * on the host with mcg_compile (flags 0), copies its n_ops ops (16 bytes
 * each) to device memory it owns (d_ops, 16-byte aligned) and passes a
 * device array d_ones of n_tally uint64 counters; smem_slots and
 * global_slots are the program's own counts from mcg_compile's info.  The
 * kernel adds each tallied node's ones over passes
 * [iteration_first, iteration_first + n_iterations) and words
 * [word_begin, word_begin + word_count) into d_ones (zero it first for fresh
 * counts), asynchronously on `stream` (NULL = the default stream) of the
 * current device.
 *
 * Values the program keeps outside shared memory go to one static device
 * array of MCG_NOALLOC_SCRATCH_BYTES per device, which every GPU that loads
 * the library holds until the process exits.  Programs whose global slots
 * need more than that at full occupancy (global_slots x SMs x 2 CTAs x 256
 * threads x 8 bytes) are rejected with MCG_ERR_INVALID; compile them with a
 * larger shared-memory budget or use mcg_create / mcg_run.  All calls share
 * the array, so calls that overlap on the GPU (concurrent streams, or
 * another device context of the same process on the same GPU) race and give
 * wrong counts; serialise them.  The first call on a device resolves the
 * array's address and sets the kernel's shared-memory limit, so make that
 * first call before any stream capture on that device.  That set-up is kept
 * for the life of the process: after cudaDeviceReset on a device, do not call
 * this entry point again in the same process. */
#define MCG_NOALLOC_SCRATCH_BYTES (32ull << 20)
mcg_status mcg_run_fused_noalloc(const void *d_ops, uint64_t n_ops, uint32_t smem_slots, uint32_t global_slots,
                                 uint64_t *d_ones, uint32_t n_tally, uint32_t iteration_first, uint32_t n_iterations,
                                 uint64_t word_begin, uint64_t word_count, void *stream);

/* Register-only sampler rate: basic-event words generated per second by a
 * kernel that only runs the Philox sampler (no memory traffic besides one
 * store per thread).  The speed of light of the fused kernel. */
mcg_status mcg_sampler_peak(int32_t device, uint64_t n_events, uint64_t n_words,
                            uint32_t repeats, double *words_per_second);
/* The same for the sampler of batches that evaluate several instances of one
 * tree per Philox call (uncertainty draws): `instances` (1 or 4) words per
 * Philox evaluation, each against its own threshold, without the per-pass
 * event table; the rate counts instance words. */
mcg_status mcg_sampler_peak_shared(int32_t device, uint64_t n_events, uint64_t n_words, uint32_t repeats,
                                   uint32_t instances, double *instance_words_per_second);

/* Message for the last failure on the calling thread ("" if none). */
const char *mcg_last_error(void);

/* Library version string. */
const char *mcg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MCG_H */
