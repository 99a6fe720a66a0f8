/*
 * mcg_tune.h -- launch shapes chosen per tree shape and device (libmcg.so).
 *
 * Replaces the reference's launch heuristic, which sizes SYCL work-groups
 * from the device's compute units and a fixed occupancy target
 * (src/mc/queue/working_set.h:518-570).  Here short timed probe passes pick
 * the evaluation mode and its launch shape (strip kernel at 6, 5 or 4 blocks
 * per SM, staged pipeline, fused interpreter at 4 or 2 CTAs per SM) for a
 * tree shape on a device, and the choice is cached in memory and in a file,
 * so that every later engine of that shape on that device starts with it.
 *
 * An engine created with mode MCG_MODE_AUTO (the value of a zero-initialised
 * mcg_run_desc) runs mcg_tune first and then uses its choice; its device
 * and stream fields are kept, its ctas_per_sm, smem_slots, chunk_words,
 * layered_max_words and sampler_blocks_per_sm are replaced by the choice.
 *
 * The shape key hashes: basic events, gates, inputs, tallied nodes, layers,
 * largest fan-in, largest ATLEAST fan-in, nodes with several parents, the
 * gate count of every connective, the fused program's largest number of
 * live values, the expected words per pass (rounded down to a power of two,
 * at most 2^24), the device's name, SM count and compute capability, and the
 * library version.  Probabilities do not enter it.
 *
 * Cache file: MCG_TUNE_CACHE if set ("" keeps the cache in memory only),
 * else $XDG_CACHE_HOME/mcscram_b200/tune.txt, else
 * $HOME/.cache/mcscram_b200/tune.txt; mcg_tune_set_cache_file overrides it.
 */
#ifndef MCG_TUNE_H
#define MCG_TUNE_H

#include <stdint.h>

#include "mcg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mcg_tune_choice {
    uint32_t mode;               /* MCG_MODE_STRIP, MCG_MODE_STAGED or MCG_MODE_FUSED */
    uint32_t ctas_per_sm;        /* strip: resident blocks per SM; fused: CTAs per SM; staged: 0 */
    uint64_t layered_max_words;  /* staged: words per chunk (0 = the engine's default) */
    double words_per_second;     /* basic-event words per second of the chosen shape in its probe */
    uint64_t probe_words;        /* words of each probe pass */
    uint64_t key;                /* the shape key */
    uint32_t from_cache;         /* 1: taken from the cache, nothing probed */
    uint32_t candidates;         /* launch shapes probed (0 on a cache hit) */
} mcg_tune_choice;

/* Measures one candidate launch shape (candidate->mode, ->ctas_per_sm,
 * ->layered_max_words on candidate->device) on `graph` over passes of
 * probe_words words; returns basic-event words per second, or a negative
 * value when the shape cannot run. */
typedef double (*mcg_tune_probe_fn)(void *user, const mcg_graph_desc *graph, const mcg_run_desc *candidate,
                                    uint64_t probe_words);

/* The launch shape for `graph` on run->device (run may be NULL: device 0)
 * when passes are `pass_words` words long (0: 2^24).  A cache hit returns
 * at once; a miss probes every candidate with `probe` (NULL: timed passes on
 * the GPU through mcg_create / mcg_time_runs / mcg_destroy, about 0.1-3 s
 * once per shape and device), keeps the fastest and stores it. */
mcg_status mcg_tune(const mcg_graph_desc *graph, const mcg_run_desc *run, uint64_t pass_words,
                    mcg_tune_probe_fn probe, void *user, mcg_tune_choice *out);

/* Cache file for later calls: a path, or "" to keep entries in memory only.
 * Entries already in memory stay. */
mcg_status mcg_tune_set_cache_file(const char *path);

/* Forgets the entries held in memory (the file stays; the next call reads it). */
mcg_status mcg_tune_forget(void);

/* The mode and CTAs per SM an engine runs with (the tuner's choice for an
 * engine created with MCG_MODE_AUTO). */
mcg_status mcg_engine_launch_shape(mcg_engine *engine, uint32_t *mode, uint32_t *ctas_per_sm);

#ifdef __cplusplus
}
#endif

#endif /* MCG_TUNE_H */
