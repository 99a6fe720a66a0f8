// autotune.cpp -- launch shapes per tree shape and device (include/mcg_tune.h).
//
// A shape key is hashed from the graph's structure and the device; on a
// miss every candidate launch shape is measured on short probe passes and
// the fastest is kept, in memory and in a small text file
// ("mcg-tune-1" header, then one "key mode ctas chunk rate probe_words" line
// per entry), so that later processes start from it.
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "error.hpp"
#include "mcg.h"
#include "mcg_tune.h"

namespace {

constexpr const char *kFileTag = "mcg-tune-1";

struct Entry {
    uint32_t mode = 0, ctas = 0;
    uint64_t chunk = 0;
    double rate = 0.0;
    uint64_t probe_words = 0;
};

struct Candidate {
    uint32_t mode, ctas;
};

// Launch shapes measured on a miss: the strip kernel at each residency it is
// built for, the staged pipeline, the fused interpreter at 4 and 2 CTAs per SM.
constexpr Candidate kCandidates[] = {{MCG_MODE_STRIP, 6}, {MCG_MODE_STRIP, 5}, {MCG_MODE_STRIP, 4},
                                     {MCG_MODE_STAGED, 0}, {MCG_MODE_FUSED, 4}, {MCG_MODE_FUSED, 2}};

std::mutex g_mu;
std::unordered_map<uint64_t, Entry> g_mem;
bool g_loaded = false;      // the file has been read into g_mem
bool g_path_given = false;  // mcg_tune_set_cache_file was called
std::string g_path;

struct Fnv {
    uint64_t h = 1469598103934665603ull;
    void add(const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
    }
    template <typename T>
    void add(T v) { add(&v, sizeof v); }
};

std::string cache_path() {
    if (g_path_given) return g_path;
    if (const char *e = std::getenv("MCG_TUNE_CACHE")) return e;
    std::string base;
    if (const char *x = std::getenv("XDG_CACHE_HOME"); x && *x) base = x;
    else if (const char *h = std::getenv("HOME"); h && *h) base = std::string(h) + "/.cache";
    return base.empty() ? std::string() : base + "/mcscram_b200/tune.txt";
}

void load_file_locked() {
    if (g_loaded) return;
    g_loaded = true;
    const std::string path = cache_path();
    if (path.empty()) return;
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) return;
    char line[256];
    bool tagged = false;
    while (std::fgets(line, sizeof line, f)) {
        if (!tagged) {
            tagged = std::strncmp(line, kFileTag, std::strlen(kFileTag)) == 0;
            if (!tagged) break;  // another format: ignore the file
            continue;
        }
        unsigned long long key = 0, chunk = 0, pw = 0;
        unsigned mode = 0, ctas = 0;
        double rate = 0.0;
        if (std::sscanf(line, "%llx %u %u %llu %lf %llu", &key, &mode, &ctas, &chunk, &rate, &pw) == 6 &&
            (mode == MCG_MODE_STRIP || mode == MCG_MODE_STAGED || mode == MCG_MODE_FUSED))
            g_mem[key] = Entry{mode, ctas, chunk, rate, pw};
    }
    std::fclose(f);
}

void make_parents(const std::string &path) {
    for (size_t i = 1; i < path.size(); ++i)
        if (path[i] == '/') ::mkdir(path.substr(0, i).c_str(), 0755);
}

// Rewrites the file from g_mem (write a temporary, then rename); a file that
// cannot be written leaves the cache in memory only.
void save_file_locked() {
    const std::string path = cache_path();
    if (path.empty()) return;
    make_parents(path);
    const std::string tmp = path + ".tmp" + std::to_string((unsigned long)::getpid());
    FILE *f = std::fopen(tmp.c_str(), "w");
    if (!f) return;
    std::fprintf(f, "%s\n", kFileTag);
    for (const auto &kv : g_mem)
        std::fprintf(f, "%016llx %u %u %llu %.9e %llu\n", (unsigned long long)kv.first, kv.second.mode,
                     kv.second.ctas, (unsigned long long)kv.second.chunk, kv.second.rate,
                     (unsigned long long)kv.second.probe_words);
    const bool ok = std::fclose(f) == 0;
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

// Structure statistics and device identity that make up the shape key.
mcg_status shape_key(const mcg_graph_desc &g, int device, uint64_t pass_words, uint64_t *key) {
    const uint64_t nn = (uint64_t)g.n_be + g.n_gates;
    std::vector<uint32_t> depth(nn, 0), parents(nn, 0);
    uint32_t layers = 0, max_fanin = 0, max_atleast = 0;
    uint64_t per_op[8] = {0};
    for (uint32_t j = 0; j < g.n_gates; ++j) {
        const uint64_t b = g.gate_in_begin[j], c = g.gate_in_count[j];
        if (b + c > g.n_inputs) return mcg::fail(MCG_ERR_INVALID, "gate inputs outside the input list");
        uint32_t d = 0;
        for (uint64_t i = b; i < b + c; ++i) {
            const uint32_t x = g.inputs[i];
            if (x >= g.n_be + j) return mcg::fail(MCG_ERR_INVALID, "gate input not below the gate");
            d = std::max(d, depth[x]);
            ++parents[x];
        }
        depth[g.n_be + j] = d + 1;
        layers = std::max(layers, d + 1);
        max_fanin = std::max<uint32_t>(max_fanin, (uint32_t)c);
        if (g.gate_op[j] < 8) ++per_op[g.gate_op[j]];
        if (g.gate_op[j] == MCG_ATLEAST) max_atleast = std::max<uint32_t>(max_atleast, (uint32_t)c);
    }
    uint64_t shared = 0;
    for (uint64_t i = 0; i < nn; ++i) shared += parents[i] > 1;
    mcg_program_info info{};
    const mcg_status st = mcg_compile(&g, 16, 0, &info, nullptr, 0);
    if (st != MCG_OK) return st;
    uint32_t pw_log2 = 0;
    while (pw_log2 < 24 && (2ull << pw_log2) <= pass_words) ++pw_log2;
    Fnv h;
    h.add(kFileTag, std::strlen(kFileTag));
    const char *ver = mcg_version();
    h.add(ver, std::strlen(ver));
    h.add(g.n_be);
    h.add(g.n_gates);
    h.add(g.n_inputs);
    h.add(g.n_tally);
    h.add(layers);
    h.add(max_fanin);
    h.add(max_atleast);
    h.add(shared);
    h.add(per_op, sizeof per_op);
    h.add(info.max_live);
    h.add(pw_log2);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
        h.add(prop.name, std::strlen(prop.name));
        h.add(prop.multiProcessorCount);
        h.add(prop.major);
        h.add(prop.minor);
    } else {
        cudaGetLastError();
        h.add("no-device", 9);
    }
    *key = h.h;
    return MCG_OK;
}

// The default probe: one warm-up pass, then the mean of two timed passes
// (CUDA events on the engine's stream) of a fresh engine of that shape.
double gpu_probe(void *, const mcg_graph_desc *g, const mcg_run_desc *cand, uint64_t words) {
    mcg_engine *e = nullptr;
    if (mcg_create(g, cand, &e) != MCG_OK) return -1.0;
    double ms = 0.0;
    mcg_status st = mcg_run(e, 1, 1, 0, words);
    if (st == MCG_OK) st = mcg_synchronize(e);
    if (st == MCG_OK) st = mcg_time_runs(e, 2, 0, words, 2, &ms);
    mcg_destroy(e);
    if (st != MCG_OK || !(ms > 0.0)) return -1.0;
    return (double)g->n_be * (double)words / (ms * 1e-3);
}

// Probe passes: as long as the real ones up to 2^20 words (four waves of the
// strip kernel on a B200), shorter for very large trees (at most ~2^33
// basic-event words per pass), whole 256-word strips.
uint64_t probe_words_for(const mcg_graph_desc &g, uint64_t pass_words) {
    uint64_t w = std::min<uint64_t>(pass_words, 1ull << 20);
    const uint64_t nb = std::max<uint32_t>(g.n_be, 1);
    if (nb * w > (1ull << 33)) w = std::max<uint64_t>(1ull << 16, (1ull << 33) / nb);
    w = std::max<uint64_t>(256, w / 256 * 256);
    return std::min<uint64_t>(w, std::max<uint64_t>(pass_words, 256));
}

}  // namespace

extern "C" {

mcg_status mcg_tune(const mcg_graph_desc *graph, const mcg_run_desc *run, uint64_t pass_words,
                    mcg_tune_probe_fn probe, void *user, mcg_tune_choice *out) {
    mcg::clear_error();
    if (!graph || !out) return mcg::fail(MCG_ERR_INVALID, "graph and out must not be NULL");
    *out = mcg_tune_choice{};
    const int device = run ? run->device : 0;
    if (!pass_words) pass_words = 1ull << 24;
    uint64_t key = 0;
    mcg_status st = shape_key(*graph, device, pass_words, &key);
    if (st != MCG_OK) return st;
    out->key = key;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        load_file_locked();
        const auto it = g_mem.find(key);
        if (it != g_mem.end()) {
            out->mode = it->second.mode;
            out->ctas_per_sm = it->second.ctas;
            out->layered_max_words = it->second.chunk;
            out->words_per_second = it->second.rate;
            out->probe_words = it->second.probe_words;
            out->from_cache = 1;
            return MCG_OK;
        }
    }
    const uint64_t words = probe_words_for(*graph, pass_words);
    Entry best;
    uint32_t tried = 0;
    for (const Candidate &c : kCandidates) {
        mcg_run_desc cand{};
        cand.mode = c.mode;
        cand.device = device;
        cand.ctas_per_sm = c.ctas;
        const double rate = probe ? probe(user, graph, &cand, words) : gpu_probe(nullptr, graph, &cand, words);
        ++tried;
        if (rate > best.rate) best = Entry{c.mode, c.ctas, 0, rate, words};
    }
    if (!(best.rate > 0.0)) return mcg::fail(MCG_ERR_CUDA, "no candidate launch shape ran on this graph");
    mcg::clear_error();  // failed candidates leave their messages behind
    {
        std::lock_guard<std::mutex> lock(g_mu);
        g_mem[key] = best;
        save_file_locked();
    }
    out->mode = best.mode;
    out->ctas_per_sm = best.ctas;
    out->layered_max_words = best.chunk;
    out->words_per_second = best.rate;
    out->probe_words = words;
    out->candidates = tried;
    return MCG_OK;
}

mcg_status mcg_tune_set_cache_file(const char *path) {
    mcg::clear_error();
    std::lock_guard<std::mutex> lock(g_mu);
    g_path = path ? path : "";
    g_path_given = true;
    g_loaded = false;  // read the new file on the next call (entries in memory stay)
    return MCG_OK;
}

mcg_status mcg_tune_forget(void) {
    mcg::clear_error();
    std::lock_guard<std::mutex> lock(g_mu);
    g_mem.clear();
    g_loaded = false;
    return MCG_OK;
}

}  // extern "C"
