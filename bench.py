#!/usr/bin/env python
"""Benchmark of the plain Monte Carlo fault-tree path on B200.

Workload (one "step" = one pass of the hot path over one batch): the 5,000
basic-event / 3,000-gate synthetic tree (seed 11, 45% AND, 40% OR, 10%
ATLEAST, 5% NOT/XOR, 20 layers, 30% of nodes with fan-out >= 2, p
log-uniform in [1e-5, 1e-2]); 2^30 samples = 2^24 uint64 words per node per
GPU; every gate tallied; strip mode (one persistent kernel per pass) unless
--mode says otherwise.  Each step is a new pass (iteration = step + 1),
exactly like the reference's pass loop.  N GPUs shard the sample-word range
(weak scaling: 2^24 words per GPU) and all-reduce the tallies after each pass.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line on rank 0.  The metric is gate-evals/s (gates x samples
per second); sample-words/s (basic-event words per second) is reported next
to it.  The CPU baseline and the reference arm run the reference-dataflow CPU
implementation (oracle/_ref: the reference's own Philox header compiled from
its sources, gate and tally loops restated) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "gate-evals/s"
UNIT = "gate-evals/s"
WORDS_PER_GPU = 1 << 24


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mcg", choices=["mcg", "reference"])
    ap.add_argument("--words", type=int, default=WORDS_PER_GPU, help="sample words per GPU per step")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-is", action="store_true",
                    help="plain workload: leave out the learned-IS time to accuracy on the 1e-8 tree")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="fused kernel CTAs per SM (0 = engine default)")
    ap.add_argument("--peak-words", type=int, default=1 << 22, help="words per register-only sampler launch")
    ap.add_argument("--mode", default="strip", choices=["fused", "staged", "layered", "strip"])
    ap.add_argument("--tree", default="config2", choices=["config1", "config2"],
                    help="plain workload's tree (config1: the small 200-event tree, for profiling captures)")
    ap.add_argument("--chunk-words", type=int, default=0, help="staged/layered chunk words (0 = engine default)")
    ap.add_argument("--sampler-blocks", type=int, default=0, help="staged: sampler blocks per SM (0 = default)")
    ap.add_argument("--mlp-rows", type=int, default=1_400_000, help="rows of the mlp workload")
    ap.add_argument("--workload", default="plain", choices=["plain", "ua", "is", "bis", "converge", "eta", "mlp"],
                    help="plain: the 5,000-event tree (headline); ua: batched uncertainty analysis; "
                         "is: GPU time to 5%% relative error on the 1e-8 tree, learned IS vs plain; "
                         "bis: the same for 1,024 rare-event trees at once with one shared network; "
                         "converge: ComputeTallies to a relative error, waiting vs pipelined convergence loop; "
                         "eta: combined event-tree pass, every sequence of a 2^n-sequence tree tallied; "
                         "mlp: proposal-network training steps at the batched set's row count")
    ap.add_argument("--eta-functional", type=int, default=8, help="functional events of the eta workload's tree")
    ap.add_argument("--converge-rel-err", type=float, default=1e-3)
    ap.add_argument("--converge-words", type=int, default=1 << 14, help="words per pass of the convergence loop")
    ap.add_argument("--converge-watch", default="top", choices=["top", "gates"],
                    help="monitored nodes: the top event, or every gate (heavier host statistics per step)")
    ap.add_argument("--converge-mode", default="fused", choices=["fused", "staged", "strip"],
                    help="engine mode of the convergence loop (short passes favour the fused kernel)")
    ap.add_argument("--is-rounds", type=int, default=5)
    ap.add_argument("--is-pipeline", default="batched", choices=["single", "batched"],
                    help="single: CE rounds + estimate on the one-tree sampler; batched: the batched pipeline "
                         "(cut-set defensive component, one CE round) on a batch of this one tree")
    ap.add_argument("--is-round-words", type=int, default=1 << 20, help="words per CE round (2^26 samples)")
    ap.add_argument("--is-tree", default="read-once", choices=["read-once", "dag"],
                    help="the 1e-8 tree: read-once, or with 20%% of its basic events read by two gates")
    ap.add_argument("--is-batch-words", type=int, default=1 << 20)
    ap.add_argument("--plain-words", type=int, default=1 << 23, help="words of the plain-MC rate measurement")
    ap.add_argument("--bis-trees", type=int, default=1024)
    ap.add_argument("--bis-only", default="", help="comma-separated tree indices of the set to run instead")
    ap.add_argument("--bis-set", default="shared", choices=["shared", "read-once"],
                    help="rare-event trees with 20%% of their basic events read by two gates (exact values from "
                         "tests/golden/config5_dag_exact.json), or read-once trees (exact by recursion)")
    ap.add_argument("--bis-ce-rounds", type=int, default=0, help="CE rounds (0 = the driver's default)")
    ap.add_argument("--bis-ce-words", type=int, default=1 << 11,
                    help="words per tree per CE round (2^17 samples: 2^18 and 2^19 measured as accurate, slower)")
    ap.add_argument("--bis-est-words", type=int, default=1 << 12, help="words per tree of the first estimate round")
    ap.add_argument("--bis-max-est-words", type=int, default=1 << 20,
                    help="estimate words per tree at most (a tree not at 5 %% by then is reported unconverged)")
    ap.add_argument("--bis-train-steps", type=int, default=150)
    ap.add_argument("--bis-plain-trees", type=int, default=64, help="trees of the plain-rate measurement")
    ap.add_argument("--bis-mode-cap", type=float, default=0.5, help="cap of the defensive mode proposals")
    ap.add_argument("--bis-defensive", default="auto", choices=["auto", "cutsets", "modes", "approx", "probe"],
                    help="defensive proposal of the mixture (ablation)")
    ap.add_argument("--bis-defensive-share", type=float, default=0.3)
    ap.add_argument("--bis-no-network", action="store_true", help="CE targets as the proposal (ablation)")
    ap.add_argument("--bis-no-importance-features", action="store_true", help="ablation")
    ap.add_argument("--bis-workers", type=int, default=0, help="generator processes (0 = host threads, max 32)")
    ap.add_argument("--ua-trees", type=int, default=512)
    ap.add_argument("--ua-draws", type=int, default=16)
    ap.add_argument("--ua-words", type=int, default=1 << 16)
    return ap.parse_args()


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        load = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU baseline

def cpu_rate(g, target_seconds: float, reference: bool = True, label: str = "the 5,000-event tree"):
    """Gate-evals/s of the CPU reference dataflow on a bounded sample of the
    workload (pass 1, leading words), using every host thread."""
    from oracle import oracle
    oracle.build()
    ref = reference and oracle.has_reference_build()
    words = 512
    t0 = time.perf_counter()
    oracle.tallies(g, 1, 1, 0, words, reference=ref)
    dt = time.perf_counter() - t0
    words = int(min(1 << 20, max(512, words * target_seconds / max(dt, 1e-3))))
    words = (words // 64) * 64 or 64
    t0 = time.perf_counter()
    oracle.tallies(g, 1, 1, 0, words, reference=ref)
    dt = time.perf_counter() - t0
    rate = g.n_gates * words * 64 / dt
    kind = "reference" if ref else "port"
    what = ("oracle/_ref/libref_mc.so: reference src/mc/prng/philox128.h compiled from its sources, "
            "gate/tally loops restated from src/mc/kernel/gate.h and tally.h" if ref else
            "oracle/liboracle.so: plain-C restatement of the reference dataflow")
    return {"value": rate, "unit": UNIT, "cores": oracle.max_threads(), "kind": kind,
            "sample": f"{words} words (pass 1, words [0, {words})) of {label}, "
                      f"{g.n_gates} gates tallied, {dt:.2f} s; {what}",
            "seconds": dt, "words": words}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return 0
    from mcscram_b200 import synth
    from oracle import oracle
    oracle.build()
    g = synth.config2()
    ref = oracle.has_reference_build()
    # size one step to ~args.cpu_seconds / 2 of CPU work
    probe = 512
    t0 = time.perf_counter()
    oracle.tallies(g, 1, 1, 0, probe, reference=ref)
    dt = time.perf_counter() - t0
    words = int(min(1 << 20, max(256, probe * (args.cpu_seconds / 2) / max(dt, 1e-3))))
    for i in range(args.warmup):
        oracle.tallies(g, 1 + i, 1, 0, min(words, 1024), reference=ref)
    times = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        oracle.tallies(g, 1 + i, 1, 0, words, reference=ref)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = g.n_gates * words * 64 * args.steps / total
    cores = oracle.max_threads()
    kind = "reference" if ref else "port"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "plain MC, 5,000-event / 3,000-gate synthetic tree (seed 11), pass-sized sample",
                   "samples_per_step": words * 64, "n_be": g.n_be, "n_gates": g.n_gates},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{words} words per step of the 5,000-event tree on {cores} host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- GPU arm

def pipe_peak_from_profile():
    """Basic-event words per second of the sampler code with the integer
    multiply (fmaheavy) pipe saturated, from the committed ncu summary of the
    sampler kernel (profiles/k_stage_be_config2.txt), at its 1.96 GHz."""
    p = ROOT / "profiles" / "k_stage_be_config2.txt"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        if ln.startswith("fmaheavy_saturated_gword_s:"):
            try:
                return float(ln.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def traffic_from_profile(kernel: str):
    """DRAM bytes per launch of `kernel` at the bench's launch size, from the
    committed ncu summary (profiles/<kernel>_config2.txt), if present."""
    p = ROOT / "profiles" / f"{kernel}_config2.txt"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        if ln.startswith("traffic_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def run_ua(args, rank: int, world: int, local: int) -> int:
    """Batched uncertainty analysis: trees x lognormal draws in one persistent
    graph-captured launch per step; trees sharded over ranks."""
    import torch
    from mcscram_b200 import synth
    from mcscram_b200.uncertainty import Batch

    torch.cuda.set_device(local)
    trees = synth.config3(args.ua_trees)
    mine = [t.with_tallies([t.root]) for i, t in enumerate(trees) if i % world == rank]
    with Batch(mine, device=local, ctas_per_sm=args.ctas_per_sm) as b:
        base = [t.be_prob for t in mine]
        for i in range(args.warmup):
            b.uncertainty(base, draws_per_tree=args.ua_draws, words_per_instance=args.ua_words, seed=i)
        clocks = ClockSampler(local)
        clocks.start()
        ms = []
        for i in range(args.steps):
            p_top, stats, kms = b.uncertainty(base, draws_per_tree=args.ua_draws, words_per_instance=args.ua_words,
                                              seed=1000 + i)
            ms.append(kms)
        clk = clocks.stop()
        info = b.info()
    be_words = sum(t.n_be for t in mine) * args.ua_draws * args.ua_words
    gates = sum(t.n_gates for t in mine) * args.ua_draws * args.ua_words * 64
    kms = statistics.mean(ms)
    # roofline: instance words per second (one launch per step) against the
    # register-only sampler that shares its Philox calls as the batch does
    from mcscram_b200 import _capi
    share = int(info.get("instances_per_item", 1)) or 1
    kernel = "k_fused_batch_k" if share > 1 else "k_fused_batch"
    achieved = be_words / (kms * 1e-3)
    peak = _capi.sampler_peak_shared(share, n_events=256, n_words=args.peak_words, repeats=3, device=local)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": gates / (kms * 1e-3) * world, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": kms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"batched uncertainty analysis: {args.ua_trees} trees x {args.ua_draws} "
                                   f"lognormal draws (EF 3), {args.ua_words * 64} samples per instance",
                       "instances": len(mine) * args.ua_draws, "l2": "inputs > L2 per launch"},
            "sample_words_per_s": be_words / (kms * 1e-3) * world,
            "roofline": {"bound": "int-alu", "kernel": kernel, "achieved": achieved / 1e9, "peak": peak / 1e9,
                         "unit": "G instance-words/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": f"register-only sampler of the batch path ({share} instance(s) per Philox "
                                        "evaluation, k_sampler_peak_shared) measured in this run",
                         "work_unit": "instance word = one basic event's 64 draws of one instance"},
            "batch": info, "clocks": clk}), flush=True)
    return 0


def measure_is(args, local: int, tree: str = "read-once") -> dict:
    """GPU time to a 5% relative error (95% confidence) on the 2,000-event tree
    whose exact top-event probability is ~1e-8: the learned-IS pipeline
    (cross-entropy rounds with on-GPU MLP training, then IS batches until the
    target) measured end to end, against the plain sampler's time derived
    from its rate measured on the same tree.  Returns the fields of the
    `is` workload's line."""
    import numpy as np
    import torch
    from mcscram_b200 import _capi, synth
    from mcscram_b200.importance import ImportanceSampler, cross_entropy, estimate

    torch.cuda.set_device(local)
    dag = tree == "dag"
    g = (synth.config4_dag() if dag else synth.config4()).with_tallies([])
    g = g.with_tallies([g.root])
    # plain sampler rate on this tree (staged pipeline, inputs resident)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    with _capi.Engine(g, device=local, stream=stream.cuda_stream, mode=_capi.MODE_STAGED) as e:
        for i in range(args.warmup):
            e.run(1 + i, 1, 0, 1 << 20)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e.run(100, 1, 0, args.plain_words)
        b.record(stream)
        torch.cuda.synchronize()
        plain_ms = a.elapsed_time(b)
        ones, total = e.tallies()
    plain_rate = args.plain_words * 64 / (plain_ms * 1e-3)  # samples / s
    if args.is_pipeline == "batched" and args.warmup:
        # one untimed run of the pipeline: the first launches of its kernels in
        # a process load their code and size the per-thread stack
        from mcscram_b200.importance import batched_learned_is
        batched_learned_is([g], target_rel_err=0.05, device=local)
        torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    if args.is_pipeline == "batched":
        from mcscram_b200.importance import batched_learned_is
        br = batched_learned_is([g], target_rel_err=0.05, device=local)
        torch.cuda.synchronize()
        is_wall = time.perf_counter() - t0
        clk = clocks.stop()
        res = {"estimate": float(br.estimate[0]), "rel_err95": float(br.rel_err95[0]), "samples": int(br.samples[0]),
               "hits": int(br.hits[0]), "ess": float(br.ess[0]), "fallback": bool(br.fallback[0]),
               "gpu_ms": sum(br.gpu_ms.values())}

        class _H:
            gpu_ms = 0.0
            rounds = [r for r in br.rounds if r["phase"] == "ce"]
        hist = _H()
    else:
        with ImportanceSampler(g, device=local) as s:
            q, mlp, hist = cross_entropy(g, rounds=args.is_rounds, words_per_round=args.is_round_words, sampler=s,
                                         device=local)
            res = estimate(s, q, target_rel_err=0.05, words_per_batch=args.is_batch_words)
        torch.cuda.synchronize()
        is_wall = time.perf_counter() - t0
        clk = clocks.stop()
        mlp.close()
    p_hat = res["estimate"]
    n_req = 1.959963984540054 ** 2 * (1 - p_hat) / (p_hat * 0.05 ** 2) if p_hat > 0 else float("inf")
    plain_s = n_req / plain_rate
    if dag:  # committed BDD value (tests/golden/make_dag_exact.py)
        exact = json.loads((ROOT / "tests" / "golden" / "config5_dag_exact.json").read_text())["config4_dag"]
    else:
        exact = float(synth.read_once_probability(g)[g.root])
    se = p_hat * res["rel_err95"] / 1.959963984540054
    return {
        "metric": "GPU time to 5% rel err at P_top~1e-8", "value": is_wall, "unit": "s", "n_gpus": 1,
        "higher_is_better": False, "vs_baseline": None, "dtype": "u64 sampling, fp64 weights, bf16/fp32 MLP",
        "data": "synthetic", "steps": 1, "warmup": args.warmup,
        "config": {"workload": (("2,000-event / 1,200-gate rare-event tree with 400 basic events read by two "
                                 "gates (seed 4)") if dag else "2,000-event / 1,200-gate rare-event tree (seed 49)") +
                               (f", learned IS (CE rounds {args.is_rounds} x {args.is_round_words * 64} samples) vs "
                                "plain MC" if args.is_pipeline == "single" else
                                ", batched learned IS pipeline on this one tree (cut-set defensive component, one "
                                "CE round) vs plain MC")},
        "is": {"estimate": p_hat, "rel_err95": res["rel_err95"], "samples": res["samples"], "hits": res["hits"],
               "ess": res["ess"], "fallback": res["fallback"], "wall_s": is_wall,
               "gpu_s": (hist.gpu_ms + res["gpu_ms"]) * 1e-3, "ce_rounds": hist.rounds,
               "exact_p_top": exact, "z_vs_exact": (p_hat - exact) / se if se > 0 else None},
        "plain": {"samples_per_s": plain_rate, "required_samples": n_req, "seconds": plain_s,
                  "measured_words": args.plain_words, "measured_ms": plain_ms,
                  "note": "time derived from the rate measured on this tree"},
        "warm_up": ("the batched pipeline once untimed on the same tree" if args.is_pipeline == "batched" and
                    args.warmup else "none"),
        "speedup": plain_s / is_wall, "clocks": clk}


def run_is(args, rank: int, world: int, local: int) -> int:
    """The `is` workload: one line with the learned-IS time to 5% on the
    2,000-event rare-event tree against plain MC (measure_is)."""
    if rank != 0:
        return 0
    print(json.dumps(measure_is(args, local, args.is_tree)), flush=True)
    return 0


def run_bis(args, rank: int, world: int, local: int) -> int:
    """Batched learned IS: the rare-event trees (events log-uniform in [50,
    10,000], AND-heavy and ATLEAST-heavy mixes, exact P_top log-uniform in
    [1e-10, 1e-5]) solved together until each reaches a 5% relative error
    (95% confidence) or falls back to plain sampling; trees sharded over
    ranks, the network's training rows gathered from all ranks.  Plain
    batched MC is timed on a subset of the trees (the staged plain path over
    their joined graph) and its time to the same accuracy is extrapolated
    from that rate, since at 1e-10 it needs ~1.5e13 samples per tree."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from mcscram_b200 import _capi, parallel, synth
    from mcscram_b200.graph import concat
    from mcscram_b200.importance import batched_learned_is

    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    n_workers = args.bis_workers or min(32, os.cpu_count() or 1)
    # one process pool for the generator, the warm-up and the timed run (a
    # service keeps its host workers the way it keeps its CUDA context)
    workers = ProcessPoolExecutor(max_workers=n_workers, mp_context=mp.get_context("spawn"))
    t_gen = time.perf_counter()
    mine_idx = parallel.shard_items(args.bis_trees, world, rank)
    if args.bis_only:  # a chosen subset of the set's trees (to profile the slowest ones)
        only = [int(x) for x in args.bis_only.split(",")]
        mine_idx = [only[i] for i in parallel.shard_items(len(only), world, rank)]
    dag = args.bis_set == "shared"
    trees = synth.config5_instances(mine_idx, workers=workers, shared=dag)
    t_gen = time.perf_counter() - t_gen
    if dag:  # exact values of the shared-event set: committed BDD results (null: BDD over its node limit)
        fx = json.loads((ROOT / "tests" / "golden" / "config5_dag_exact.json").read_text())["config5_dag"]
        for k, i in enumerate(mine_idx):
            trees[k].meta["exact_p_top"] = fx[i] if i < len(fx) and fx[i] is not None else float("nan")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    exact = np.array([g.meta["exact_p_top"] for g in trees])
    # warm-up: the whole pipeline on a few small trees, then once untimed on
    # every tree (the step itself: first use of its device allocations)
    small = sorted(range(len(trees)), key=lambda k: trees[k].n_be)[:8]
    for i in range(args.warmup):
        batched_learned_is([trees[k] for k in small], device=local, ce_rounds=1, est_words=1 << 10,
                           max_est_words=1 << 12, train_steps=5, workers=workers)
    if args.warmup:
        batched_learned_is(trees, target_rel_err=0.05, device=local, ce_rounds=args.bis_ce_rounds or None,
                           ce_words=args.bis_ce_words, est_words=args.bis_est_words, max_est_words=args.bis_max_est_words,
                           train_steps=args.bis_train_steps, mode_cap=args.bis_mode_cap, workers=workers,
                           defensive_proposal=args.bis_defensive, defensive=args.bis_defensive_share,
                           use_network=not args.bis_no_network,
                           importance_features=not args.bis_no_importance_features)
    torch.cuda.synchronize()
    # plain rate on a subset: joined graph of the first trees, plain staged pass
    sub = trees[: min(args.bis_plain_trees, len(trees))]
    u, bb, roots = concat(sub)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    with _capi.Engine(u, device=local, stream=stream.cuda_stream, mode=_capi.MODE_STAGED) as e:
        e.run(1, 1, 0, 1 << 12)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e.run(2, 1, 0, args.plain_words >> 6)
        b.record(stream)
        torch.cuda.synchronize()
        plain_ms = a.elapsed_time(b)
    torch.cuda.set_stream(torch.cuda.default_stream())
    be_word_s = u.n_be * (args.plain_words >> 6) / (plain_ms * 1e-3)  # event words per second, plain path
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = batched_learned_is(trees, target_rel_err=0.05, device=local, ce_rounds=args.bis_ce_rounds or None,
                             ce_words=args.bis_ce_words, est_words=args.bis_est_words, max_est_words=args.bis_max_est_words,
                             train_steps=args.bis_train_steps, mode_cap=args.bis_mode_cap, workers=workers,
                             defensive_proposal=args.bis_defensive, defensive=args.bis_defensive_share,
                             use_network=not args.bis_no_network,
                             importance_features=not args.bis_no_importance_features)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    gpu_s = sum(res.gpu_ms.values()) * 1e-3
    z = 1.959963984540054
    p_ref = np.where(np.isfinite(exact), exact, res.estimate)
    n_req = z * z * (1 - p_ref) / (p_ref * 0.05 ** 2)  # plain samples per tree to 5% at 95%
    nb = np.array([g.n_be for g in trees], dtype=np.float64)
    plain_s = float(np.sum(n_req / 64 * nb / be_word_s))
    checked = np.isfinite(exact)
    exact = np.where(checked, exact, res.estimate)
    err = np.abs(res.estimate - exact) / exact
    se = res.estimate * res.rel_err95 / z
    within3 = (np.abs(res.estimate - exact) <= 3 * se) & checked
    within5 = (np.abs(res.estimate - exact) <= 5 * se) & checked
    with np.errstate(divide="ignore", invalid="ignore"):
        zs = np.where(se > 0, (res.estimate - exact) / se, np.inf)
    worst = [{"tree": int(mine_idx[k]), "events": trees[k].n_be, "p_exact": float(exact[k]),
              "est_over_exact": float(res.estimate[k] / exact[k]), "rel_err95": float(res.rel_err95[k]),
              "z": float(zs[k]), "converged": bool(res.converged[k]), "fallback": bool(res.fallback[k])}
             for k in np.argsort(-np.abs(np.nan_to_num(zs, nan=np.inf)))[:12] if checked[k] and not within3[k]]
    wall_max, gpu_max = wall, gpu_s
    if world > 1:
        wall_max, gpu_max = parallel.allreduce_max([wall, gpu_s])
        counts = parallel.allreduce_tallies(np.array([res.converged.sum(), res.fallback.sum(), within3.sum(),
                                                      len(trees), checked.sum(), within5.sum()], dtype=np.uint64))
        plain_s = parallel.allreduce_max([plain_s])[0]
    else:
        counts = [int(res.converged.sum()), int(res.fallback.sum()), int(within3.sum()), len(trees),
                  int(checked.sum()), int(within5.sum())]
    if rank == 0:
        print(json.dumps({
            "metric": "GPU time to 5% rel err, batched rare-event trees", "value": wall_max, "unit": "s",
            "n_gpus": world, "steps": 1, "warmup": args.warmup, "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "u64 sampling, fp64 weights, bf16/fp32 MLP", "data": "synthetic",
            "config": {"workload": f"batched learned IS: {args.bis_trees} rare-event trees "
                                   f"({'20% of basic events read by two gates' if dag else 'read-once'}; events "
                                   "log-uniform [50, 10000], AND-/ATLEAST-heavy, target P_top log-uniform "
                                   "[1e-10, 1e-5]), one shared 16-64-64-1 proposal network, until 5% rel err "
                                   "(95%) per tree or plain fallback",
                       "tree_set": args.bis_set,
                       "ce_rounds": sum(1 for r in res.rounds if r["phase"] == "ce"),
                       "ce_samples_per_tree": args.bis_ce_words * 64,
                       "defensive": args.bis_defensive, "defensive_share": args.bis_defensive_share,
                       "network": not args.bis_no_network, "importance_features": not args.bis_no_importance_features,
                       "events": int(nb.sum()), "gates": int(sum(g.n_gates for g in trees)),
                       "warm_up": "the pipeline on the 8 smallest trees x warmup, then once untimed on every tree; "
                                  "host process pool kept from the generator"},
            "is": {"wall_s": wall_max, "gpu_s": gpu_max, "gpu_ms_by_phase": res.gpu_ms,
                   "wall_s_by_phase": res.seconds, "trees": int(counts[3]), "converged": int(counts[0]),
                   "fallback": int(counts[1]), "within_3_sigma_of_exact": int(counts[2]),
                   "checked_against_exact": int(counts[4]), "within_5_sigma_of_exact": int(counts[5]),
                   "median_abs_rel_err_vs_exact": float(np.median(err)), "max_abs_rel_err_vs_exact": float(err.max()),
                   "max_rel_err95": float(res.rel_err95.max()), "samples_total": int(res.samples.sum()),
                   "rounds": len(res.rounds), "converged_outside_3_sigma": int((res.converged & ~within3).sum()),
                   "round_log": [[r["phase"], int(r.get("trees", r.get("trees_left", 0))), int(r.get("words", 0)),
                                  round(float(r["ms"]), 1)] + ([[int(mine_idx[k]) for k in r["tree_ids"]]]
                                                               if 0 < len(r.get("tree_ids", [])) < 8 else [])
                                 for r in res.rounds],
                   "outside_3_sigma_rank0": worst},
            "plain": {"event_words_per_s": be_word_s, "measured_on_trees": len(sub), "measured_words": args.plain_words >> 6,
                      "measured_ms": plain_ms, "required_samples_total": float(n_req.sum()), "seconds": plain_s,
                      "note": "plain batched MC time to the same accuracy, extrapolated from the plain staged "
                              "rate measured on the joined graph of a subset of the trees, with each tree's "
                              "required samples from its exact P_top"},
            "speedup": plain_s / wall_max, "generation_s": t_gen, "clocks": clk}), flush=True)
    workers.shutdown()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_mlp(args, rank: int, world: int, local: int) -> int:
    """Training of the proposal network at the batched rare-event set's size:
    `--mlp-rows` rows (1.4 M, the 1,024 trees' events) of 16 features,
    `--steps` Adam steps timed with CUDA events after `--warmup` steps.  The
    dense products are 2 x (16x64 + 64x64 + 64) multiply-adds per row
    forward, twice that backward (activation and weight gradients): 3 x that
    per row and step in all."""
    if rank != 0:
        return 0
    import numpy as np
    import torch
    from mcscram_b200.importance import ProposalMLP

    torch.cuda.set_device(local)
    rng = np.random.default_rng(1)
    n = args.mlp_rows
    feats = rng.normal(size=(n, 16)).astype(np.float32)
    tgt = rng.uniform(0.0, 0.5, n).astype(np.float32)
    w = rng.uniform(0.5, 1.5, n).astype(np.float32)
    mlp = ProposalMLP(device=local)
    mlp.train(feats, tgt, w, steps=max(args.warmup, 1), lr=1e-3)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    loss = mlp.train(feats, tgt, w, steps=args.steps, lr=1e-3)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    ms = mlp.last_train_ms / args.steps if getattr(mlp, "last_train_ms", None) else wall * 1e3 / args.steps
    mlp.close()
    flops = 3 * 2 * (16 * 64 + 64 * 64 + 64) * n  # per Adam step
    peak = None
    peaks_file = ROOT / "MEASURED_PEAKS.json"
    if peaks_file.exists():
        peak = json.loads(peaks_file.read_text()).get("bf16_tflops")
    achieved = flops / (ms * 1e-3) / 1e12
    print(json.dumps({
        "metric": "proposal-network training step", "value": ms, "unit": "ms/step", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "vs_baseline": None,
        "dtype": "bf16 operands, fp32 accumulation", "data": "synthetic",
        "config": {"workload": f"16-64-64-1 network, weighted cross-entropy, {n} rows, Adam",
                   "rows": n, "timing": "CUDA events around the training steps (gradient, reduction, Adam, "
                                        "weight packing) with rows resident"},
        "loss": loss, "wall_s": wall,
        "roofline": {"bound": "tensor", "kernel": "k_mlp_grad", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "peak_source": "MEASURED_PEAKS.json bf16_tflops (cuBLAS bf16 GEMM, burst)",
                     "work_unit": "3 x 2 x 5,184 flops per row and step"},
        "clocks": clk}), flush=True)
    return 0


def run_converge(args, rank: int, world: int, local: int) -> int:
    """ComputeTallies (the reference's ProbabilityAnalyzer<DirectEval> path) on
    the 200-event / 100-gate tree to a relative error of the top event:
    the convergence loop that waits for every pass against the pipelined one
    that judges pass k while pass k + 1 runs (same tallies and stopping
    point).  Wall time of the whole call, median of the steps."""
    if rank != 0:
        return 0
    import torch
    from mcscram_b200 import _capi, host, synth

    torch.cuda.set_device(local)
    g = synth.config1()
    p = host.Pdag.from_flat(g)
    watch = [] if args.converge_watch == "top" else [int(x) for x in g.gate_pdag_idx[:-1]]
    res = {}
    for pipelined in (0, 1):
        kw = {} if args.converge_watch == "top" else dict(num_trials=1 << 26, early_stop=0)  # rare gates never converge
        s = host.Settings.default(ci_rel_margin_error=args.converge_rel_err, pipelined=pipelined,
                                  max_words_per_iteration=args.converge_words, **kw)
        for _ in range(args.warmup):
            host.compute_tallies(p, s, watch, device=local, mode=_capi.MODES[args.converge_mode])
        times = []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tallies, rep = host.compute_tallies(p, s, watch, device=local, mode=_capi.MODES[args.converge_mode])
            times.append(time.perf_counter() - t0)
        res[pipelined] = {"seconds": statistics.median(times), "passes": rep["passes"], "trials": rep["trials"],
                          "p_top": tallies[0]["mean"], "steps": rep["steps"], "burn_in_steps": rep["burn_in_steps"]}
    assert res[0]["trials"] == res[1]["trials"] and res[0]["p_top"] == res[1]["p_top"]
    print(json.dumps({
        "metric": "ComputeTallies wall time to convergence", "value": res[1]["seconds"], "unit": "s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "data": "synthetic",
        "dtype": "u64", "vs_baseline": None,
        "config": {"workload": f"200-event / 100-gate tree (seed 372), monitored: {args.converge_watch}, Bayes policy, relative "
                               f"error {args.converge_rel_err}, {args.converge_words} words per pass, {args.converge_mode} mode"},
        "waiting_loop": res[0], "pipelined_loop": res[1],
        "speedup": res[0]["seconds"] / res[1]["seconds"]}), flush=True)
    return 0


def run_eta(args, rank: int, world: int, local: int) -> int:
    """The combined event-tree path (the reference's RunCombinedEtaAnalysis):
    a complete binary event tree over `--eta-functional` functional events
    whose fault trees are the top gates of the 5,000-event / 3,000-gate tree,
    written as MEF, loaded, and sampled as one PDAG with the OR root, every
    sequence gate (2^n) and the fault tree's top tallied.  One step = one
    pass of 2^30 samples.  `value` = samples/s with every sequence evaluated;
    `e2e` = eta.run_combined (PDAG from the MEF model, layering, engine, pass,
    tallies) for the same samples.  The sequences partition the outcomes, so
    their tallies must add up to the samples exactly."""
    if rank != 0:
        return 0
    import torch
    from mcscram_b200 import _capi, eta, host, mef, synth

    torch.cuda.set_device(local)
    g0 = synth.config2()
    xml = synth.event_tree_xml(g0, args.eta_functional)
    t0 = time.perf_counter()
    model = mef.parse(xml)
    c = eta.combined_pdag(model, "IE")
    g = c.flat()
    host_s = time.perf_counter() - t0
    n_seq = len(c.sequences)
    W = args.words
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    mode = _capi.MODES[args.mode]
    eng = _capi.Engine(g, device=local, stream=stream.cuda_stream, mode=mode)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    for i in range(args.warmup):
        flush.zero_()
        eng.run(i + 1, 1, 0, W)
    torch.cuda.synchronize()
    eng.reset_tallies()
    if args.mode in ("staged", "strip"):
        eng.profile_sampler(True)
    launches0 = eng.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        flush.zero_()
        eng.run(args.warmup + i + 1, 1, 0, W)
    t_end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = eng.launch_count() - launches0
    ms_per_step = t_start.elapsed_time(t_end) / args.steps
    ones, total = eng.tallies()
    partition_exact = int(ones[0]) == total and sum(int(x) for x in ones[1:1 + n_seq]) == total
    samples = W * 64
    value = samples / (ms_per_step * 1e-3)
    kernel, roof = None, None
    if args.mode in ("staged", "strip"):
        kernel = "k_stage_be" if args.mode == "staged" else "k_strip"
        n_a, ms_a = eng.profile_sampler_read()
        eng.profile_sampler(False)
        avg_launch_s = ms_a * 1e-3 / max(n_a, 1)
        achieved = g.n_be * W * args.steps / max(n_a, 1) / avg_launch_s
        peak = _capi.sampler_peak(n_events=256, n_words=args.peak_words, repeats=3, device=local)
        roof = {"bound": "int-alu", "kernel": kernel, "achieved": achieved / 1e9, "peak": peak / 1e9,
                "unit": "Gword/s", "frac": achieved / peak, "traffic": None, "launches": n_a,
                "avg_launch_ms": avg_launch_s * 1e3,
                "peak_source": "register-only Philox sampler kernel (k_sampler_peak) measured in this run",
                "work_unit": "basic-event word = 16 Philox4x32-10 calls"}
    eng.close()
    e2e = None
    if args.e2e_steps > 0:
        s = host.Settings.default(num_trials=samples, early_stop=0, ci_rel_margin_error=1e-9,
                                  max_words_per_iteration=W)
        ts = []
        for _ in range(args.e2e_steps):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            r = eta.run_combined(model, "IE", s, mode=mode, device=local)
            ts.append(time.perf_counter() - t1)
        e2e_s = statistics.median(ts)
        h2d = g.n_be * 16 + g.n_gates * 20 + g.inputs.size * 4 + g.tally_nodes.size * 4
        e2e = {"value": samples / e2e_s, "unit": "samples/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(g.tally_nodes.size * 8), "seconds_per_step": e2e_s,
               "sequences_reported": len(r.sequences)}
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cpu_rate(g, args.cpu_seconds, reference=True,
                       label=f"the {n_seq}-sequence event tree's combined PDAG")
        cpu = dict(cpu, value=cpu["value"] / g.n_gates, unit="samples/s")
    line = {
        "metric": "event-tree samples/s", "value": value, "unit": "samples/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"combined event-tree pass: {args.eta_functional} functional events over the top gates "
                               f"of the 5,000-event / 3,000-gate tree (seed 11), {n_seq} sequences, every sequence "
                               "tallied, loaded from generated MEF", "samples_per_step": samples,
                   "n_be": g.n_be, "n_gates": g.n_gates, "tallied_nodes": int(g.tally_nodes.size),
                   "l2": "256 MB buffer written between steps", "mode": args.mode},
        "gate_evals_per_s": g.n_gates * value, "sequence_tallies_per_s": n_seq * value,
        "partition_exact": partition_exact, "host_model_seconds": host_s, "gpu_launches": int(launches),
        "clocks": clk,
    }
    if roof:
        line["roofline"] = roof
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    args = parse_args()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # N ranks, one per GPU, on this node (the same launch as torchrun's)
        from mcscram_b200 import parallel
        return parallel.launch_local_ranks(args.gpus, str(Path(__file__).resolve()), sys.argv[1:],
                                           need_gpus=args.impl != "reference")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus not in (1, world):
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "ua":
        return run_ua(args, rank, world, local)
    if args.workload == "is":
        return run_is(args, rank, world, local)
    if args.workload == "bis":
        return run_bis(args, rank, world, local)
    if args.workload == "converge":
        return run_converge(args, rank, world, local)
    if args.workload == "mlp":
        return run_mlp(args, rank, world, local)
    if args.workload == "eta":
        return run_eta(args, rank, world, local)

    import numpy as np
    import torch
    import torch.distributed as dist

    from mcscram_b200 import _capi, parallel, synth

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    g = synth.config2() if args.tree == "config2" else synth.config1()
    W = args.words
    word_begin, W = parallel.weak_shard(W, rank)  # weak scaling: W words per rank
    # one dedicated stream for the engine and for every torch op and event here
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng_kw = dict(device=local, stream=stream.cuda_stream, ctas_per_sm=args.ctas_per_sm, mode=_capi.MODES[args.mode],
                  layered_max_words=args.chunk_words, sampler_blocks_per_sm=args.sampler_blocks)
    eng = _capi.Engine(g, **eng_kw)
    info = eng.program_info()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # the one exchange of the multi-GPU path: after every pass, the sum over
    # ranks of the engine's uint64 tallies, device to device over NCCL
    local_ones = global_ones = None
    if world > 1:
        local_ones = parallel.device_counters(eng.tally_device_ptr(), eng.n_tally)
        global_ones = torch.zeros_like(local_ones)

    def allreduce_tallies():
        if world == 1:
            return
        global_ones.copy_(local_ones)
        parallel.allreduce_counters_(global_ones)

    # warm-up passes (iterations 1..W); then the timed passes continue the numbering
    for i in range(args.warmup):
        flush.zero_()
        eng.run(i + 1, 1, word_begin, W)
        allreduce_tallies()
    torch.cuda.synchronize()
    eng.reset_tallies()
    if args.mode in ("staged", "strip"):
        eng.profile_sampler(True)  # events around every sampler-phase (strip: whole-pass) launch
    launches0 = eng.launch_count()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev_run = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        flush.zero_()
        ev_run[i][0].record(stream)
        eng.run(args.warmup + i + 1, 1, word_begin, W)
        ev_run[i][1].record(stream)
        allreduce_tallies()
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = eng.launch_count() - launches0
    elapsed_ms = t_start.elapsed_time(t_end)
    run_ms = sum(a.elapsed_time(b) for a, b in ev_run)
    allreduced = None
    if world > 1:
        # the reduced counters equal the sum of every rank's own counters
        own = torch.tensor(eng.tallies()[0].astype(np.int64), device="cuda")
        parallel.allreduce_counters_(own)
        allreduced = bool(torch.equal(own, global_ones))
        local_ones = None
    if world > 1:
        elapsed_ms, run_ms = parallel.allreduce_max([elapsed_ms, run_ms])
    ms_per_step = elapsed_ms / args.steps
    samples = W * 64 * world
    value = g.n_gates * samples / (ms_per_step * 1e-3)
    be_words_per_s = g.n_be * W * world / (ms_per_step * 1e-3)

    # Roofline of the dominant kernel: basic-event words per launch / its mean
    # launch duration (CUDA events on its own stream), against the
    # register-only sampler measured on this GPU in this run.
    if args.mode in ("staged", "strip"):
        kernel = "k_stage_be" if args.mode == "staged" else "k_strip"
        n_a, ms_a = eng.profile_sampler_read()
        eng.profile_sampler(False)
        kernel_launches = max(n_a, 1)
        avg_launch_s = ms_a * 1e-3 / kernel_launches
    else:
        kernel = "k_fused" if args.mode == "fused" else "k_layer_be"
        kernel_launches = max(launches, 1) if args.mode == "fused" else args.steps
        avg_launch_s = run_ms * 1e-3 / kernel_launches
    be_words_per_launch = g.n_be * W * args.steps / kernel_launches
    achieved = be_words_per_launch / avg_launch_s
    peak = _capi.sampler_peak(n_events=256, n_words=args.peak_words, repeats=3, device=local)
    traffic = traffic_from_profile(kernel)

    # end to end: host descriptor -> engine (tables to HBM) -> one pass -> tallies to host
    e2e = None
    if args.e2e_steps > 0:
        ts, phases = [], []
        for i in range(args.e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2 = _capi.Engine(g, **eng_kw)
            t1 = time.perf_counter()
            e2.run(1, 1, word_begin, W)
            ones, total = e2.tallies()
            t2 = time.perf_counter()
            e2.close()
            t3 = time.perf_counter()
            ts.append(t3 - t0)
            phases.append({"create_s": t1 - t0, "pass_and_tallies_s": t2 - t1, "destroy_s": t3 - t2})
        if world > 1:
            ts = parallel.allreduce_max([max(ts)])
        e2e_s = statistics.median(ts)
        h2d = ((info["n_ops"] * 16 if args.mode == "fused" else 0) + g.n_be * 16 + g.n_gates * 20 +
               g.inputs.size * 4 + g.tally_nodes.size * 4)
        e2e = {"value": g.n_gates * samples / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(g.tally_nodes.size * 8), "seconds_per_step": e2e_s, "steps": phases}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_rate(g, args.cpu_seconds, reference=True)

    if rank == 0:
        peaks_file = ROOT / "MEASURED_PEAKS.json"
        hbm_peak = None
        if peaks_file.exists():
            hbm_peak = json.loads(peaks_file.read_text()).get("hbm_gbs")
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "plain MC pass, 5,000-event / 3,000-gate synthetic tree (seed 11)"
                       if args.tree == "config2" else "plain MC pass, 200-event / 100-gate synthetic tree (seed 372)",
                       "samples_per_gpu": W * 64, "words_per_gpu": W, "n_be": g.n_be, "n_gates": g.n_gates,
                       "tallied_nodes": int(g.tally_nodes.size), "parallelism": f"word-range shards x{world}",
                       "l2": "256 MB buffer written between steps", "mode": args.mode},
            "sample_words_per_s": be_words_per_s,
            "gpu_launches": int(launches),
            "roofline": {"bound": "int-alu", "kernel": kernel, "achieved": achieved / 1e9, "peak": peak / 1e9,
                         "unit": "Gword/s", "frac": achieved / peak, "traffic": traffic,
                         "launches": kernel_launches, "avg_launch_ms": avg_launch_s * 1e3,
                         "peak_source": "register-only Philox sampler kernel (k_sampler_peak) measured in this run",
                         "work_unit": "basic-event word = 16 Philox4x32-10 calls"},
            "pipeline": {"be_words_per_s": be_words_per_s, "frac_of_peak": be_words_per_s / world / peak},
            "tally_allreduce": None if world == 1 else {"backend": "nccl", "device_to_device": True,
                                                        "bytes_per_step": int(g.tally_nodes.size) * 8,
                                                        "sum_checked": allreduced},
            "clocks": clk,
            "program": info,
        }
        pipe = pipe_peak_from_profile()
        if pipe and clk.get("sm_mhz"):
            pk = pipe * clk["sm_mhz"] / 1960.0  # the pipe's rate follows the SM clock
            line["roofline_pipe"] = {"bound": "fmaheavy (integer multiply) pipe", "kernel": kernel,
                                     "achieved": achieved / 1e9, "peak": pk, "unit": "Gword/s",
                                     "frac": achieved / 1e9 / pk,
                                     "peak_source": "ncu: the sampler kernel's words/s over its fmaheavy pipe "
                                                    "utilisation (profiles/k_stage_be_config2.txt), scaled to "
                                                    "the median SM clock of this run"}
        if traffic and hbm_peak:
            line["roofline_hbm"] = {"achieved": traffic / avg_launch_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
                                    "frac": traffic / avg_launch_s / 1e9 / hbm_peak}
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
    eng.close()
    if rank == 0 and world == 1 and not args.no_is:
        # the metric's second half: learned-IS time to 5 % at P_top ~ 1e-8,
        # after the timed region (its own clocks inside)
        torch.cuda.set_stream(torch.cuda.default_stream())
        for key, tree in (("is", "read-once"), ("is_dag", "dag")):
            m = measure_is(args, local, tree)
            line[key] = {"workload": m["config"]["workload"], "metric": m["metric"], "wall_s": m["value"],
                         "unit": "s", **{k: v for k, v in m["is"].items() if k != "ce_rounds"},
                         "plain_samples_per_s": m["plain"]["samples_per_s"],
                         "plain_seconds_derived": m["plain"]["seconds"], "speedup_vs_plain": m["speedup"],
                         "warm_up": m["warm_up"], "clocks": m["clocks"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
