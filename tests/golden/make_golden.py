"""Generates the committed golden fixtures from the reference's own sampler.

Run here, where the reference sources exist:  python tests/golden/make_golden.py

Every word in these fixtures comes from oracle/_ref/libref_mc.so, i.e. from
the reference's src/mc/prng/philox128.h compiled from its sources by
oracle/Makefile, driven through the reference dataflow restated in
oracle/mc_oracle.c.  The graphs are stored alongside so the fixtures do not
depend on the generator staying the same.

  philox_vectors.json      packed words for explicit counters and thresholds
  small_trees.npz          words of every node of small DAGs (all connectives)
  config1_tallies.npz      per-gate ones of config 1 at 2^20 samples (pass 1)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from mcscram_b200 import synth  # noqa: E402
from oracle import oracle  # noqa: E402


def graph_arrays(prefix: str, g) -> dict:
    return {f"{prefix}be_pdag_idx": g.be_pdag_idx, f"{prefix}be_event_idx": g.be_event_idx,
            f"{prefix}be_threshold": g.be_threshold, f"{prefix}gate_op": g.gate_op, f"{prefix}gate_k": g.gate_k,
            f"{prefix}gate_in_begin": g.gate_in_begin, f"{prefix}gate_in_count": g.gate_in_count,
            f"{prefix}gate_neg_count": g.gate_neg_count, f"{prefix}inputs": g.inputs,
            f"{prefix}tally_nodes": g.tally_nodes}


def main() -> None:
    if not oracle.has_reference_build():
        oracle.build(force=True)
    if not oracle.has_reference_build():
        raise SystemExit("oracle/_ref/libref_mc.so is missing: the reference sources are needed")

    rng = np.random.default_rng(20250601)
    vectors = []
    # The probe vector: counter {3, 1, 1, 128}, p = 0.5.
    cases = [((3, 1, 1, 128), 1 << 31)]
    thresholds = [0, 1, 2, 1 << 16, 1 << 31, (1 << 32) - 1, 1 << 32, 4294967, 42949672, 429496729]
    for thr in thresholds:
        cases.append(((3, 1, 1, 128), thr))
    for _ in range(200):
        c = tuple(int(x) for x in rng.integers(0, 1 << 32, size=4, dtype=np.uint64))
        thr = int(rng.integers(0, (1 << 32) + 1))
        cases.append((c, thr))
    for c, thr in cases:
        vectors.append({"counter": list(c), "threshold": thr, "word": oracle.word(*c, thr, reference=True)})
    # basic-event words at boundary positions of the counter layout
    be_cases = []
    for pdag in (2, 3, 1000, (1 << 31) - 2):
        for ev in (0, 1, 4999, (1 << 24) - 2, (1 << 32) - 2):
            for sample in (0, 1, (1 << 24) - 1, 1 << 24, (1 << 32) - 2):
                for it in (1, 2, 7, 1000):
                    thr = int(rng.integers(1, 1 << 32))
                    be_cases.append({"pdag_idx": pdag, "event_idx": ev, "sample_idx": sample, "iteration": it,
                                     "threshold": thr,
                                     "word": oracle.be_word(pdag, ev, sample, it, thr, reference=True)})
    (HERE / "philox_vectors.json").write_text(json.dumps({
        "source": "reference src/mc/prng/philox128.h compiled by oracle/Makefile",
        "packed": vectors, "basic_event": be_cases}, indent=1))

    # Small DAGs with every connective, negated inputs included.
    arrays = {}
    names = []
    for seed in range(6):
        g = synth.small_tree(seed, n_be=30, n_gates=16, p_range=(0.02, 0.6))
        # complement the last input of a few gates so negated inputs are covered
        neg = np.zeros(g.n_gates, dtype=np.uint32)
        for gi in range(g.n_gates):
            if g.gate_in_count[gi] >= 2 and gi % 3 == seed % 3:
                neg[gi] = 1
        g.gate_neg_count = neg
        name = f"t{seed}_"
        names.append(name)
        arrays.update(graph_arrays(name, g))
        arrays[name + "words_it1_w0"] = oracle.eval_words(g, 1, 0, 96, reference=True)
        arrays[name + "words_it3_whigh"] = oracle.eval_words(g, 3, (1 << 32) - 64, 64, reference=True)
    arrays["names"] = np.array(names)
    np.savez_compressed(HERE / "small_trees.npz", **arrays)

    # Config 1 at 2^20 samples: 16,384 words, pass 1.
    g1 = synth.config1()
    ones = oracle.tallies(g1, 1, 1, 0, 16384, reference=True)
    np.savez_compressed(HERE / "config1_tallies.npz", ones=ones, words=np.uint64(16384), iteration=np.uint32(1),
                        **graph_arrays("", g1))
    print("wrote", sorted(p.name for p in HERE.iterdir() if p.suffix in (".json", ".npz")))


if __name__ == "__main__":
    main()
