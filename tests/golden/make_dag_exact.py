"""Exact top-event probabilities of the rare-event trees with shared events
(synth.config4_dag and synth.config5_dag_instance 0..1023), by the FP64 BDD
of oracle/bdd_oracle.cc at the quantised probabilities the sampler draws.

Test infrastructure: the committed file config5_dag_exact.json is read by
the tests and by bench.py's accuracy check of the batched learned-IS
workload; an instance whose BDD exceeds the node limit is stored as null
(its estimate is then reported as not checked).

  python tests/golden/make_dag_exact.py [--workers N]
"""
from __future__ import annotations

import argparse
import json
import sys
from concurrent.futures import ProcessPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

N_INSTANCES = 1024
MAX_NODES = 40_000_000


def _exact(i: int):
    from mcscram_b200 import synth
    from oracle import oracle
    g = synth.config4_dag() if i < 0 else synth.config5_dag_instance(i)
    try:
        return i, oracle.bdd_probability(g, max_nodes=MAX_NODES), g.n_be, g.meta["approx_p_top"]
    except MemoryError:
        return i, None, g.n_be, g.meta["approx_p_top"]


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=8)
    args = ap.parse_args()
    import multiprocessing as mp
    with ProcessPoolExecutor(max_workers=args.workers, mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_exact, [-1] + list(range(N_INSTANCES)), chunksize=4))
    out = {"source": "oracle/bdd_oracle.cc (FP64 BDD) at the quantised probabilities, node limit "
                     f"{MAX_NODES}; null = limit exceeded",
           "config4_dag": res[0][1],
           "config5_dag": [r[1] for r in res[1:]],
           "config5_dag_events": [r[2] for r in res[1:]],
           "config5_dag_approx": [r[3] for r in res[1:]]}
    (HERE / "config5_dag_exact.json").write_text(json.dumps(out, indent=0) + "\n")
    n_none = sum(r[1] is None for r in res[1:])
    print(f"config4_dag {res[0][1]:.6e}; config5_dag: {N_INSTANCES - n_none} exact, {n_none} over the limit")
    return 0


if __name__ == "__main__":
    sys.exit(main())
