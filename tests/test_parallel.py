"""Multi-rank path on CPU: world-size-2 gloo ranks shard the sample words,
compute their tallies (the oracle stands in for each rank's device), and the
product's all-reduce gives exactly the single-rank tallies of the whole range."""
import os
import socket

import numpy as np
import pytest

from mcscram_b200 import parallel, synth


@pytest.mark.parametrize("count,world", [(0, 2), (1, 2), (7, 3), (16384, 2), (1000003, 8)])
def test_shard_words_partition(count, world):
    spans = [parallel.shard_words(123, count, world, r) for r in range(world)]
    pos = 123
    for b, c in spans:
        assert b == pos
        pos += c
    assert pos == 123 + count
    assert max(c for _, c in spans) - min(c for _, c in spans) <= 1


def test_weak_shard_bounds():
    assert parallel.weak_shard(1 << 24, 3) == (3 << 24, 1 << 24)
    with pytest.raises(ValueError):
        parallel.weak_shard(1 << 30, 4)


def test_shard_items_round_robin():
    parts = [parallel.shard_items(10, 3, r) for r in range(3)]
    assert sorted(sum(parts, [])) == list(range(10))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, words, queue):
    import torch.distributed as dist
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = synth.config1()
    b, c = parallel.shard_words(0, words, world, rank)
    local = oracle.tallies(g, 1, 1, b, c, threads=1)
    total = parallel.allreduce_tallies(local)
    slowest = parallel.allreduce_max([float(rank)])
    import torch
    in_place = parallel.allreduce_counters_(torch.from_numpy(local.astype(np.int64)))
    if rank == 0:
        queue.put((total, slowest, in_place.numpy().astype(np.uint64)))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_allreduce_equals_single_rank(oracle_mod):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    words = 3001
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, words, q)) for r in range(2)]
    for p in procs:
        p.start()
    total, slowest, in_place = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = oracle_mod.tallies(synth.config1(), 1, 1, 0, words)
    assert np.array_equal(total, expect)
    assert np.array_equal(in_place, expect)
    assert slowest == [1.0]


def test_bench_gpus_two_launches_two_ranks(oracle_mod):
    """`bench.py --gpus 2` without a launcher around it starts two ranks on
    this node (here the CPU reference arm: rank 0 measures and prints one
    line, rank 1 exits without work)."""
    import json
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "0", "--cpu-seconds", "0.2"], capture_output=True, text=True, env=env,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference"
    assert lines[0]["value"] > 0


def test_launcher_refuses_more_ranks_than_gpus():
    from mcscram_b200 import parallel
    import torch
    have = torch.cuda.device_count() if torch.cuda.is_available() else 0
    with pytest.raises(RuntimeError, match="GPUs"):
        parallel.launch_local_ranks(have + 1, "bench.py", [])
