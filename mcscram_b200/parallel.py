"""Multi-GPU plumbing: sample-word sharding and the tally all-reduce.

Word w of a pass depends only on (pdag_idx, event_idx, w, pass) (mcSCRAM
src/mc/kernel/basic_event.h:112-122), so any partition of the word range
gives bit-identical words on every GPU, and tallies are plain sums.  Ranks
take contiguous word ranges (or whole instances for batched work) and the
only exchange is one all-reduce of the uint64 tallies per convergence step,
over NCCL (NVLink / NVSwitch) on GPUs or gloo on CPUs.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np


def shard_words(word_begin: int, word_count: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous, balanced share [begin, begin + count) of a word range for
    `rank` of `world` (the first word_count % world ranks get one more)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(word_count, world)
    begin = word_begin + rank * base + min(rank, extra)
    return begin, base + (1 if rank < extra else 0)


def weak_shard(words_per_rank: int, rank: int, word_begin: int = 0) -> Tuple[int, int]:
    """Fixed work per rank: rank r takes [begin + r * W, begin + (r + 1) * W)."""
    b = word_begin + rank * words_per_rank
    if b + words_per_rank > (1 << 32):
        raise ValueError("word range exceeds the 32-bit sample counter")
    return b, words_per_rank


def shard_items(n_items: int, world: int, rank: int) -> List[int]:
    """Round-robin assignment of independent items (trees, instances)."""
    return list(range(rank, n_items, world))


def launch_local_ranks(n: int, script: str, argv: Sequence[str], need_gpus: bool = True,
                       timeout_s: Optional[float] = None) -> int:
    """Runs `script argv` as n ranks on this node under torch.distributed.run
    (one process per GPU; RANK, LOCAL_RANK, WORLD_SIZE and MASTER_* set for
    each, rendezvous on 127.0.0.1) and returns the launcher's exit code.
    Refuses to start when `need_gpus` and fewer than n GPUs are visible."""
    import socket
    import subprocess
    import sys

    if n < 1:
        raise ValueError("at least one rank")
    if need_gpus:
        import torch
        have = torch.cuda.device_count() if torch.cuda.is_available() else 0
        if have < n:
            raise RuntimeError(f"{n} ranks need {n} GPUs; {have} visible")
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", script, *argv]
    return subprocess.run(cmd, timeout=timeout_s).returncode


def device_counters(ptr: int, n: int):
    """n uint64 counters in device memory at `ptr` (an engine's tallies,
    mcg_tally_device_ptr) as an int64 CUDA tensor over the same memory, no
    copy.  The memory stays the engine's: drop the tensor before the engine."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (int(n),), "typestr": "<i8", "data": (int(ptr), False),
                                    "version": 3, "strides": None}

    return torch.as_tensor(_View(), device="cuda")


def allreduce_counters_(counters, group=None):
    """In-place sum over ranks of an int64 tensor of counters, on its own
    device (CUDA tensors over NCCL, CPU tensors over gloo); the uint64 sums
    wrap the same way in two's complement, and tallies stay below 2^63."""
    import torch.distributed as dist

    dist.all_reduce(counters, op=dist.ReduceOp.SUM, group=group)
    return counters


def allreduce_tallies(ones: np.ndarray, group=None, device: Optional[str] = None) -> np.ndarray:
    """Sum of every rank's uint64 counters (tallies stay below 2^63)."""
    import torch
    import torch.distributed as dist

    a = np.ascontiguousarray(ones, dtype=np.uint64)
    if np.any(a >= np.uint64(1 << 63)):
        raise OverflowError("tally does not fit a signed 64-bit reduction")
    t = torch.from_numpy(a.astype(np.int64))
    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().astype(np.uint64)


def allreduce_max(values: Sequence[float], group=None, device: Optional[str] = None) -> List[float]:
    """Element-wise maximum over ranks (for timings: the slowest rank counts)."""
    import torch
    import torch.distributed as dist

    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(x) for x in t.cpu()]


def allgather_rows(feats: np.ndarray, targets: np.ndarray, group=None, device: Optional[str] = None):
    """Concatenates every rank's (features [n_r, F], targets [n_r]) rows in rank
    order, on every rank (for fitting one shared network to all ranks' trees).
    Ranks may hold different row counts; rows are padded to the largest."""
    import torch
    import torch.distributed as dist

    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    world = dist.get_world_size(group)
    feats = np.ascontiguousarray(feats, dtype=np.float32)
    targets = np.ascontiguousarray(targets, dtype=np.float32)
    rows = np.concatenate([feats, targets[:, None]], axis=1)
    n = torch.tensor([rows.shape[0]], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    width = rows.shape[1]
    pad = np.zeros((max(counts), width), dtype=np.float32)
    pad[: rows.shape[0]] = rows
    t = torch.from_numpy(pad).to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out = np.concatenate([parts[r].cpu().numpy()[: counts[r]] for r in range(world)])
    return np.ascontiguousarray(out[:, :-1]), np.ascontiguousarray(out[:, -1])


def broadcast_params(params: np.ndarray, src: int = 0, group=None, device: Optional[str] = None) -> np.ndarray:
    """Rank src's float32 parameter vector on every rank."""
    import torch
    import torch.distributed as dist

    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)).to(device)
    dist.broadcast(t, src=src, group=group)
    return t.cpu().numpy()
