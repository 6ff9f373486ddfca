"""Multi-GPU use of the DMRG path: independent replicas, one process per GPU.

A two-site DMRG sweep is sequential (every step depends on the previous one),
so one problem does not shard across GPUs.  Several GPUs run independent
problems instead -- the independent chains of a batch, or N copies of the
same workload in the benchmark -- with no collective on the data path.
``torch.distributed`` (NCCL on GPUs, gloo on CPU) is used only for the
plumbing: a barrier, the max-over-ranks time and gathering the per-chain
results on rank 0.
"""
from __future__ import annotations

import os
from typing import Any, Callable, List, Sequence, Tuple


def world() -> Tuple[int, int]:
    """(rank, world size) from the launcher's environment (1 process if unset)."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def partition(n_items: int, world_size: int, rank: int) -> range:
    """Contiguous, balanced share of ``n_items`` for ``rank`` (sizes differ by at most 1)."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("bad rank / world size")
    base, extra = divmod(n_items, world_size)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of ``value`` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(obj: Any) -> List[Any]:
    """All ranks' objects on rank 0 (rank order), ``[obj]`` without a process group."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out if out is not None else []


def run_chains(items: Sequence[Any], solve: Callable[[Any], Any]) -> List[Any]:
    """Solve this rank's contiguous share of ``items``; rank 0 returns all
    results in item order, other ranks return []."""
    rank, size = world()
    mine = [(i, solve(items[i])) for i in partition(len(items), size, rank)]
    parts = gather_to_rank0(mine)
    if rank != 0:
        return []
    flat = sorted((p for part in parts for p in part), key=lambda t: t[0])
    return [r for _, r in flat]



def run_chains_concurrent(items: Sequence[Any], solve: Callable[[Any], Any], streams: int = 8,
                          device: int = 0) -> List[Any]:
    """Solve independent problems concurrently on one GPU.

    `streams` worker threads each create their own device context (a CUDA
    stream, the thread's plan cache and scalars), take items from a shared
    queue, and close the context when the queue is empty -- all on the same
    thread, since a context is bound to the thread that created it.  One DMRG
    sweep is a chain of small dependent launches that leaves most of the GPU
    idle, so independent chains on separate streams fill it; the C ABI
    releases the GIL inside every call.  `solve` must return plain values (no
    device objects, which belong to the worker's context).  Results come back
    in item order; the first exception raised by `solve` is re-raised."""
    import queue
    import threading

    import tt_b200

    todo: "queue.Queue" = queue.Queue()
    for k, it in enumerate(items):
        todo.put((k, it))
    out: List[Any] = [None] * len(items)
    errors: List[BaseException] = []

    def worker():
        try:
            ctx = tt_b200.Context(device)
        except BaseException as e:  # no device: report once
            errors.append(e)
            return
        try:
            while not errors:
                try:
                    k, it = todo.get_nowait()
                except queue.Empty:
                    break
                out[k] = solve(it)
        except BaseException as e:
            errors.append(e)
        finally:
            ctx.close()

    threads = [threading.Thread(target=worker, daemon=True) for _ in range(max(1, min(streams, len(items))))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return out
