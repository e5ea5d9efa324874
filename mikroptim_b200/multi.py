"""Several GPUs, one process per GPU: the variants (or LM runs) of a batch are independent, so
each rank works on its own contiguous range and the per-variant results are gathered in rank
order. There is no data-path collective; the only communication is the final gather of the
results (a few bytes per variant) over the process group.

The split follows the reference's MultiTraceEngine (split_variants,
include/mikroptim/cuda/multi_trace_engine.hpp:93): contiguous ranges whose sizes differ by at
most one, earlier ranks taking the larger ones.
"""

from __future__ import annotations

from typing import Callable

import numpy as np

from .batch import SystemBatchHost


def partition(count: int, world: int, rank: int) -> tuple[int, int]:
    """(first, size) of rank's contiguous share of `count` items."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"partition: rank {rank} of world {world}")
    if count < 0:
        raise ValueError("partition: count must be >= 0")
    base, extra = divmod(count, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def gather_rows(local: dict[str, np.ndarray], group=None) -> dict[str, np.ndarray]:
    """Concatenates every rank's per-variant arrays (leading axis) in rank order, on all ranks."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts: list = [None] * world
    dist.all_gather_object(parts, {k: np.asarray(v) for k, v in local.items()}, group=group)
    return {k: np.concatenate([p[k] for p in parts], axis=0) for k in local}


def run_sharded(batch: SystemBatchHost, fn: Callable[[SystemBatchHost, int], dict],
                group=None, x0: np.ndarray | None = None) -> dict[str, np.ndarray]:
    """Runs fn(shard, first) -- or fn(shard, first, x0_shard) when run points are given -- on
    this rank's contiguous share of the variants and gathers the per-variant results of all
    ranks. A batch of one variant shared by all runs (LM templates) is passed whole."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    count = batch.variants if x0 is None else len(x0)
    first, size = partition(count, world, rank)
    shard = batch if (x0 is not None and batch.variants == 1) else batch.subset(first, size)
    local = fn(shard, first) if x0 is None else fn(shard, first, np.asarray(x0)[first:first + size])
    return gather_rows(local, group)


def merit_sharded(batch: SystemBatchHost, settings, group=None,
                  merit: Callable | None = None) -> dict[str, np.ndarray]:
    """MERIT of all variants, each rank tracing its share on its own GPU.

    `merit(shard, settings) -> (merit, failed, hard_failed)` replaces the trace (default:
    TraceEngine.run in MERIT mode on the current device); the split and the gather are the
    same either way."""
    if merit is None:
        from .engine import TraceEngine, TraceMode
        import torch
        engine = TraceEngine(torch.cuda.current_device())

        def merit(shard, st):
            out = engine.run(shard, TraceMode.MERIT, st).merit
            return out.merit, out.failed, out.hard_failed

    def fn(shard, first):
        m, f, h = merit(shard, settings)
        return {"merit": m, "failed": f, "hard_failed": h}
    return run_sharded(batch, fn, group)


def optimize_lm_sharded(batch: SystemBatchHost, layout, variables, x0, options=None,
                        group=None, optimize: Callable | None = None) -> dict[str, np.ndarray]:
    """Batched LM of all runs, each rank optimising its share of the runs on its own GPU.

    `variables` is one VariableSet for all runs or a list of one per run (uneven batches: x0
    rows padded to the largest count; each rank gets its runs' sets).
    `optimize(shard, layout, variables, x_shard, options) -> dict` replaces the optimiser
    (default: optimize_lm_gpu on the current device)."""
    if optimize is None:
        from .engine import optimize_lm_gpu
        import torch

        def optimize(shard, lay, vs, x_shard, opt):
            return optimize_lm_gpu(shard, lay, vs, x_shard, opt,
                                   device=torch.cuda.current_device())
    per_run = isinstance(variables, (list, tuple))
    width = max(v.size for v in variables) if per_run else variables.size
    x0 = np.asarray(x0, dtype=np.float64).reshape(-1, width)

    def fn(shard, first, x_shard):
        vs = list(variables[first:first + len(x_shard)]) if per_run else variables
        out = optimize(shard, layout, vs, x_shard, options)
        return {k: v for k, v in out.items()
                if isinstance(v, np.ndarray) and v.ndim >= 1 and len(v) == len(x_shard)}
    return run_sharded(batch, fn, group, x0=x0)
