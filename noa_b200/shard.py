"""Multi-GPU sharding of the central-slice path: one process per GPU, slices split across ranks.

* Extraction is independent per slice: each rank extracts its shard of the orientations from its own
  replica of the volume; nothing is exchanged (``gather_slices`` assembles the shards where a caller
  wants them on one rank).
* Insertion (rasterization or gather insertion) is linear in the slices: each rank inserts its shard
  into zeroed partial value + weight grids and ONE sum all-reduce of the grids (12 bytes per rfft
  voxel: 101 MB at 256^3) gives every rank the full insertion. That is the reconstruction's only
  exchange step.
* Times are reduced with MAX over ranks (the job is as slow as its slowest rank).

The compute step is passed in, so the same host logic runs with the CUDA kernels on NCCL ranks and
with a CPU implementation on gloo ranks.
"""
from __future__ import annotations


def shard_bounds(n: int, world: int, rank: int) -> tuple[int, int]:
    """[start, stop) of rank's contiguous shard of n items; shard sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist
    return dist


def allreduce_grids(*grids, group=None) -> None:
    """Sums partial insertion grids across ranks in place (complex grids travel as their real view)."""
    import torch
    dist = _dist()
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return
    for g in grids:
        dist.all_reduce(torch.view_as_real(g) if g.is_complex() else g, op=dist.ReduceOp.SUM, group=group)


def max_over_ranks(values, device=None, group=None) -> list[float]:
    """Element-wise maximum of per-rank floats (timings) across ranks."""
    import torch
    dist = _dist()
    vals = [float(v) for v in values]
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return t.tolist()


def sharded_insert(insert_fn, n_slices: int, grids: tuple, group=None) -> tuple[int, int]:
    """Runs ``insert_fn(start, stop)`` — which must add slices [start, stop) into ``grids`` — on this
    rank's shard, then sums the grids across ranks. Returns the shard bounds."""
    dist = _dist()
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    start, stop = shard_bounds(n_slices, world, rank)
    if stop > start:
        insert_fn(start, stop)
    allreduce_grids(*grids, group=group)
    return start, stop


def gather_slices(local, n_slices: int, group=None):
    """Assembles per-rank extraction shards (contiguous, ``shard_bounds`` order) into the full stack on
    every rank. Shards are padded to the largest one for the collective and trimmed after."""
    import torch
    dist = _dist()
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return local
    world = dist.get_world_size(group)
    sizes = [b - a for a, b in (shard_bounds(n_slices, world, r) for r in range(world))]
    m = max(sizes)
    tail = tuple(local.shape[1:])
    padded = torch.zeros((m,) + tail, dtype=local.dtype, device=local.device)
    padded[:local.shape[0]] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    real = (lambda t: torch.view_as_real(t)) if local.is_complex() else (lambda t: t)
    dist.all_gather([real(p) for p in parts], real(padded), group=group)
    return torch.cat([p[:n] for p, n in zip(parts, sizes)], dim=0)
