"""One gloo rank of tests/test_shard.py: shards a rasterization and an extraction across ranks with
noa_b200.shard, computing each shard with the C oracle (CPU), and writes what it got to a JSON file.

Usage (environment: RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT): python tests/shard_worker.py OUT.json
"""
import json
import os
import sys
from datetime import timedelta

import numpy as np
import torch
import torch.distributed as dist

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from cases import build, clone, default_case, rel_l2  # noqa: E402
from oracle.oracle import FpOracle  # noqa: E402
from noa_b200 import shard  # noqa: E402


def sub_call(call, start, stop):
    c = clone(call)
    c.inp = np.ascontiguousarray(call.inp[start:stop])
    c.in_shape = (stop - start,) + tuple(call.in_shape[1:])
    c.rot = np.ascontiguousarray(call.rot[start:stop])
    return c


def main():
    out_path = sys.argv[1]
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    oracle = FpOracle()
    res = {"rank": rank, "world": world}

    # Insertion: each rank rasterizes its shard into zeroed partial grids; one all-reduce sums them.
    full = build(default_case("rasterize", remap="h2hc", n=24, nslices=7, out_w=True, seed=11))
    grid = torch.zeros(full.out.shape, dtype=torch.complex64)
    grid_w = torch.zeros(full.out_w.shape, dtype=torch.float32)

    def insert(start, stop):
        c = sub_call(full, start, stop)
        c.out = grid.numpy()
        c.out_w = grid_w.numpy()
        assert oracle.run(c) == 0

    bounds = shard.sharded_insert(insert, full.in_shape[0], (grid, grid_w))
    ref = clone(full)
    assert oracle.run(ref) == 0
    res["insert_bounds"] = list(bounds)
    res["insert_rel_l2"] = rel_l2(grid.numpy(), ref.out)
    res["insert_w_rel_l2"] = rel_l2(grid_w.numpy(), ref.out_w)

    # Extraction: each rank extracts its shard; the shards are gathered in order.
    ext = build(default_case("extract", remap="hc2h", n=24, nslices=5, seed=12))
    a, b = shard.shard_bounds(ext.out_shape[0], world, rank)
    mine = clone(ext)
    mine.rot = np.ascontiguousarray(ext.rot[a:b])
    mine.out = np.zeros((b - a,) + ext.out.shape[1:], dtype=ext.out.dtype)
    mine.out_shape = (b - a,) + tuple(ext.out_shape[1:])
    assert oracle.run(mine) == 0
    gathered = shard.gather_slices(torch.from_numpy(mine.out), ext.out_shape[0]).numpy()
    ref = clone(ext)
    assert oracle.run(ref) == 0
    res["extract_equal"] = bool(np.array_equal(gathered, ref.out))

    # Timings reduce with MAX.
    res["max"] = shard.max_over_ranks([float(rank), 10.0 - rank])
    dist.barrier()
    dist.destroy_process_group()
    with open(out_path, "w") as f:
        json.dump(res, f)


if __name__ == "__main__":
    main()
