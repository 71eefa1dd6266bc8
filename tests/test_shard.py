"""Multi-rank host logic (noa_b200.shard) on the CPU: two gloo ranks, each computing its shard with the
C oracle. The all-reduced insertion equals the single-process one (up to the order of float sums) and
the gathered extraction is bit-identical; timings reduce with MAX."""
import json
import os
import socket
import subprocess
import sys

import pytest

from noa_b200.shard import shard_bounds

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle.oracle import fp_available  # noqa: E402


def test_shard_bounds_cover_and_balance():
    for n in (0, 1, 5, 7, 4096):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.skipif(not fp_available(), reason="oracle/libfp_oracle.so not built")
def test_two_gloo_ranks_shard_insert_and_extract(tmp_path):
    world = 2
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "shard_worker.py"),
                                       str(tmp_path / f"rank{rank}.json")], env=env))
    for p in procs:
        assert p.wait(timeout=180) == 0
    results = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert [tuple(r["insert_bounds"]) for r in results] == [(0, 4), (4, 7)]
    for r in results:
        assert r["insert_rel_l2"] <= 1e-6
        assert r["insert_w_rel_l2"] <= 1e-6
        assert r["extract_equal"]
        assert r["max"] == [1.0, 10.0]
