"""CPU: bench.py's contract pieces that need no GPU — the reference arm's JSON line, its rank handling,
and the sizing of noa's CPU sample."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_cpu_sample_gives_every_thread_its_indices():
    import bench
    px = bench.N * (bench.N // 2 + 1)
    for threads in (1, 2, 8, 16, 48, 128):
        k = bench.cpu_sample_slices(threads)
        assert k % 32 == 0 and k >= 32
        assert k * px >= threads * bench.NOA_INDICES_PER_THREAD


def _run(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                          env=e, cwd=ROOT, timeout=600)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "libfp_oracle.so")),
                    reason="the oracle library is built by build()")
def test_reference_arm_prints_one_contract_line():
    r = _run(["--impl", "reference", "--steps", "1", "--warmup", "1", "--ref-batch", "32"])
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "slices/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] >= 1
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "slices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = _run(["--impl", "reference", "--steps", "1", "--warmup", "1", "--ref-batch", "32"],
             env={"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
