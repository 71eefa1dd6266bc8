"""Secondary workloads, measured on one GPU; each prints one JSON line.

    python -m noa_b200.workloads batched   # uneven batched LANCZOS8 extraction (persistent kernel + graph)

Inputs are synthetic and seeded (no dataset is involved). Times are CUDA-event times on the launching
stream after warm-up, with an L2 flush (256 MB write) before every timed repetition.
"""
from __future__ import annotations

import argparse
import json
import statistics
import sys

import numpy as np

L2_FLUSH_BYTES = 256 << 20


def _timer(fn, reps: int, flush) -> list[float]:
    import torch
    times = []
    for _ in range(reps):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return times


def batched(args) -> dict:
    """12,000 LANCZOS8 extractions over 12 resident volumes (3 each of 128, 192, 256, 384; hc2h,
    cutoff 0.5), slice counts lognormal (median 1000, sigma 0.5, seeded) rescaled to 12,000."""
    import torch
    from . import fourier_project as fp
    from . import synthetic
    from .batch import ExtractBatch, ExtractRequest
    torch.cuda.set_device(0)
    rng = np.random.default_rng(args.seed)
    boxes = [128, 192, 256, 384] * 3
    counts = rng.lognormal(mean=np.log(1000), sigma=0.5, size=len(boxes))
    counts = np.maximum(1, np.round(counts / counts.sum() * args.total)).astype(int)
    counts[-1] += args.total - counts.sum()
    reqs = []
    for i, (n, c) in enumerate(zip(boxes, counts)):
        vol = torch.from_numpy(synthetic.make_volume(n, seed=args.seed + i)).cuda()
        rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(int(c), seed=args.seed + 100 + i)).cuda())
        out = torch.empty((int(c), 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        reqs.append(ExtractRequest(volume=vol, volume_shape=(1, n, n, n), slice=out, slice_shape=(int(c), 1, n, n),
                                   fwd_rotation=rot))
    flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def flush():
        flush_buf.fill_(1.0)

    def per_call():
        for r in reqs:
            fp.extract_central_slices_3d("hc2h", r.volume, None, r.volume_shape, r.slice, None, r.slice_shape,
                                         None, r.fwd_rotation, interp=args.interp)

    batch = ExtractBatch("hc2h", reqs, interp=args.interp, autotune=not args.no_autotune)
    for _ in range(args.warmup):
        per_call()
        batch.run()
    torch.cuda.synchronize()
    t_call = _timer(per_call, args.steps, flush)
    t_batch = _timer(batch.run, args.steps, flush)
    total = int(counts.sum())
    return {
        "workload": "batched uneven extraction",
        "config": {"boxes": sorted(set(boxes)), "volumes": len(boxes), "slices": total,
                   "slices_per_volume": [int(c) for c in counts], "interp": args.interp, "remap": "hc2h",
                   "cutoff": 0.5, "l2": "flushed before each repetition"},
        "unit": "slices/s",
        "batched": {"value": total / (statistics.median(t_batch) * 1e-3), "ms": statistics.median(t_batch),
                    "launch": batch.info()},
        "per_call": {"value": total / (statistics.median(t_call) * 1e-3), "ms": statistics.median(t_call),
                     "launches": len(reqs)},
        "speedup_batched_vs_per_call": statistics.median(t_call) / statistics.median(t_batch),
        "steps": args.steps, "warmup": args.warmup, "data": "synthetic (seeded)",
    }


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("workload", choices=["batched"])
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--total", type=int, default=12000)
    p.add_argument("--interp", default="lanczos8")
    p.add_argument("--no-autotune", action="store_true")
    args = p.parse_args()
    result = {"batched": batched}[args.workload](args)
    print(json.dumps(result), flush=True)


if __name__ == "__main__":
    sys.exit(main())
