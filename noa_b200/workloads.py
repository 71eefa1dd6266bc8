"""Secondary workloads, measured on one GPU; each prints one JSON line.

    python -m noa_b200.workloads batched   # uneven batched LANCZOS8 extraction (persistent kernel + graph)
    python -m noa_b200.workloads served    # Poisson stream of extract/insert requests through the server

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
    """12,000 extractions (LANCZOS8 by default) over 12 resident volumes (3 each of 128, 192, 256, 384;
    hc2h, cutoff 0.5), in `requests` requests (default 12, one per volume; request i reads volume
    i mod 12) whose slice counts are lognormal (median 1000, sigma 0.5, seeded) rescaled to 12,000.
    Legs: every request through the per-call API, the captured batch graph (ExtractBatch) and, for
    LINEAR, the same graph with every request in the persistent kernel (persistent_only) and one launch
    over resident pair copies of the volumes (extract_batch_launch), the form the serving loop uses."""
    import torch
    from . import fourier_project as fp
    from . import synthetic
    from .batch import ExtractBatch, ExtractRequest, extract_batch_launch, volume_pairs
    torch.cuda.set_device(0)
    rng = np.random.default_rng(args.seed)
    boxes = [128, 192, 256, 384] * 3
    n_req = getattr(args, "requests", None) or len(boxes)
    counts = rng.lognormal(mean=np.log(1000), sigma=0.5, size=n_req)
    counts = np.maximum(1, np.round(counts / counts.sum() * args.total)).astype(int)
    counts[-1] += args.total - counts.sum()
    vols = [torch.from_numpy(synthetic.make_volume(n, seed=args.seed + i)).cuda() for i, n in enumerate(boxes)]
    reqs = []
    for i, c in enumerate(counts):
        n = boxes[i % len(boxes)]
        rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(int(c), seed=args.seed + 100 + i)).cuda())
        out = torch.empty((int(c), 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        reqs.append(ExtractRequest(volume=vols[i % len(boxes)], volume_shape=(1, n, n, n), slice=out,
                                   slice_shape=(int(c), 1, n, n), fwd_rotation=rot))
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
    resident = persistent = None
    if args.interp == "linear":
        # the same batch with every request in the persistent kernel (no direct grids)
        pbatch = ExtractBatch("hc2h", reqs, interp=args.interp, autotune=not args.no_autotune, persistent_only=True)
        for _ in range(args.warmup):
            pbatch.run()
        torch.cuda.synchronize()
        t_pers = _timer(pbatch.run, args.steps, flush)
        persistent = {"ms": statistics.median(t_pers),
                      "speedup_vs_per_call": statistics.median(t_call) / statistics.median(t_pers)}
        pbatch.close()
        pairs_v = [volume_pairs(v, (1, n, n, n)) for v, n in zip(vols, boxes)]
        pairs = [pairs_v[i % len(boxes)] for i in range(len(reqs))]

        def launch():
            extract_batch_launch("hc2h", reqs, pairs, interp=args.interp)

        for _ in range(args.warmup):
            launch()
        torch.cuda.synchronize()
        t_res = _timer(launch, args.steps, flush)
        resident = {"value": total / (statistics.median(t_res) * 1e-3), "ms": statistics.median(t_res),
                    "speedup_vs_per_call": statistics.median(t_call) / statistics.median(t_res)}
    return {
        "workload": "batched uneven extraction",
        "config": {"boxes": sorted(set(boxes)), "volumes": len(boxes), "requests": len(reqs), "slices": total,
                   "slices_per_volume" if len(reqs) == len(boxes) else "slices_per_request": [int(c) for c in counts],
                   "interp": args.interp, "remap": "hc2h", "cutoff": 0.5, "l2": "flushed before each repetition"},
        "resident_pairs_launch": resident,
        "persistent_only_graph": persistent,
        "unit": "slices/s",
        "batched": {"value": total / (statistics.median(t_batch) * 1e-3), "ms": statistics.median(t_batch),
                    "launch": batch.info()},
        "per_call": {"value": total / (statistics.median(t_call) * 1e-3), "ms": statistics.median(t_call),
                     "launches": len(reqs)},
        "speedup_batched_vs_per_call": statistics.median(t_call) / statistics.median(t_batch),
        "steps": args.steps, "warmup": args.warmup, "data": "synthetic (seeded)",
    }


SERVED_BOXES = (128, 192, 256, 320, 384)


def _device_volume(n: int, gen, device):
    """synthetic.make_volume's distribution (hc layout), drawn on the device."""
    import torch
    wp = n // 2 + 1
    f = (torch.arange(n, device=device, dtype=torch.float32) - n // 2) / n
    fx = torch.arange(wp, device=device, dtype=torch.float32) / n
    norm = torch.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + fx[None, None, :] ** 2)
    amp = 1.0 / torch.clamp(norm, min=1.0 / 64)
    re = torch.randn((n, n, wp), generator=gen, device=device)
    im = torch.randn((n, n, wp), generator=gen, device=device)
    return (torch.complex(re, im) * (amp * (0.5 ** 0.5)))[None].contiguous()


def _device_slices(count: int, n: int, gen, device, bfactor: float = 100.0, centered: bool = False):
    """synthetic.make_slices's distribution, drawn on the device (non-centered or centered layout)."""
    import torch
    wp = n // 2 + 1
    i = torch.arange(n, device=device)
    fy = (i - n // 2 if centered else torch.where(i < (n + 1) // 2, i, i - n)).to(torch.float32) / n
    fx = torch.arange(wp, device=device, dtype=torch.float32) / n
    env = torch.exp(-bfactor * (fy[:, None] ** 2 + fx[None, :] ** 2) / 4)
    out = torch.empty((count, 1, n, wp), dtype=torch.complex64, device=device)
    for c0 in range(0, count, 1024):
        c1 = min(count, c0 + 1024)
        re = torch.randn((c1 - c0, n, wp), generator=gen, device=device)
        im = torch.randn((c1 - c0, n, wp), generator=gen, device=device)
        out[c0:c1, 0] = torch.complex(re, im) * (env * (0.5 ** 0.5))
    return out


def served(args) -> dict:
    """A Poisson stream of requests through ProjectionServer: ``--volumes`` resident volumes with boxes
    drawn uniformly from {128, 192, 256, 320, 384}; arrivals at ``--rate`` per second for ``--seconds``;
    256..8192 orientations per request, log-uniform; 70 % extraction (LINEAR, hc2h), 30 % insertion
    (rasterization, h2hc) into a per-request zeroed value + weight accumulator; ``--budget-gb`` of device
    memory for volumes and admitted requests. Insertion slices come from device-resident pools (one
    per box), orientations from a pinned host pool and are uploaded per request."""
    import torch
    from . import fourier_project as fp
    from . import synthetic
    from .serve import CudaExecutor, ProjectionServer, Request, latency_summary, run_stream
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(args.seed)
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed)
    boxes = [int(b) for b in rng.choice(SERVED_BOXES, size=args.volumes)]
    ex = CudaExecutor(dev, insert_streams=args.insert_streams, timing=args.timing)
    server = ProjectionServer(ex, int(args.budget_gb * 1e9), max_batch_slices=args.max_batch_slices,
                              max_inflight_batches=2, keep_outputs=False)
    for vid, n in enumerate(boxes):
        server.add_volume(vid, _device_volume(n, gen, dev), (1, n, n, n))
    pools = {n: _device_slices(args.pool, n, gen, dev) for n in sorted(set(boxes))}
    rot_pool = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(args.rot_pool, seed=args.seed + 7)))
    rot_pool = rot_pool.pin_memory()
    torch.cuda.synchronize()

    def make(t, rng_):
        kind = "extract" if rng_.random() < 0.7 else "insert"
        n_sl = int(round(float(np.exp(rng_.uniform(np.log(256), np.log(8192))))))
        vid = int(rng_.integers(len(boxes)))
        off = int(rng_.integers(0, args.rot_pool - n_sl + 1))
        slices = None
        if kind == "insert":
            s0 = int(rng_.integers(0, args.pool - n_sl + 1))
            slices = pools[boxes[vid]][s0:s0 + n_sl]
        return Request(kind, vid, rot_pool[off:off + n_sl], slices, arrival=t)

    # Warm-up (untimed): a few requests of each kind, drained.
    wrng = np.random.default_rng(args.seed + 1)
    for _ in range(8):
        server.submit(make(0.0, wrng))
    server.drain()
    ex.synchronize()

    reqs, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / args.rate))
        if t >= args.seconds:
            break
        reqs.append(make(t, rng))
    stats0 = dict(vars(server.stats))
    ex.spans.clear()
    ex.host_seconds = 0.0
    mem0 = torch.cuda.memory_stats(dev)
    t0, t1 = run_stream(server, reqs)
    ex.synchronize()
    mem1 = torch.cuda.memory_stats(dev)
    done = [r for r in reqs if r.error is None]
    total_slices = sum(r.n_slices for r in done)
    t_last = max(r.done for r in done)
    st = {k: v - stats0.get(k, 0) if k not in ("max_waiting", "peak_bytes") else v
          for k, v in vars(server.stats).items()}
    offered = sum(r.n_slices for r in reqs) / args.seconds
    return {
        "workload": "served stream",
        "config": {"volumes": args.volumes, "boxes": boxes, "rate_per_s": args.rate, "seconds": args.seconds,
                   "orientations": [256, 8192], "extract_fraction": 0.7, "interp": "linear",
                   "remaps": {"extract": "hc2h", "insert": "h2hc"}, "budget_gb": args.budget_gb,
                   "max_batch_slices": args.max_batch_slices, "insert_streams": args.insert_streams},
        "requests": len(reqs), "completed": len(done), "rejected": len(reqs) - len(done),
        "offered_slices_per_s": offered,
        "slices_per_s": total_slices / (t_last - t0),
        "makespan_s": t_last - t0,
        "latency": latency_summary(done),
        "latency_extract": latency_summary([r for r in done if r.kind == "extract"]),
        "latency_insert": latency_summary([r for r in done if r.kind == "insert"]),
        "server": {"batches": st["batches"], "mean_batch_requests": st["batch_requests"] / max(1, st["batches"]),
                   "mean_batch_slices": st["batch_slices"] / max(1, st["batches"]), "inserts": st["inserts"],
                   "max_waiting": st["max_waiting"], "peak_gb": st["peak_bytes"] / 1e9,
                   "resident_gb": server.resident / 1e9, "host_poll_s": st["poll_seconds"],
                   "host_launch_s": ex.host_seconds},
        "device": ex.busy_time(),
        "allocator": {k: mem1.get(k, 0) - mem0.get(k, 0) for k in ("num_alloc_retries", "num_device_alloc",
                                                                   "num_device_free", "num_sync_all_streams")},
        "latency_definition": "arrival to completion seen by the polling host loop (CUDA event query)",
        "data": "synthetic (seeded); insertion slices from device-resident pools",
    }


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("workload", choices=["batched", "served"])
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--total", type=int, default=12000)
    p.add_argument("--requests", type=int, default=None, help="batched: requests over the 12 volumes (default 12)")
    p.add_argument("--interp", default="lanczos8")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--volumes", type=int, default=32)
    p.add_argument("--rate", type=float, default=2000.0)
    p.add_argument("--seconds", type=float, default=60.0)
    p.add_argument("--budget-gb", type=float, default=120.0)
    p.add_argument("--max-batch-slices", type=int, default=65536)
    p.add_argument("--insert-streams", type=int, default=2)
    p.add_argument("--pool", type=int, default=8192, help="insertion slices per box in the device pool")
    p.add_argument("--rot-pool", type=int, default=65536)
    p.add_argument("--timing", action="store_true", help="bracket every launch with timed events")
    args = p.parse_args()
    result = {"batched": batched, "served": served}[args.workload](args)
    print(json.dumps(result), flush=True)


if __name__ == "__main__":
    sys.exit(main())
