"""Benchmark of the Fourier central-slice hot path on B200 (one JSON line on rank 0).

Workload (one step = one pass of the hot path over one batch):
  extract_central_slices_3d<"hc2h">   4096 slices of 256x129 complex64 from a 256^3 rfft volume (LINEAR, cutoff 0.5)
  rasterize_central_slices_3d<"h2hc"> 4096 slices of 256x129 complex64 into a 256^3 rfft volume + f32 weights
Synthetic, seeded inputs: volume amplitude 1/max(|f|,1/64), slices complex Gaussian x exp(-100 f^2/4),
uniform SO(3) orientations. Metric: slices/s (extract + insert slices per second, whole job).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload insert_512          # 512^3 x 20,000 windowed-sinc insertion, gather vs scatter
    python bench.py --workload insert_extract_256  # insert_and_extract, 4096 input -> 256 output slices
    python bench.py --workload batched             # 12,000 LANCZOS8 extractions, 12 volumes, one launch
    python bench.py --workload extract_wwindow_256 # 4096 extractions with a 7-sample w-windowed sinc
Each workload line carries noa's CPU path timed on this host beside it (cpu_baseline).

N > 1 runs under torchrun, one rank per GPU: every rank processes its own 4096 + 4096 slices (weak
scaling; extraction needs no exchange, and the insertion's partial grids are summed by one NCCL
all-reduce after the timed region, as a reconstruction does once at its end).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 256
SLICES = 4096
BFACTOR = 100.0
L2_FLUSH_BYTES = 256 << 20      # > 126 MB L2
REFERENCE_SECONDS = 150.0       # bound on the timed steps of the reference arm
E2E_CHUNKS = 16                 # slice chunks of the end-to-end step (overlapped copies; 16 vs 8: 26.5-26.9 vs 27.0-28.2 ms)


def algorithmic_bytes(n: int, b: int) -> dict:
    """Compulsory bytes per launch (volume/slices read or written once; Mat33 read once per slice)."""
    v = n * n * (n // 2 + 1)
    p = n * (n // 2 + 1)
    return {"extract": 8 * v + b * (8 * p + 48),
            "rasterize": b * (8 * p + 48) + 2 * (8 * v + 4 * v)}


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic() -> dict:
    """DRAM bytes per launch from the committed ncu summary (profiles/), if present."""
    path = os.path.join(ROOT, "profiles", "extract_rasterize_256.md")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            m = re.match(r"\s*traffic_bytes_per_launch\.(\w+)\s*[:=]\s*([0-9.eE+]+)", line)
            if m:
                out[m.group(1)] = float(m.group(2))
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def make_inputs(seed: int):
    import torch
    from noa_b200 import synthetic
    from noa_b200.fourier_project import pack_rotations
    dev = "cuda"
    vol = torch.from_numpy(synthetic.make_volume(N, seed=seed)).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 1)
    shape = (SLICES, 1, N, N // 2 + 1)
    re = torch.randn(shape, generator=g, device=dev)
    im = torch.randn(shape, generator=g, device=dev)
    env = torch.from_numpy(np.exp(-BFACTOR * synthetic.slice_fftfreq_norm((N, N), centered=False) ** 2 / 4)
                           .astype(np.float32)).to(dev)
    slices = (torch.complex(re, im) * (env / math.sqrt(2))).contiguous()
    del re, im
    rot_e = pack_rotations(torch.from_numpy(synthetic.random_rotations(SLICES, seed=seed + 2)).to(dev))
    rot_i = pack_rotations(torch.from_numpy(synthetic.random_rotations(SLICES, seed=seed + 3)).to(dev))
    return vol, slices, rot_e, rot_i


def run_gpu(args) -> None:
    import torch
    import torch.distributed as dist
    from noa_b200 import fourier_project as fp
    from noa_b200 import shard

    world, rank, local = dist_setup()
    vol, slices_in, rot_e, rot_i = make_inputs(seed=1000 * rank)
    out = torch.empty((SLICES, 1, N, N // 2 + 1), dtype=torch.complex64, device="cuda")
    grid = torch.zeros((1, N, N, N // 2 + 1), dtype=torch.complex64, device="cuda")
    grid_w = torch.zeros((1, N, N, N // 2 + 1), dtype=torch.float32, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    vshape, sshape = (1, N, N, N), (SLICES, 1, N, N)

    def extract():
        fp.extract_central_slices_3d("hc2h", vol, None, vshape, out, None, sshape, None, rot_e,
                                     fftfreq_cutoff=0.5, stream=stream)

    def rasterize():
        fp.rasterize_central_slices_3d("h2hc", slices_in, None, sshape, grid, grid_w, vshape, None, rot_i,
                                       fftfreq_cutoff=0.5, stream=stream)

    for _ in range(args.warmup):
        extract()
        rasterize()
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    refusals0 = fp.scratch_refusals()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.fill_(float(k))          # L2 flush between timed steps (outside the events)
            e0, e1, e2 = ev[k]
            e0.record(stream)
            extract()
            e1.record(stream)
            rasterize()
            e2.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    refusals = fp.scratch_refusals() - refusals0
    t_ext = [a.elapsed_time(b) for a, b, _ in ev]
    t_ras = [b.elapsed_time(c) for _, b, c in ev]
    step_ms = sum(t_ext + t_ras) / args.steps
    ext_ms, ras_ms = statistics.mean(t_ext), statistics.mean(t_ras)
    if world > 1:
        step_ms, ext_ms, ras_ms = shard.max_over_ranks([step_ms, ext_ms, ras_ms], device="cuda")
        # The reconstruction's one exchange: sum the per-rank partial grids (after the timed region).
        shard.allreduce_grids(grid, grid_w)
        torch.cuda.synchronize()

    # End to end through the public API with host buffers: H2D of the step's inputs (volume,
    # slices to insert, rotations) from pinned memory, both calls, D2H of the results. The step is cut
    # into E2E_CHUNKS slice chunks on three streams (copies in, compute, copies out), so the PCIe
    # transfers of both directions overlap each other and the kernels, as a streaming caller would.
    # (Issuing every extraction chunk first, so that their results stream out from the start, was
    # slower: 27.1 against 25.6 ms. Both directions at once run at ~47 GB/s each against 55-57 GB/s
    # alone, so the step is bound by its busier direction at the bidirectional rate, see pcie_gbs.)
    h_vol = vol.cpu().pin_memory()
    h_slices = slices_in.cpu().pin_memory()
    h_rot_e, h_rot_i = rot_e.cpu().pin_memory(), rot_i.cpu().pin_memory()
    h_out = torch.empty(out.shape, dtype=out.dtype).pin_memory()
    h_grid = torch.empty(grid.shape, dtype=grid.dtype).pin_memory()
    h_grid_w = torch.empty(grid_w.shape, dtype=grid_w.dtype).pin_memory()
    bi = (h_vol.numel() * 8 + h_slices.numel() * 8 + h_rot_e.numel() * 4 + h_rot_i.numel() * 4)
    bo = h_out.numel() * 8 + h_grid.numel() * 8 + h_grid_w.numel() * 4
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    bounds = [shard.shard_bounds(SLICES, E2E_CHUNKS, c) for c in range(E2E_CHUNKS)]

    def e2e_step():
        ev_small = torch.cuda.Event()
        ev_in = [torch.cuda.Event() for _ in bounds]
        ev_ext = [torch.cuda.Event() for _ in bounds]
        with torch.cuda.stream(s_in):
            vol.copy_(h_vol, non_blocking=True)
            rot_e.copy_(h_rot_e, non_blocking=True)
            rot_i.copy_(h_rot_i, non_blocking=True)
            ev_small.record(s_in)
            for (a, b), ev in zip(bounds, ev_in):
                slices_in[a:b].copy_(h_slices[a:b], non_blocking=True)
                ev.record(s_in)
        stream.wait_event(ev_small)
        for (a, b), e_in, e_ext in zip(bounds, ev_in, ev_ext):
            k = b - a
            fp.extract_central_slices_3d("hc2h", vol, None, vshape, out[a:b], None, (k, 1, N, N), None, rot_e[a:b],
                                         fftfreq_cutoff=0.5, stream=stream)
            e_ext.record(stream)
            s_out.wait_event(e_ext)
            with torch.cuda.stream(s_out):
                h_out[a:b].copy_(out[a:b], non_blocking=True)
            stream.wait_event(e_in)
            fp.rasterize_central_slices_3d("h2hc", slices_in[a:b], None, (k, 1, N, N), grid, grid_w, vshape, None,
                                           rot_i[a:b], fftfreq_cutoff=0.5, stream=stream)
        ev_done = torch.cuda.Event()
        ev_done.record(stream)
        s_out.wait_event(ev_done)
        with torch.cuda.stream(s_out):
            h_grid.copy_(grid, non_blocking=True)
            h_grid_w.copy_(grid_w, non_blocking=True)

    e2e_steps = max(2, min(args.e2e_steps, args.steps))
    e2e_ms = []
    torch.cuda.synchronize()
    for k in range(e2e_steps + 1):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        s_in.wait_event(s0)
        s_out.wait_event(s0)
        e2e_step()
        s1.record(s_out)
        torch.cuda.synchronize()
        if k > 0:
            e2e_ms.append(s0.elapsed_time(s1))
    e2e = statistics.mean(e2e_ms)
    if world > 1:
        e2e = shard.max_over_ranks([e2e], device="cuda")[0]
    pcie = pcie_bandwidth(h_slices, slices_in, h_out, out, s_in, s_out)

    if rank == 0:
        ab = algorithmic_bytes(N, SLICES)
        peaks = measured_peaks()
        traffic = profiled_traffic()
        dom = "rasterize" if ras_ms >= ext_ms else "extract"
        dom_ms = ras_ms if dom == "rasterize" else ext_ms
        achieved = ab[dom] / (dom_ms * 1e-3) / 1e9
        total_slices = 2 * SLICES * world
        line = {
            "metric": "slices/sec extract & insert at 256^3",
            "value": total_slices / (step_ms * 1e-3),
            "unit": "slices/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": step_ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded; no dataset)",
            "config": {"workload": "extract 4096 + rasterize 4096 slices of 256x129 c64, 256^3 rfft volume (+f32 weights)",
                       "volume": [N, N, N // 2 + 1], "slices_per_op": SLICES, "remaps": ["hc2h", "h2hc"],
                       "interp": "linear", "fftfreq_cutoff": 0.5, "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"slice shards x{world}"},
            "per_op": {"extract_ms": ext_ms, "rasterize_ms": ras_ms,
                       "extract_slices_per_s": SLICES * world / (ext_ms * 1e-3),
                       "insert_slices_per_s": SLICES * world / (ras_ms * 1e-3),
                       "extract_gbs": ab["extract"] / (ext_ms * 1e-3) / 1e9,
                       "rasterize_gbs": ab["rasterize"] / (ras_ms * 1e-3) / 1e9},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "peak_source": peaks["source"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "algorithmic_bytes": ab[dom], "traffic": traffic.get(dom),
                         # what ncu shows bounds the kernel on chip (HBM is not the limit of either)
                         "limiter": {"rasterize": "L2 tag requests of the scatter's reductions",
                                     "extract": "L1 data pipe of the tap gathers"}[dom]},
            "e2e": {"value": total_slices / (e2e * 1e-3), "unit": "slices/s", "h2d_bytes_per_step": bi,
                    "d2h_bytes_per_step": bo, "ms_per_step": e2e,
                    "schedule": f"{E2E_CHUNKS} slice chunks; copies in, kernels and copies out on 3 streams",
                    # the same pinned buffers copied alone and both directions at once: the e2e step moves
                    # max(Bi, Bo) bytes in its busier direction, so that / the bidirectional rate bounds it
                    "pcie_gbs": pcie,
                    "pcie_bound_ms": max(bi, bo) / (pcie["both_per_direction"] * 1e9) * 1e3},
            # per step: extract = pair copy + extraction kernel; rasterize = scatter kernel + finalize
            "gpu_launches": 4 * args.steps,
            # the library's own allocations refused during the timed steps (each a call on a slower path)
            "scratch_refusals": refusals,
            "clocks": clocks.summary(),
        }
        if not args.no_secondary and world == 1:
            line["secondary"] = secondary(args)
        if not args.no_cpu_baseline and world == 1:   # the CPU baseline is taken at N = 1 only
            line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def pcie_bandwidth(h_a, d_a, h_b, d_b, s_in, s_out, reps: int = 3) -> dict:
    """Pinned host<->device copy rates (GB/s) of the e2e buffers: h_a -> d_a alone, d_b -> h_b alone,
    and both at once on two streams (per direction: the smaller of the two bytes / elapsed)."""
    import torch

    def timed(fn, streams):
        best = 0.0
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = torch.cuda.Event(enable_timing=True)
            t0.record()
            done = []
            for s in streams:
                s.wait_event(t0)
            fn()
            for s in streams:
                e = torch.cuda.Event(enable_timing=True)
                e.record(s)
                done.append(e)
            torch.cuda.synchronize()
            best = max(best, 1.0 / max(t0.elapsed_time(e) for e in done))
        return best  # 1 / ms

    na = h_a.numel() * h_a.element_size()
    nb = h_b.numel() * h_b.element_size()

    def h2d():
        with torch.cuda.stream(s_in):
            d_a.copy_(h_a, non_blocking=True)

    def d2h():
        with torch.cuda.stream(s_out):
            h_b.copy_(d_b, non_blocking=True)

    def both():
        h2d()
        d2h()

    return {"h2d": na * timed(h2d, [s_in]) * 1e3 / 1e9, "d2h": nb * timed(d2h, [s_out]) * 1e3 / 1e9,
            "both_per_direction": min(na, nb) * timed(both, [s_in, s_out]) * 1e3 / 1e9,
            "bytes": [na, nb]}


# ---------------------------------------------------------------------------------------------------
# Secondary workloads of the default line, bounded to well under a minute: the small per-call case
# (64^3), the batched uneven LANCZOS8 and LINEAR extractions against their per-call forms in the same
# run, and the 512^3 windowed-sinc insertion on a subset of its slices, gather against scatter.
# ---------------------------------------------------------------------------------------------------
def _events_ms(fn, reps: int, warmup: int = 3, flush=None) -> float:
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def secondary(args) -> dict:
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic, workloads
    t_start = time.perf_counter()
    out = {}

    # 64^3: extract 64 slices (hc2h) then rasterize 64 slices (h2hc, + weights), one call each.
    n, b = 64, 64
    vol = torch.from_numpy(synthetic.make_volume(n, seed=0)).cuda()
    rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(b, seed=2)).cuda())
    sl = torch.empty((b, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grid = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grid_w = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.float32, device="cuda")
    ext = _events_ms(lambda: fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), sl, None, (b, 1, n, n),
                                                          None, rot), 50)
    ras = _events_ms(lambda: fp.rasterize_central_slices_3d("h2hc", sl, None, (b, 1, n, n), grid, grid_w,
                                                            (1, n, n, n), None, rot), 50)
    out["per_call_64"] = {"workload": "extract 64 slices of 64x33 c64 (hc2h) from a 64^3 rfft volume; rasterize "
                                      "them (h2hc) into 64^3 + f32 weights; LINEAR, cutoff 0.5",
                          "extract_ms": ext, "rasterize_ms": ras,
                          "slices_per_s": 2 * b / ((ext + ras) * 1e-3), "timing": "median of 50 calls, L2 warm"}
    del vol, sl, grid, grid_w

    # Batched uneven LANCZOS8: 12,000 extractions over 12 volumes of 128-384, graph vs per call.
    wargs = argparse.Namespace(seed=0, total=12000, interp="lanczos8", no_autotune=False, steps=3, warmup=2)
    r = workloads.batched(wargs)
    out["batched_lanczos8_12000"] = {
        "workload": "12,000 LANCZOS8 extractions (hc2h) over 12 volumes of 128, 192, 256, 384, lognormal slice "
                    "counts; one graph-captured persistent launch vs one call per request, same run",
        "batched_ms": r["batched"]["ms"], "per_call_ms": r["per_call"]["ms"],
        "batched_slices_per_s": r["batched"]["value"], "speedup_batched_vs_per_call": r["speedup_batched_vs_per_call"],
        "timing": "median of 3, L2 flushed before each"}
    torch.cuda.empty_cache()

    # Batched uneven LINEAR: the same 12,000 extractions as 12 and as 120 requests; in the graph, the
    # requests over pair copies run as grids of their own on parallel branches.
    for n_req in (12, 120):
        wargs = argparse.Namespace(seed=0, total=12000, interp="linear", no_autotune=False, steps=3, warmup=2,
                                   requests=n_req)
        r = workloads.batched(wargs)
        out[f"batched_linear_12000_{n_req}req"] = {
            "workload": f"12,000 LINEAR extractions (hc2h) over 12 volumes of 128, 192, 256, 384 as {n_req} "
                        "requests, lognormal slice counts; the captured batch graph vs one call per request, "
                        "same run (both rebuild the volumes' pair copies every run)",
            "batched_ms": r["batched"]["ms"], "per_call_ms": r["per_call"]["ms"],
            "persistent_only_ms": r["persistent_only_graph"]["ms"], "direct_grids": r["batched"]["launch"]["n_direct"],
            "speedup_batched_vs_per_call": r["speedup_batched_vs_per_call"],
            "timing": "median of 3, L2 flushed before each"}
        torch.cuda.empty_cache()

    # 512^3 windowed-sinc insertion (half-width 6 voxels), gather vs scatter form, on 1000 of the slices.
    n, k = 512, 1000
    wp = n // 2 + 1
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11)
    slices = workloads._device_slices(k, n, gen, torch.device("cuda"), bfactor=150.0, centered=True)
    rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(k, seed=16)).cuda())
    ws = fp.WindowedSinc(-1.0, 6.0 / n)
    grids = {}
    times = {}
    refused = {}
    for name, fn in (("gather", fp.insert_central_slices_3d), ("scatter", fp.insert_central_slices_3d_scatter)):
        v = torch.zeros((1, n, n, wp), dtype=torch.complex64, device="cuda")
        w = torch.zeros((1, n, n, wp), dtype=torch.float32, device="cuda")

        def call():
            fn("hc2hc", slices, None, (k, 1, n, n), v, w, (1, n, n, n), None, rot, interp="linear",
               windowed_sinc=ws, fftfreq_cutoff=0.5)

        r0 = fp.scratch_refusals()
        call()
        torch.cuda.synchronize()
        refused[name] = fp.scratch_refusals() - r0
        grids[name] = v.clone()
        times[name] = _events_ms(call, 3, warmup=0)
        del v, w
    x, y = grids["scatter"].to(torch.complex128), grids["gather"].to(torch.complex128)
    agree = (torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)).item()
    del grids, x, y, slices
    torch.cuda.empty_cache()
    out["insert_512_subset"] = {
        "workload": f"windowed-sinc insertion (half-width 6 voxels, LINEAR in-plane, hc2hc, + weights) of {k} of "
                    f"the 20,000 slices of 512x257 c64 into a 512^3 rfft volume",
        "gather_ms": times["gather"], "scatter_ms": times["scatter"],
        "gather_slices_per_s": k / (times["gather"] * 1e-3), "scatter_slices_per_s": k / (times["scatter"] * 1e-3),
        "scatter_vs_gather_rel_l2": agree,
        # a refused accumulator sends the scatter call to the gather form (the agreement is then exact;
        # it is also exact, with the accumulator, when every voxel's atomics arrive in slice order)
        "scatter_first_call_without_its_accumulator": refused["scatter"] > 0,
        "timing": "median of 3 accumulating calls"}
    out["seconds"] = time.perf_counter() - t_start
    return out


# ---------------------------------------------------------------------------------------------------
# CPU: noa's own CPU path (oracle/_ref, built from the reference sources) or the C restatement.
# ---------------------------------------------------------------------------------------------------
def _cpu_sample(batch: int, seed: int = 7):
    from noa_b200 import synthetic
    from oracle.oracle import Call
    vol = synthetic.make_volume(N, seed=seed)
    slices = synthetic.make_slices(batch, N, seed=seed + 1, bfactor=BFACTOR)
    rot_e = synthetic.random_rotations(batch, seed=seed + 2)
    rot_i = synthetic.random_rotations(batch, seed=seed + 3)
    ext = Call(func="extract", remap="hc2h", inp=vol, in_shape=(1, N, N, N),
               out=np.zeros((batch, 1, N, N // 2 + 1), np.complex64), out_shape=(batch, 1, N, N), rot=rot_e)
    ras = Call(func="rasterize", remap="h2hc", inp=slices, in_shape=(batch, 1, N, N),
               out=np.zeros((1, N, N, N // 2 + 1), np.complex64), out_shape=(1, N, N, N), rot=rot_i,
               out_w=np.zeros((1, N, N, N // 2 + 1), np.float32))
    return ext, ras


def _cpu_impl():
    from oracle.oracle import FpOracle, RefLib, ref_available
    if ref_available():
        lib = RefLib()
        return "reference", (lambda call, thr: lib.run(call, thr)[0])
    lib = FpOracle()
    return "port", (lambda call, thr: lib.run(call, thr))


# noa's CPU backend gives each thread at least 2^20 indices (runtime/Iwise.hpp:34-35) and runs a call
# serially below that, so a sample must hold threads x 2^20 pixels for noa to use every host thread.
NOA_INDICES_PER_THREAD = 1 << 20


def cpu_sample_slices(threads: int) -> int:
    """Slices per CPU call: enough pixels for noa to spread a call over `threads`, a multiple of 32."""
    need = -(-threads * NOA_INDICES_PER_THREAD // (N * (N // 2 + 1)))
    return max(32, -(-need // 32) * 32)


def cpu_baseline(seconds: float) -> dict:
    """noa's CPU path timed on this host's cores over a bounded sample of the workload."""
    kind, run = _cpu_impl()
    threads = os.cpu_count() or 1
    batch = cpu_sample_slices(threads)
    ext, ras = _cpu_sample(batch)
    run(ext, threads)           # warm-up
    run(ras, threads)
    done, t0, iters = 0, time.perf_counter(), []
    while time.perf_counter() - t0 < seconds or len(iters) < 5:
        ti = time.perf_counter()
        run(ext, threads)
        run(ras, threads)
        iters.append(time.perf_counter() - ti)
        done += 2 * batch
    dt = time.perf_counter() - t0
    # the same sample on one thread, over a quarter of the time
    done1, t1 = 0, time.perf_counter()
    while time.perf_counter() - t1 < seconds / 4:
        run(ext, 1)
        run(ras, 1)
        done1 += 2 * batch
    dt1 = time.perf_counter() - t1
    return {"value": 2 * batch / statistics.median(iters), "unit": "slices/s", "cores": threads, "kind": kind,
            "value_1_thread": done1 / dt1, "cpu_model": _cpu_model(),
            "sample": f"median of {len(iters)} repetitions; "
                      f"{done} slices ({batch}-slice extract + {batch}-slice rasterize calls, 256^3, "
                      f"{dt:.1f} s, threads={threads}; {batch} slices per call so that noa spreads each call "
                      f"over all threads (it gives a thread at least 2^20 pixels); rasterize runs with noa's "
                      f"per-float omp atomics); 1 thread: {done1} slices in {dt1:.1f} s"}


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    kind, run = _cpu_impl()
    threads = os.cpu_count() or 1
    batch = args.ref_batch or cpu_sample_slices(threads)
    ext, ras = _cpu_sample(batch)
    t0 = time.perf_counter()
    for _ in range(max(args.warmup, 1)):
        run(ext, threads)
        run(ras, threads)
    per_step = (time.perf_counter() - t0) / max(args.warmup, 1)
    # K steps of a sample large enough for noa's threading can take long: keep the run within about
    # three minutes, and report the number of steps timed.
    steps = min(args.steps, max(3, int(REFERENCE_SECONDS / max(per_step, 1e-6))))
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        run(ext, threads)
        run(ras, threads)
        times.append(time.perf_counter() - t0)
    step = statistics.mean(times)
    value = 2 * batch / step
    print(json.dumps({
        "impl": "reference",
        "metric": "slices/sec extract & insert at 256^3",
        "value": value, "unit": "slices/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": steps, "steps_requested": args.steps, "warmup": max(args.warmup, 1), "ms_per_step": step * 1e3,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no dataset)",
        "config": {"workload": "extract + rasterize slices of 256x129 c64, 256^3 rfft volume (+f32 weights)",
                   "slices_per_op_per_step": batch, "remaps": ["hc2h", "h2hc"], "interp": "linear"},
        "cpu_baseline": {"value": value, "unit": "slices/s", "cores": threads, "kind": kind,
                         "sample": f"{batch}-slice extract + {batch}-slice rasterize per step, {threads} threads "
                                   f"({batch} slices per call so that noa spreads each call over all threads)"},
        "e2e": {"value": value, "unit": "slices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------------------------------
# Second workload: windowed-sinc insertion at 512^3 (gather form vs slice-major scatter form).
# ---------------------------------------------------------------------------------------------------
def run_large(args) -> None:
    """insert_central_slices_3d<"hc2hc">: 20,000 slices of 512x257 c64 (complex Gaussian x
    exp(-150 f^2/4), centered) into a zeroed 512^3 rfft value + weight grid, LINEAR in-plane,
    WindowedSinc{-1, 6/512} (half-width 6 voxels), cutoff 0.5. Times the deterministic gather form and
    the atomic scatter form (same terms) and checks they agree. The reference's CPU loop is
    O(voxels x slices), so it is timed on a few slices of the full volume and scaled linearly."""
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    from noa_b200.workloads import _device_slices
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n, nsl = args.n, args.slices
    wp = n // 2 + 1
    gen = torch.Generator(device=dev)
    gen.manual_seed(11)
    slices = _device_slices(nsl, n, gen, dev, bfactor=150.0, centered=True)
    rot_h = synthetic.random_rotations(nsl, seed=16)
    rot = fp.pack_rotations(torch.from_numpy(rot_h).to(dev))
    ws = fp.WindowedSinc(-1.0, 6.0 / n)
    vshape, sshape = (1, n, n, n), (nsl, 1, n, n)
    times, grids = {}, {}
    with ClockSampler(0) as clocks:
        for name, fn in (("gather", fp.insert_central_slices_3d), ("scatter", fp.insert_central_slices_3d_scatter)):
            v = torch.zeros((1, n, n, wp), dtype=torch.complex64, device=dev)
            w = torch.zeros((1, n, n, wp), dtype=torch.float32, device=dev)

            def call():
                fn("hc2hc", slices, None, sshape, v, w, vshape, None, rot, interp="linear", windowed_sinc=ws,
                   fftfreq_cutoff=0.5)

            call()
            torch.cuda.synchronize()
            grids[name] = (v.clone(), w.clone())
            ts = []
            for _ in range(args.steps):
                v.zero_()
                w.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                call()
                b.record()
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b))
            times[name] = statistics.median(ts)
            del v, w

    def rl2(x, y):
        x = x.to(torch.complex128) if x.is_complex() else x.to(torch.float64)
        y = y.to(x.dtype)
        return (torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)).item()

    agree = {"values_rel_l2": rl2(grids["scatter"][0], grids["gather"][0]),
             "weights_rel_l2": rl2(grids["scatter"][1], grids["gather"][1])}
    del grids
    best = min(times, key=times.get)
    alg = nsl * (8 * n * wp + 48) + 2 * 12 * n * n * wp
    peaks = measured_peaks()
    achieved = alg / (times[best] * 1e-3) / 1e9
    line = {
        "metric": f"slices/sec windowed-sinc insert at {n}^3", "value": nsl / (times[best] * 1e-3),
        "unit": "slices/s", "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": times[best],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": f"insert {nsl} slices of {n}x{wp} c64 into a {n}^3 rfft volume + f32 weights, "
                               f"windowed sinc half-width 6, hc2hc, LINEAR", "form": best},
        "forms": {k: {"ms": t, "slices_per_s": nsl / (t * 1e-3)} for k, t in times.items()},
        "scatter_vs_gather": agree,
        "roofline": {"bound": "hbm", "kernel": f"insert ({best})", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "peak_source": peaks["source"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "algorithmic_bytes": alg, "traffic": None},
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = _large_cpu_baseline(slices[:args.ref_slices].cpu().numpy(),
                                                   rot_h[:args.ref_slices], n, nsl)
    print(json.dumps(line), flush=True)


def _large_cpu_baseline(h_slices, h_rot, n: int, total: int) -> dict:
    from oracle.oracle import Call
    kind, run = _cpu_impl()
    k = h_slices.shape[0]
    wp = n // 2 + 1
    c = Call(func="insert", remap="hc2hc", inp=h_slices, in_shape=(k, 1, n, n),
             out=np.zeros((1, n, n, wp), dtype=np.complex64), out_shape=(1, n, n, n),
             rot=h_rot.astype(np.float32), out_w=np.zeros((1, n, n, wp), dtype=np.float32), interp=1,
             cutoff=0.5, sinc=(-1.0, 6.0 / n))
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    run(c, threads)
    dt = time.perf_counter() - t0
    return {"value": k / dt, "unit": "slices/s", "cores": threads, "kind": kind,
            "sample": f"{k} of the {total} slices into the full {n}^3 volume in {dt:.1f} s, threads={threads}; "
                      f"noa's loop visits every (voxel, slice) pair, so its time is linear in the slice count "
                      f"and the rate extrapolates to the full job"}


# ---------------------------------------------------------------------------------------------------
# Third workload: insert_and_extract_central_slices_3d at large slice counts (no volume in between).
# ---------------------------------------------------------------------------------------------------
def run_insert_extract(args) -> None:
    """insert_and_extract_central_slices_3d<"h2h">: 4096 input slices of 256x129 c64 (complex Gaussian
    x exp(-100 f^2/4)) are inserted into a virtual 256^3 volume and 256 output slices extracted from it,
    LINEAR in-plane, the default input windowed sinc (half-width one voxel), cutoff 0.5, output weights
    f32. Orientations uniform on SO(3). The reference's CPU loop visits every (output pixel, input
    slice) pair, so it is timed on a few output slices and scaled linearly."""
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    from noa_b200.workloads import _device_slices
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n, n_in, n_out = args.n, args.slices, args.out_slices
    wp = n // 2 + 1
    gen = torch.Generator(device=dev)
    gen.manual_seed(21)
    inp = _device_slices(n_in, n, gen, dev, bfactor=100.0, centered=False)
    rot_in_h = np.ascontiguousarray(np.transpose(synthetic.random_rotations(n_in, seed=22), (0, 2, 1)))
    rot_out_h = synthetic.random_rotations(n_out, seed=23)
    rot_in = fp.pack_rotations(torch.from_numpy(rot_in_h).to(dev))
    rot_out = fp.pack_rotations(torch.from_numpy(rot_out_h).to(dev))
    out = torch.zeros((n_out, 1, n, wp), dtype=torch.complex64, device=dev)
    out_w = torch.zeros((n_out, 1, n, wp), dtype=torch.float32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def call():
        fp.insert_and_extract_central_slices_3d("h2h", inp, None, (n_in, 1, n, n), out, out_w, (n_out, 1, n, n),
                                                None, rot_in, None, rot_out, interp="linear")

    for _ in range(max(args.warmup, 3)):
        call()
    torch.cuda.synchronize()
    ts = []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            call()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
    ms = statistics.median(ts)
    alg = n_in * (8 * n * wp + 48) + n_out * (12 * n * wp + 48)
    peaks = measured_peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    line = {
        "metric": f"output slices/sec insert_and_extract at {n}^3", "value": n_out / (ms * 1e-3),
        "unit": "slices/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": f"insert {n_in} slices of {n}x{wp} c64 and extract {n_out} (+f32 weights), "
                               f"h2h, LINEAR, default windowed sinc", "l2": "flushed between steps"},
        "input_slices_per_s": n_in / (ms * 1e-3),
        "roofline": {"bound": "hbm", "kernel": "insert_extract_kernel", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "peak_source": peaks["source"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "algorithmic_bytes": alg, "traffic": None},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        k = args.ref_slices
        line["cpu_baseline"], ref_out, ref_w = _insert_extract_cpu_baseline(
            inp.cpu().numpy(), rot_in_h, rot_out_h[:k], n, n_out)
        # the CPU sample is the first k output slices of the same job: compare them
        o, ow = out[:k].cpu().numpy().astype(np.complex128), out_w[:k].cpu().numpy().astype(np.float64)
        line["cpu_sample_rel_l2"] = {
            "values": float(np.linalg.norm(o - ref_out) / np.linalg.norm(ref_out)),
            "weights": float(np.linalg.norm(ow - ref_w) / np.linalg.norm(ref_w))}
    print(json.dumps(line), flush=True)


def _insert_extract_cpu_baseline(h_in, h_rot_in, h_rot_out, n: int, total: int) -> dict:
    from oracle.oracle import Call
    kind, run = _cpu_impl()
    k = h_rot_out.shape[0]
    b = h_in.shape[0]
    wp = n // 2 + 1
    c = Call(func="insert_extract", remap="h2h", inp=h_in, in_shape=(b, 1, n, n),
             out=np.zeros((k, 1, n, wp), dtype=np.complex64), out_shape=(k, 1, n, n),
             rot=h_rot_in.astype(np.float32), rot2=h_rot_out.astype(np.float32),
             out_w=np.zeros((k, 1, n, wp), dtype=np.float32), interp=1, cutoff=0.5)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    run(c, threads)
    dt = time.perf_counter() - t0
    # noa gives a thread at least 2^20 output pixels, so a call over k < 32 output slices of 256x129 runs
    # on one thread, and any call of >= 32 slices takes as long as one thread's 32 slices (over a minute
    # here). The sample is therefore serial; its rate times the host's threads bounds noa's parallel rate.
    used = max(1, min(threads, (k * n * wp) // NOA_INDICES_PER_THREAD))
    return ({"value": k / dt, "unit": "slices/s", "cores": used, "kind": kind,
             "value_all_threads_bound": k / dt * threads / used, "host_threads": threads,
             "sample": f"{k} of the {total} output slices from all {b} input slices in {dt:.1f} s; noa ran it "
                       f"on {used} thread(s) (it gives a thread at least 2^20 output pixels); its loop visits "
                       f"every (output pixel, input slice) pair, so its time is linear in the output slice "
                       f"count and the rate extrapolates to the full job; value_all_threads_bound assumes "
                       f"perfect scaling over the {threads} host threads"},
            c.out.astype(np.complex128), c.out_w.astype(np.float64))


# ---------------------------------------------------------------------------------------------------
# w-windowed-sinc extraction (noa's 4-D FourierExtract): every pixel sums the windowed samples of a
# short z window of the volume.
# ---------------------------------------------------------------------------------------------------
WW_SINC, WW_BLACKMAN = 2.0, 4.0   # in voxels of the z axis: fftfreq 2/256 and 4/256 (a 7-sample window)


def run_extract_wwindow(args) -> None:
    """extract_central_slices_3d<"hc2h"> of 4096 slices of 256x129 c64 from a 256^3 volume, LINEAR, with
    the w-windowed sinc {fftfreq_sinc 2/256, fftfreq_blackman 4/256} (7 z samples per pixel), cutoff 0.5.
    noa's CPU path runs the first slices of the same job beside it, and they are compared."""
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n, nsl = args.n, args.slices
    wp = n // 2 + 1
    h_vol = synthetic.make_volume(n, seed=31)
    vol = torch.from_numpy(h_vol).to(dev)
    rot_h = synthetic.random_rotations(nsl, seed=32)
    rot = fp.pack_rotations(torch.from_numpy(rot_h).to(dev))
    out = torch.empty((nsl, 1, n, wp), dtype=torch.complex64, device=dev)
    wws = fp.WindowedSinc(WW_SINC / n, WW_BLACKMAN / n)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def call():
        fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), out, None, (nsl, 1, n, n), None, rot,
                                     interp="linear", w_windowed_sinc=wws)

    for _ in range(max(args.warmup, 3)):
        call()
    torch.cuda.synchronize()
    ts = []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            call()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
    ms = statistics.median(ts)
    alg = 8 * n * n * wp + nsl * (8 * n * wp + 48)
    peaks = measured_peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    line = {
        "metric": f"slices/sec w-windowed extraction at {n}^3", "value": nsl / (ms * 1e-3), "unit": "slices/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": f"extract {nsl} slices of {n}x{wp} c64 from a {n}^3 rfft volume, hc2h, LINEAR, "
                               f"w-windowed sinc {{{WW_SINC:g}/{n}, {WW_BLACKMAN:g}/{n}}} (7 z samples per pixel)",
                   "l2": "flushed between steps"},
        "roofline": {"bound": "hbm", "kernel": "extract_kernel", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "peak_source": peaks["source"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                     "algorithmic_bytes": alg, "traffic": None},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        from oracle.oracle import Call
        kind, run = _cpu_impl()
        threads = os.cpu_count() or 1
        # noa iterates (slice, w, y, x) and gives a thread at least 2^20 of them
        k = min(nsl, max(8, -(-threads * NOA_INDICES_PER_THREAD // (7 * n * wp))))
        c = Call(func="extract", remap="hc2h", inp=h_vol, in_shape=(1, n, n, n),
                 out=np.zeros((k, 1, n, wp), np.complex64), out_shape=(k, 1, n, n), rot=rot_h[:k],
                 interp=1, cutoff=0.5, w_sinc=(WW_SINC / n, WW_BLACKMAN / n))
        t0 = time.perf_counter()
        run(c, threads)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": k / dt, "unit": "slices/s", "cores": threads, "kind": kind,
                                "sample": f"the first {k} of the {nsl} slices in {dt:.1f} s, threads={threads}"}
        o = out[:k].cpu().numpy().astype(np.complex128)
        ref = c.out.astype(np.complex128)
        line["cpu_sample_rel_l2"] = float(np.linalg.norm(o - ref) / np.linalg.norm(ref))
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------------
# Fourth workload: batched uneven LANCZOS8 extraction (persistent kernel in a CUDA graph).
# ---------------------------------------------------------------------------------------------------
def run_batched(args) -> None:
    """12,000 LANCZOS8 extractions over 12 resident volumes of 128-384 (noa_b200.workloads.batched):
    the graph-captured persistent launch against per-call launches, with noa's CPU path beside it."""
    import torch
    from noa_b200 import workloads
    wargs = argparse.Namespace(seed=0, total=args.slices, interp="lanczos8", no_autotune=False,
                               steps=args.steps, warmup=max(args.warmup, 3))
    r = workloads.batched(wargs)
    boxes = [128, 192, 256, 384] * 3
    counts = r["config"]["slices_per_volume"]
    alg = sum(8 * n * n * (n // 2 + 1) + c * (8 * n * (n // 2 + 1) + 48) for n, c in zip(boxes, counts))
    ms = r["batched"]["ms"]
    peaks = measured_peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    line = {
        "metric": "slices/sec batched uneven LANCZOS8 extraction", "value": r["batched"]["value"],
        "unit": "slices/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": f"{sum(counts)} LANCZOS8 extractions (hc2h, cutoff 0.5) over 12 volumes of "
                               f"128-384 in one graph-captured persistent launch", **r["config"]},
        "per_call": r["per_call"], "speedup_batched_vs_per_call": r["speedup_batched_vs_per_call"],
        "launch": r["batched"]["launch"],
        "roofline": {"bound": "hbm", "kernel": "batch_extract_kernel", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "peak_source": peaks["source"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "algorithmic_bytes": alg, "traffic": None},
        "gpu_launches": args.steps,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = _batched_cpu_baseline(boxes, counts)
    print(json.dumps(line), flush=True)


def _batched_cpu_baseline(boxes, counts, pixels_per_box: int = 200_000) -> dict:
    """noa's CPU LANCZOS8 extraction timed per box size on a serial sample (fewer than 2^20 pixels, so
    noa runs it on one thread), then the full job's time as the sum over volumes of count x time per
    slice of its box."""
    from noa_b200 import synthetic
    from oracle.oracle import Call, INTERPS
    kind, run = _cpu_impl()
    per_slice, notes = {}, []
    for n in sorted(set(boxes)):
        wp = n // 2 + 1
        k = max(1, pixels_per_box // (n * wp))
        vol = synthetic.make_volume(n, seed=n)
        c = Call(func="extract", remap="hc2h", inp=vol, in_shape=(1, n, n, n),
                 out=np.zeros((k, 1, n, wp), np.complex64), out_shape=(k, 1, n, n),
                 rot=synthetic.random_rotations(k, seed=n + 1), interp=INTERPS["lanczos8"])
        t0 = time.perf_counter()
        run(c, 1)
        per_slice[n] = (time.perf_counter() - t0) / k
        notes.append(f"{n}: {k} slices, {per_slice[n] * 1e3:.0f} ms/slice")
    job = sum(c * per_slice[n] for n, c in zip(boxes, counts))
    threads = os.cpu_count() or 1
    return {"value": sum(counts) / job, "unit": "slices/s", "cores": 1, "kind": kind,
            "value_all_threads_bound": sum(counts) / job * threads, "host_threads": threads,
            "sample": "per box, one serial call (noa runs calls under 2^20 pixels on one thread): "
                      + "; ".join(notes) + f"; job time = sum of count x time per slice = {job:.0f} s; "
                      f"value_all_threads_bound assumes perfect scaling over {threads} threads"}


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=400)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["noa_b200", "reference"], default="noa_b200")
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-secondary", action="store_true",
                   help="skip the secondary workloads of the default line (64^3 per call, batched LANCZOS8, "
                        "512^3 insertion subset)")
    p.add_argument("--ref-batch", type=int, default=None,
                   help="slices per CPU call of the reference arm (default: enough for noa to use every thread)")
    p.add_argument("--n", type=int, default=None, help="box size (default 256, or 512 for insert_512)")
    p.add_argument("--slices", type=int, default=None, help="slices per op per step")
    p.add_argument("--workload", choices=["extract_insert_256", "insert_512", "insert_extract_256", "batched",
                                          "extract_wwindow_256"],
                   default="extract_insert_256",
                   help="insert_512: the 512^3 x 20,000 windowed-sinc insertion, gather vs scatter form; "
                        "insert_extract_256: insert_and_extract_central_slices_3d, 4096 in, 256 out; "
                        "batched: 12,000 LANCZOS8 extractions over 12 volumes in one persistent launch; "
                        "extract_wwindow_256: 4096 extractions with a 7-sample w-windowed sinc")
    p.add_argument("--out-slices", type=int, default=256, help="insert_extract_256: output slices")
    p.add_argument("--ref-slices", type=int, default=None,
                   help="slices of the CPU reference sample (insert_512: 64 input, insert_extract_256: 2 output)")
    args = p.parse_args()
    global N, SLICES
    if args.workload == "extract_wwindow_256":
        args.n = args.n or 256
        args.slices = args.slices or 4096
        args.steps = min(args.steps, 20)
        run_extract_wwindow(args)
        return
    if args.workload == "batched":
        args.slices = args.slices or 12000
        args.steps = min(args.steps, 5)
        run_batched(args)
        return
    if args.workload == "insert_extract_256":
        args.n = args.n or 256
        args.slices = args.slices or 4096
        args.ref_slices = args.ref_slices or 2
        args.steps = min(args.steps, 20)
        run_insert_extract(args)
        return
    args.ref_slices = args.ref_slices or 64
    if args.workload == "insert_512":
        args.n = args.n or 512
        args.slices = args.slices or 20000
        args.steps = min(args.steps, 3)
        run_large(args)
        return
    N, SLICES = args.n or 256, args.slices or 4096
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
