"""Serving loop for central-slice extraction and insertion: admission by HBM budget and continuous batching.

Requests name one of the server's resident volumes and carry their orientations (and, for insertion,
their slices). ``ProjectionServer.poll()`` runs one scheduling round:

1. completions — launches whose CUDA event has fired complete their requests, whose memory returns to
   the budget;
2. admission — waiting requests are admitted in arrival order while their device footprint (outputs,
   accumulators, staged orientations, the insertion's transient accumulator) fits in what the budget
   leaves after the resident volumes; a request larger than the whole budget is rejected;
3. launches — admitted extractions are packed, up to ``max_batch_slices`` slices, into ONE batched
   launch (``nb_extract_batch_launch``: each volume read through its resident pair copy, requests of
   2^21 output pixels or more as grids of their own, the rest through one device work queue) on the
   extraction stream, with at most ``max_inflight_batches`` batches
   queued there; the insertions admitted in the round are packed the same way into ONE batched
   rasterization (``nb_rasterize_batch_launch``: one scatter and one finalize launch, each request into
   its own zeroed value + weight grids) on one of the insertion streams, round robin.

Backpressure and cancellation: with ``max_waiting`` set, ``submit()`` refuses a request while that many
wait for admission (it raises ``ServerBusy``; the client keeps the request and offers it again, as
``run_stream`` does), so the queue and the host memory it pins stay bounded under overload.
``cancel()`` withdraws a request that has not been launched yet (waiting, or admitted but not yet
packed into a launch, whose memory returns to the budget); work already on the device cannot be
recalled, so such a request completes normally.

Continuous batching: extractions that arrive while a batch runs are admitted as memory frees up and
form the next batch, which is already queued behind the running one, so the device never waits for
the host; insertion batches run concurrently on their own streams. The scheduling logic is independent of
CUDA (``Executor``), so it is tested on the CPU with a simulated executor.

No function of the reference corresponds to this module; it drives extract_central_slices_3d
(FourierProject.hpp:1869-1914) and rasterize_central_slices_3d (:1653-1692) through this library's
batched entry points.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Any

import numpy as np


@dataclass
class Volume:
    """A resident volume: (1, N, N, N/2+1) complex64 rfft on the device, plus its pair copy."""
    vid: int
    data: Any
    shape: tuple            # logical (1, N, N, N)
    pairs: Any = None

    @property
    def box(self) -> int:
        return int(self.shape[1])

    @property
    def nbytes(self) -> int:
        n = self.box
        b = n * n * (n // 2 + 1) * 8
        return b + (0 if self.pairs is None else n * n * (n // 2 + 1) * 16)


@dataclass
class Request:
    """One projection (``kind="extract"``) or backprojection (``kind="insert"``) request.

    ``rotations``: (n, 12) float32 — noa's Mat33<f32> layout (``fourier_project.pack_rotations``) —
    on the host (pinned memory makes its upload asynchronous) or on the device; forward rotations for
    both kinds. ``slices``: insertion input, (n, 1, N, N/2+1) complex64 on the device."""
    kind: str
    volume_id: int
    rotations: Any
    slices: Any = None
    arrival: float = 0.0
    rid: int = -1
    # Filled by the server.
    output: Any = None       # extract: slices (n, 1, N, N/2+1); insert: (values, weights)
    error: str | None = None
    admitted: float = math.nan
    launched: float = math.nan
    done: float = math.nan
    batch: int = -1
    keep: list = field(default_factory=list)

    @property
    def n_slices(self) -> int:
        return int(self.rotations.shape[0])

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def footprint(req: Request, box: int) -> int:
    """Device bytes a request holds while admitted."""
    wp = box // 2 + 1
    rot = req.n_slices * 48
    if req.kind == "extract":
        return req.n_slices * box * wp * 8 + rot
    # value + weight accumulators, and the rasterizer's padded float4 accumulator while it runs
    pad = (box + 5) * (box + 5) * (wp + 4) * 16
    return box * box * wp * 12 + pad + rot


class Executor:
    """What the server needs from the device. ``launch_*`` return a token; ``done(token)`` polls it."""

    def prepare_volume(self, vol: Volume) -> None:
        raise NotImplementedError

    def launch_extracts(self, reqs: list[Request], vols: list[Volume]) -> Any:
        raise NotImplementedError

    def launch_inserts(self, reqs: list[Request], vols: list[Volume]) -> Any:
        raise NotImplementedError

    def done(self, token) -> bool:
        raise NotImplementedError


class CudaExecutor(Executor):
    """Launches on one CUDA device through noa_b200: one extraction stream, ``insert_streams`` streams
    for insertions. Extractions are ``remap_extract`` (default hc2h), insertions rasterize with
    ``remap_insert`` (default h2hc), both LINEAR with ``fftfreq_cutoff``."""

    def __init__(self, device=None, insert_streams=2, remap_extract="hc2h", remap_insert="h2hc",
                 fftfreq_cutoff=0.5, timing=False):
        import torch
        from . import batch, fourier_project
        self.torch, self.batch, self.fp = torch, batch, fourier_project
        self.device = torch.device(device if device is not None else "cuda")
        self.extract_stream = torch.cuda.Stream(self.device)
        self.insert_streams = [torch.cuda.Stream(self.device) for _ in range(insert_streams)]
        self._next = 0
        self.remap_extract, self.remap_insert = remap_extract, remap_insert
        self.cutoff = fftfreq_cutoff
        # timing=True: every launch is bracketed by timed events, for busy_time(); host seconds spent
        # issuing launches are counted either way.
        self.timing = timing
        self.spans: list = []
        self.host_seconds = 0.0

    def _span_start(self, stream):
        if not self.timing:
            return None
        ev = self.torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        return ev

    def _span_end(self, start, stream, kind, slices):
        ev = self.torch.cuda.Event(enable_timing=self.timing)
        ev.record(stream)
        if start is not None:
            self.spans.append((start, ev, kind, slices))
        return ev

    def busy_time(self) -> dict:
        """Device time of the timed launches (after synchronize()): per kind, the sum of launch
        durations, and the union of all launch intervals (device busy time with overlap counted once)."""
        if not self.spans:
            return {}
        ref = self.spans[0][0]
        iv = sorted((ref.elapsed_time(a), ref.elapsed_time(b), k, n) for a, b, k, n in self.spans)
        out = {"extract_ms": 0.0, "insert_ms": 0.0, "extract_slices": 0, "insert_slices": 0}
        union, cur0, cur1 = 0.0, None, None
        for t0, t1, k, n in iv:
            out[f"{k}_ms"] += t1 - t0
            out[f"{k}_slices"] += n
            if cur1 is None or t0 > cur1:
                if cur1 is not None:
                    union += cur1 - cur0
                cur0, cur1 = t0, t1
            else:
                cur1 = max(cur1, t1)
        union += cur1 - cur0
        out["busy_union_ms"] = union
        out["span_ms"] = iv[-1][1] - iv[0][0]
        return out

    def _rotations(self, req: Request):
        r = req.rotations
        if r.device != self.device:
            r = r.to(self.device, non_blocking=True)
        req.keep.append(r)
        return r

    def prepare_volume(self, vol: Volume) -> None:
        with self.torch.cuda.stream(self.extract_stream):
            vol.pairs = self.batch.volume_pairs(vol.data, vol.shape, stream=self.extract_stream)
        self.extract_stream.synchronize()

    def launch_extracts(self, reqs, vols):
        torch = self.torch
        s = self.extract_stream
        h0 = time.perf_counter()
        calls, pairs = [], []
        start = self._span_start(s)
        with torch.cuda.stream(s):
            for r, v in zip(reqs, vols):
                n, box = r.n_slices, v.box
                r.output = torch.empty((n, 1, box, box // 2 + 1), dtype=torch.complex64, device=self.device)
                calls.append(self.batch.ExtractRequest(volume=v.data, volume_shape=v.shape, slice=r.output,
                                                       slice_shape=(n, 1, box, box),
                                                       fwd_rotation=self._rotations(r)))
                pairs.append(v.pairs)
            self.batch.extract_batch_launch(self.remap_extract, calls, pairs, fftfreq_cutoff=self.cutoff,
                                            stream=s)
        ev = self._span_end(start, s, "extract", sum(r.n_slices for r in reqs))
        self.host_seconds += time.perf_counter() - h0
        return ev

    def launch_inserts(self, reqs, vols):
        torch = self.torch
        s = self.insert_streams[self._next % len(self.insert_streams)]
        self._next += 1
        h0 = time.perf_counter()
        start = self._span_start(s)
        calls = []
        with torch.cuda.stream(s):
            for req, vol in zip(reqs, vols):
                box = vol.box
                values = torch.zeros((1, box, box, box // 2 + 1), dtype=torch.complex64, device=self.device)
                weights = torch.zeros((1, box, box, box // 2 + 1), dtype=torch.float32, device=self.device)
                req.output = (values, weights)
                n = req.n_slices
                calls.append(self.batch.RasterizeRequest(
                    slice=req.slices, slice_shape=(n, 1, box, box), volume=values, volume_shape=(1, box, box, box),
                    volume_weight=weights, fwd_rotation=self._rotations(req)))
            self.batch.rasterize_batch_launch(self.remap_insert, calls, fftfreq_cutoff=self.cutoff, stream=s)
        ev = self._span_end(start, s, "insert", sum(r.n_slices for r in reqs))
        self.host_seconds += time.perf_counter() - h0
        return ev

    def done(self, token) -> bool:
        return token.query()

    def synchronize(self) -> None:
        self.extract_stream.synchronize()
        for s in self.insert_streams:
            s.synchronize()


class ServerBusy(RuntimeError):
    """``submit()`` refused a request because ``max_waiting`` requests already wait for admission."""


@dataclass
class ServerStats:
    submitted: int = 0
    completed: int = 0
    rejected: int = 0
    refused: int = 0         # submit() calls turned away by backpressure (the client may retry)
    cancelled: int = 0
    batches: int = 0
    batch_requests: int = 0
    batch_slices: int = 0
    inserts: int = 0
    insert_batches: int = 0
    max_waiting: int = 0
    peak_bytes: int = 0
    poll_seconds: float = 0.0


class ProjectionServer:
    """Admission by device-memory budget and continuous batching (see the module docstring).

    ``budget_bytes`` caps resident volumes plus admitted requests. ``keep_outputs=False`` drops each
    request's outputs when it completes (a benchmark's client), else they stay on the request.
    ``max_waiting`` (None: unbounded) is the length of the admission queue beyond which ``submit()``
    raises ``ServerBusy``."""

    def __init__(self, executor: Executor, budget_bytes: int, *, max_batch_slices=65536,
                 max_inflight_batches=2, keep_outputs=True, max_waiting: int | None = None,
                 clock=time.perf_counter):
        self.ex = executor
        self.budget = int(budget_bytes)
        self.max_waiting = None if max_waiting is None else int(max_waiting)
        self.max_batch_slices = int(max_batch_slices)
        self.max_inflight_batches = int(max_inflight_batches)
        self.keep_outputs = keep_outputs
        self.clock = clock
        self.volumes: dict[int, Volume] = {}
        self.resident = 0
        self.used = 0
        self.waiting: deque[Request] = deque()
        self.ready_extract: deque[Request] = deque()
        self.ready_insert: deque[Request] = deque()
        self.inflight: list[tuple[Any, list[Request], bool]] = []  # (token, requests, is_batch)
        self.stats = ServerStats()
        self._rid = 0

    # -- resident volumes --------------------------------------------------------------------------
    def add_volume(self, vid: int, data, shape) -> Volume:
        vol = Volume(vid, data, tuple(int(x) for x in shape))
        self.ex.prepare_volume(vol)
        if self.resident + vol.nbytes > self.budget:
            raise MemoryError(f"volume {vid} ({vol.nbytes} B) does not fit in the budget")
        self.volumes[vid] = vol
        self.resident += vol.nbytes
        return vol

    def add_volume_file(self, vid: int, path: str, logical_width: int | None = None) -> Volume:
        """Makes an rfft volume stored in an MRC file (mode 4, complex64, physical shape
        (1, D, H, W/2+1)) resident on the executor's device. The logical width defaults to the even
        W = 2 (W/2+1 - 1)."""
        import torch
        from . import mrc
        data, h = mrc.read(path)
        if data.dtype != np.complex64 or data.shape[0] != 1:
            raise ValueError(f"{path}: expected one complex64 rfft volume, got {data.dtype} {data.shape}")
        _, d, hh, wp = data.shape
        w = logical_width if logical_width is not None else 2 * (wp - 1)
        if w // 2 + 1 != wp:
            raise ValueError(f"{path}: width {wp} is not the rfft width of {w}")
        device = getattr(self.ex, "device", "cuda")
        return self.add_volume(vid, torch.from_numpy(np.ascontiguousarray(data)).to(device), (1, d, hh, w))

    # -- requests ------------------------------------------------------------------------------------
    def submit(self, req: Request) -> Request:
        if req.kind not in ("extract", "insert"):
            raise ValueError(f"unknown request kind {req.kind!r}")
        if req.volume_id not in self.volumes:
            raise KeyError(f"volume {req.volume_id} is not resident")
        if self.max_waiting is not None and len(self.waiting) >= self.max_waiting:
            self.stats.refused += 1
            raise ServerBusy(f"{len(self.waiting)} requests wait for admission (max_waiting={self.max_waiting})")
        if req.rid < 0:
            req.rid = self._rid
        self._rid += 1
        self.waiting.append(req)
        self.stats.submitted += 1
        self.stats.max_waiting = max(self.stats.max_waiting, len(self.waiting))
        return req

    def cancel(self, req: Request) -> bool:
        """Withdraws ``req`` if it has not been launched: it leaves the admission queue, or, for an
        admitted extraction not yet in a batch, the launch queue (its memory returns to the budget).
        Returns True then, with ``req.error == "cancelled"``. Returns False for a request already on the
        device (it completes normally: its work cannot be recalled from the GPU), finished, or unknown."""
        for queue, admitted in ((self.waiting, False), (self.ready_extract, True), (self.ready_insert, True)):
            for i, r in enumerate(queue):
                if r is req:
                    del queue[i]
                    if admitted:
                        self.used -= footprint(r, self.volumes[r.volume_id].box)
                    r.error = "cancelled"
                    r.done = self.clock()
                    r.keep.clear()
                    self.stats.cancelled += 1
                    return True
        return False

    def busy(self) -> bool:
        return bool(self.waiting or self.ready_extract or self.ready_insert or self.inflight)

    def poll(self) -> list[Request]:
        """One scheduling round; returns the requests completed (or rejected) in it."""
        h0 = time.perf_counter()
        finished = self._complete()
        finished += self._admit()
        self._launch()
        self.stats.poll_seconds += time.perf_counter() - h0
        return finished

    def drain(self, sleep=0.0) -> list[Request]:
        out = []
        while self.busy():
            out += self.poll()
            if sleep:
                time.sleep(sleep)
        return out

    # -- internals -----------------------------------------------------------------------------------
    def _complete(self) -> list[Request]:
        finished, still = [], []
        for token, reqs, is_batch in self.inflight:
            if self.ex.done(token):
                now = self.clock()
                for r in reqs:
                    r.done = now
                    self.used -= footprint(r, self.volumes[r.volume_id].box)
                    r.keep.clear()
                    if not self.keep_outputs:
                        r.output = None
                    finished.append(r)
                self.stats.completed += len(reqs)
            else:
                still.append((token, reqs, is_batch))
        self.inflight = still
        return finished

    def _admit(self) -> list[Request]:
        rejected = []
        while self.waiting:
            r = self.waiting[0]
            need = footprint(r, self.volumes[r.volume_id].box)
            if self.resident + need > self.budget:
                self.waiting.popleft()
                r.error = f"needs {need} B, more than the budget leaves ({self.budget - self.resident} B)"
                r.done = self.clock()
                self.stats.rejected += 1
                rejected.append(r)
                continue
            if self.resident + self.used + need > self.budget:
                break  # in arrival order: wait for memory to free up
            self.waiting.popleft()
            self.used += need
            self.stats.peak_bytes = max(self.stats.peak_bytes, self.resident + self.used)
            r.admitted = self.clock()
            (self.ready_extract if r.kind == "extract" else self.ready_insert).append(r)
        return rejected

    def _launch(self) -> None:
        # Insertions admitted in this round: one batched rasterization, on the next insertion stream.
        while self.ready_insert:
            batch, slices = [], 0
            while self.ready_insert and (not batch or slices + self.ready_insert[0].n_slices <= self.max_batch_slices):
                r = self.ready_insert.popleft()
                batch.append(r)
                slices += r.n_slices
            now = self.clock()
            for r in batch:
                r.launched = now
            token = self.ex.launch_inserts(batch, [self.volumes[r.volume_id] for r in batch])
            self.inflight.append((token, batch, False))
            self.stats.inserts += len(batch)
            self.stats.insert_batches += 1
        while self.ready_extract:
            n_batches = sum(1 for _, _, b in self.inflight if b)
            if n_batches >= self.max_inflight_batches:
                return
            batch, slices = [], 0
            while self.ready_extract and (not batch or slices + self.ready_extract[0].n_slices <= self.max_batch_slices):
                r = self.ready_extract.popleft()
                batch.append(r)
                slices += r.n_slices
            now = self.clock()
            for r in batch:
                r.launched = now
                r.batch = self.stats.batches
            token = self.ex.launch_extracts(batch, [self.volumes[r.volume_id] for r in batch])
            self.inflight.append((token, batch, True))
            self.stats.batches += 1
            self.stats.batch_requests += len(batch)
            self.stats.batch_slices += slices


def latency_summary(reqs: list[Request]) -> dict:
    """p50 / p99 / mean / max latency in milliseconds (completed requests only)."""
    lat = np.array([r.latency for r in reqs if r.error is None and not math.isnan(r.done)]) * 1e3
    if lat.size == 0:
        return {"n": 0}
    return {"n": int(lat.size), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}


def run_stream(server: ProjectionServer, requests: list[Request], *, clock=time.perf_counter,
               idle_sleep=5e-5) -> tuple[float, float]:
    """Feeds ``requests`` (sorted by ``arrival``, seconds from the start) to the server in real time and
    polls it until every request is finished. Arrival times are rebased onto ``clock``. A request the
    server refuses (``ServerBusy``) is offered again after the next poll, its latency still counted from
    its arrival. Returns the (start, end) clock values."""
    t0 = clock()
    for r in requests:
        r.arrival = t0 + r.arrival
    i = 0
    while i < len(requests) or server.busy():
        now = clock()
        while i < len(requests) and requests[i].arrival <= now:
            try:
                server.submit(requests[i])
            except ServerBusy:
                break  # backpressure: offer it again after the next scheduling round
            i += 1
        server.poll()
        if not server.busy() and i < len(requests):
            wait = requests[i].arrival - clock()
            if wait > 0:
                time.sleep(min(wait, 1e-3))
        elif idle_sleep:
            time.sleep(idle_sleep)
    return t0, clock()
