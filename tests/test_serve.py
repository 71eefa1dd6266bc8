"""Scheduling logic of the serving loop (noa_b200.serve), on the CPU with a simulated executor.

The executor completes a launch after a simulated duration proportional to its slices; a manual clock
drives both, so admission by budget, arrival order, continuous batching and completion accounting are
checked deterministically.
"""
import numpy as np
import pytest

from noa_b200.serve import (Executor, ProjectionServer, Request, ServerBusy, footprint, latency_summary,
                            run_stream)


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class FakeExecutor(Executor):
    """Launches finish `per_slice` seconds per slice after the previous launch on the same queue."""

    def __init__(self, clock, per_slice=1e-3, insert_queues=2):
        self.clock = clock
        self.per_slice = per_slice
        self.queue_end = {"extract": 0.0}
        for i in range(insert_queues):
            self.queue_end[f"insert{i}"] = 0.0
        self.n_insert_queues = insert_queues
        self.launches = []
        self._next = 0

    def prepare_volume(self, vol):
        vol.pairs = None

    def _enqueue(self, queue, slices):
        start = max(self.clock(), self.queue_end[queue])
        end = start + slices * self.per_slice
        self.queue_end[queue] = end
        return end

    def launch_extracts(self, reqs, vols):
        self.launches.append(("extract", [r.rid for r in reqs]))
        for r in reqs:
            r.output = ("slices", r.rid)
        return self._enqueue("extract", sum(r.n_slices for r in reqs))

    def launch_inserts(self, reqs, vols):
        q = f"insert{self._next % self.n_insert_queues}"
        self._next += 1
        self.launches.append((q, [r.rid for r in reqs]))
        for r in reqs:
            r.output = ("grid", r.rid)
        return self._enqueue(q, sum(r.n_slices for r in reqs))

    def done(self, token):
        return self.clock() >= token


def rot(n):
    return np.zeros((n, 12), dtype=np.float32)


def make_server(budget, box=32, n_volumes=2, **kw):
    clock = Clock()
    ex = FakeExecutor(clock)
    s = ProjectionServer(ex, budget, clock=clock, **kw)
    for v in range(n_volumes):
        s.add_volume(v, object(), (1, box, box, box))
    return s, ex, clock


def test_footprint_counts_outputs_and_accumulators():
    r = Request("extract", 0, rot(10))
    assert footprint(r, 64) == 10 * 64 * 33 * 8 + 10 * 48
    r = Request("insert", 0, rot(10))
    assert footprint(r, 64) == 64 * 64 * 33 * 12 + 69 * 69 * 37 * 16 + 10 * 48


def test_extractions_batch_together_and_complete():
    s, ex, clock = make_server(10 ** 9)
    reqs = [s.submit(Request("extract", i % 2, rot(100 + i))) for i in range(5)]
    s.poll()
    assert ex.launches == [("extract", [0, 1, 2, 3, 4])]
    assert all(r.batch == 0 for r in reqs)
    clock.t = 10.0
    done = s.poll()
    assert sorted(r.rid for r in done) == [0, 1, 2, 3, 4]
    assert s.used == 0 and not s.busy()
    assert s.stats.completed == 5


def test_batch_respects_max_slices_and_inflight_cap():
    s, ex, clock = make_server(10 ** 9, max_batch_slices=250, max_inflight_batches=2)
    for i in range(6):
        s.submit(Request("extract", 0, rot(100)))
    s.poll()
    # 2 requests (200 slices) per batch, at most 2 batches queued at once
    assert [l[1] for l in ex.launches] == [[0, 1], [2, 3]]
    clock.t = 0.2 + 1e-9  # first batch (200 slices at 1 ms) done
    s.poll()
    assert [l[1] for l in ex.launches] == [[0, 1], [2, 3], [4, 5]]


def test_continuous_batching_admits_arrivals_while_a_batch_runs():
    s, ex, clock = make_server(10 ** 9, max_inflight_batches=1)
    s.submit(Request("extract", 0, rot(100)))
    s.poll()
    assert len(ex.launches) == 1
    clock.t = 0.05  # batch 0 still running (100 ms)
    s.submit(Request("extract", 1, rot(50)))
    s.submit(Request("extract", 0, rot(50)))
    s.poll()
    assert len(ex.launches) == 1  # admitted, waiting for the batch slot
    assert len(s.ready_extract) == 2
    clock.t = 0.1
    done = s.poll()
    assert [r.rid for r in done] == [0]
    assert ex.launches[1] == ("extract", [1, 2])  # the two arrivals form the next batch


def test_admission_is_bounded_by_the_budget_and_in_arrival_order():
    box = 32
    one = footprint(Request("extract", 0, rot(100)), box)
    s, ex, clock = make_server(2 * one + 1000, box=box, n_volumes=1)
    s.resident = 0  # the fake volumes hold no memory
    reqs = [s.submit(Request("extract", 0, rot(100))) for _ in range(4)]
    s.poll()
    assert [r.rid for r in s.ready_extract] == [] and ex.launches == [("extract", [0, 1])]
    assert s.used == 2 * one
    assert len(s.waiting) == 2
    clock.t = 1.0
    s.poll()
    assert ex.launches[1] == ("extract", [2, 3])
    assert s.stats.peak_bytes <= s.budget
    clock.t = 2.0
    s.poll()
    assert all(not np.isnan(r.done) for r in reqs)


def test_request_larger_than_the_budget_is_rejected_not_blocking():
    box = 32
    s, ex, clock = make_server(footprint(Request("extract", 0, rot(100)), box) + 100, box=box, n_volumes=1)
    s.resident = 0
    big = s.submit(Request("extract", 0, rot(1000)))
    small = s.submit(Request("extract", 0, rot(100)))
    out = s.poll()
    assert big.error is not None and big in out
    assert ex.launches == [("extract", [small.rid])]
    assert s.stats.rejected == 1


def test_insertions_of_a_round_form_one_batch_on_their_own_queue():
    s, ex, clock = make_server(10 ** 9)
    a = s.submit(Request("insert", 0, rot(100)))
    b = s.submit(Request("insert", 1, rot(100)))
    c = s.submit(Request("extract", 0, rot(100)))
    s.poll()
    assert ex.launches == [("insert0", [a.rid, b.rid]), ("extract", [c.rid])]
    d = s.submit(Request("insert", 1, rot(50)))
    s.poll()
    assert ex.launches[-1] == ("insert1", [d.rid])  # the next round's insertions take the next queue
    assert s.stats.inserts == 3 and s.stats.insert_batches == 2
    clock.t = 0.25
    done = s.poll()
    assert {r.rid for r in done} == {a.rid, b.rid, c.rid, d.rid}


def test_outputs_dropped_when_not_kept():
    s, ex, clock = make_server(10 ** 9, keep_outputs=False)
    r = s.submit(Request("extract", 0, rot(10)))
    s.poll()
    clock.t = 1.0
    s.poll()
    assert r.output is None and r.done == 1.0


def test_unknown_volume_and_kind():
    s, ex, clock = make_server(10 ** 9)
    with pytest.raises(KeyError):
        s.submit(Request("extract", 99, rot(1)))
    with pytest.raises(ValueError):
        s.submit(Request("project", 0, rot(1)))


def test_latency_summary_percentiles():
    reqs = []
    for i in range(100):
        r = Request("extract", 0, rot(1), arrival=0.0)
        r.done = (i + 1) * 1e-3
        reqs.append(r)
    s = latency_summary(reqs)
    assert s["n"] == 100
    assert abs(s["p50_ms"] - 50.5) < 1e-6
    assert abs(s["p99_ms"] - 99.01) < 1e-6
    assert s["max_ms"] == pytest.approx(100.0)


def test_run_stream_real_time_with_instant_executor():
    class Instant(FakeExecutor):
        def done(self, token):
            return True

    clock = Clock()
    ex = Instant(clock)
    import time
    s = ProjectionServer(ex, 10 ** 9)
    s.add_volume(0, object(), (1, 16, 16, 16))
    reqs = [Request("extract" if i % 3 else "insert", 0, rot(8), arrival=i * 1e-3) for i in range(20)]
    t0, t1 = run_stream(s, reqs, clock=time.perf_counter)
    assert all(r.error is None and r.done >= r.arrival for r in reqs)
    assert s.stats.completed == 20
    assert t1 >= t0


def test_add_volume_file_reads_an_mrc_rfft_volume(tmp_path):
    import torch
    from noa_b200 import mrc
    vol = (np.arange(8 * 8 * 5, dtype=np.float32).reshape(1, 8, 8, 5) * (1 + 1j)).astype(np.complex64)
    p = str(tmp_path / "v.mrc")
    mrc.write(p, vol)
    clock = Clock()
    ex = FakeExecutor(clock)
    ex.device = "cpu"
    s = ProjectionServer(ex, 10 ** 9, clock=clock)
    v = s.add_volume_file(3, p)
    assert v.shape == (1, 8, 8, 8) and torch.equal(v.data, torch.from_numpy(vol))
    with pytest.raises(ValueError):
        s.add_volume_file(4, p, logical_width=10)


def test_backpressure_refuses_beyond_max_waiting_and_recovers():
    box = 32
    one = footprint(Request("extract", 0, rot(100)), box)
    s, ex, clock = make_server(one + 1000, box=box, n_volumes=1, max_waiting=2)
    s.resident = 0
    a = s.submit(Request("extract", 0, rot(100)))
    s.poll()  # a admitted and launched; the budget holds one request at a time
    b = s.submit(Request("extract", 0, rot(100)))
    c = s.submit(Request("extract", 0, rot(100)))
    with pytest.raises(ServerBusy):
        s.submit(Request("extract", 0, rot(100)))
    assert s.stats.refused == 1 and s.stats.submitted == 3 and len(s.waiting) == 2
    clock.t = 1.0
    s.poll()  # a completes, b is admitted: the queue has room again
    d = s.submit(Request("extract", 0, rot(100)))
    for t in (2.0, 3.0, 4.0, 5.0):
        clock.t = t
        s.poll()
    assert all(r.error is None and not np.isnan(r.done) for r in (a, b, c, d))


def test_run_stream_retries_refused_requests():
    class Instant(FakeExecutor):
        def done(self, token):
            return True

    import time
    clock = Clock()
    s = ProjectionServer(Instant(clock), 10 ** 9, max_waiting=1)
    s.add_volume(0, object(), (1, 16, 16, 16))
    reqs = [Request("extract", 0, rot(4), arrival=0.0) for _ in range(12)]  # all at once
    run_stream(s, reqs, clock=time.perf_counter)
    assert s.stats.completed == 12 and s.stats.refused > 0
    assert all(r.error is None for r in reqs)


def test_cancel_waiting_and_admitted_but_not_running_requests():
    box = 32
    one = footprint(Request("extract", 0, rot(100)), box)
    s, ex, clock = make_server(10 * one, box=box, n_volumes=1, max_inflight_batches=1)
    s.resident = 0
    running = s.submit(Request("extract", 0, rot(100)))
    s.poll()  # launched
    queued = s.submit(Request("extract", 0, rot(100)))
    s.poll()  # admitted, waiting for the batch slot
    assert queued in s.ready_extract and s.used == 2 * one
    assert s.cancel(queued)
    assert queued.error == "cancelled" and s.used == one and queued not in s.ready_extract
    waiting = Request("insert", 0, rot(10))
    s.waiting.append(waiting)  # not yet admitted
    assert s.cancel(waiting) and waiting.error == "cancelled" and not s.waiting
    assert not s.cancel(running)  # on the device: it completes normally
    assert not s.cancel(queued)   # already cancelled
    clock.t = 1.0
    done = s.poll()
    assert done == [running] and running.error is None
    assert s.stats.cancelled == 2 and s.used == 0 and not s.busy()
    assert [l[1] for l in ex.launches] == [[running.rid]]
