"""The entry points called from several host threads at once, each on its own CUDA stream.

A serving process runs request handlers on several threads; the library's shared state (the memory
pool and its cap, the cached SM count, the autotune cache) is guarded, and errors are reported per
thread. Four threads each extract and rasterize their own data concurrently, and each thread's results
equal the same calls made one after another on the main thread (extraction bit for bit, rasterization
to 1e-6, its atomics summing in an unspecified order); a thread whose call fails reads its own error
message, not another thread's.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _job(seed, n=64, count=160):
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    vol = torch.from_numpy(synthetic.make_volume(n, seed=seed)).cuda()
    rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(count, seed=seed + 1)).cuda())
    out = torch.empty((count, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grid = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grid_w = torch.zeros(grid.shape, dtype=torch.float32, device="cuda")

    def run(stream=None):
        fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), out, None, (count, 1, n, n), None, rot,
                                     stream=stream)
        fp.rasterize_central_slices_3d("h2hc", out, None, (count, 1, n, n), grid, grid_w, (1, n, n, n), None, rot,
                                       stream=stream)

    return run, out, grid, grid_w


def _rel(a, b):
    return float(((a - b).abs().pow(2).sum() / b.abs().pow(2).sum()).sqrt())


def test_concurrent_threads_match_sequential_calls():
    import torch
    jobs = [_job(100 + 10 * k) for k in range(4)]
    refs = []
    for run, out, grid, grid_w in jobs:
        run()
        torch.cuda.synchronize()
        refs.append((out.clone(), grid.clone(), grid_w.clone()))
        out.fill_(7)
        grid.zero_()
        grid_w.zero_()
    torch.cuda.synchronize()

    errors = []
    barrier = threading.Barrier(len(jobs))

    def worker(k):
        try:
            run = jobs[k][0]
            stream = torch.cuda.Stream()
            with torch.cuda.stream(stream):
                barrier.wait()
                for _ in range(3):  # the grids accumulate three rasterizations
                    run(stream)
            stream.synchronize()
        except Exception as e:  # reported on the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(jobs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    torch.cuda.synchronize()
    assert not errors, errors
    for (_, out, grid, grid_w), (r_out, r_grid, r_w) in zip(jobs, refs):
        assert torch.equal(out, r_out)
        assert _rel(grid, 3 * r_grid) <= 1e-6 and _rel(grid_w, 3 * r_w) <= 1e-6


def test_errors_are_reported_per_thread():
    import torch
    from noa_b200 import fourier_project as fp
    n = 32
    vol = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    out = torch.empty((4, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    rot = fp.pack_rotations(torch.eye(3).repeat(4, 1, 1).cuda())
    messages = {}

    def bad():
        try:  # the slice shape disagrees with the output's physical shape
            fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), out, None, (4, 1, n, n + 2), None, rot)
        except fp.NoaB200Error as e:
            messages["bad"] = str(e)

    def good():
        fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), out, None, (4, 1, n, n), None, rot)
        messages["good"] = fp.lib().nb_last_error().decode()

    threads = [threading.Thread(target=bad), threading.Thread(target=good)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    torch.cuda.synchronize()
    assert messages.get("bad"), messages
    assert messages["good"] != messages["bad"]  # the other thread's message does not leak into this one
