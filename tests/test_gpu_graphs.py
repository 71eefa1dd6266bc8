"""The entry points inside a caller's CUDA graph.

A serving or reconstruction loop captures its calls once (torch.cuda.graph, or cudaStreamBeginCapture on
its own stream) and replays them. Every call must therefore be capturable: its stream-ordered scratch
(the pair copy, the padded accumulator, batch descriptors) becomes the graph's own allocation, and
nothing in it may synchronise. Each test captures calls after eager warm-up calls, replays the graph
twice over refilled outputs, and compares with the eager results (bit for bit where the path is
deterministic, to 1e-6 where float atomics sum in a different order).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(((a - b).abs().pow(2).sum() / b.abs().pow(2).sum().clamp_min(1e-30)).sqrt())


def _inputs(n, count, seed):
    import torch
    from noa_b200 import synthetic
    vol = torch.from_numpy(synthetic.make_volume(n, seed=seed)).cuda()
    rot = torch.from_numpy(synthetic.quaternion_to_matrix(synthetic.random_quaternions(count, seed=seed + 1))
                           .astype(np.float32)).cuda()
    return vol, rot


def _capture(fn):
    import torch
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        fn()
    torch.cuda.synchronize()
    return g


def test_extract_and_rasterize_replay_equals_eager():
    import torch
    from noa_b200 import fourier_project as fp
    n, count = 64, 200  # enough pixels for the pair copy (200 x 64 x 33 > 2 x 64 x 64 x 33)
    vol, rot = _inputs(n, count, seed=1)
    vshape, sshape = (1, n, n, n), (count, 1, n, n)
    out = torch.empty((count, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grid = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grid_w = torch.zeros(grid.shape, dtype=torch.float32, device="cuda")

    def step():
        fp.extract_central_slices_3d("hc2h", vol, None, vshape, out, None, sshape, None, rot)
        fp.rasterize_central_slices_3d("h2hc", out, None, sshape, grid, grid_w, vshape, None, rot)

    step()
    torch.cuda.synchronize()
    ref_out, ref_grid, ref_w = out.clone(), grid.clone(), grid_w.clone()
    g = _capture(step)
    for _ in range(2):
        out.fill_(7)
        grid.zero_()
        grid_w.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(out, ref_out)
        assert _rel(grid, ref_grid) <= 1e-6 and _rel(grid_w, ref_w) <= 1e-6


def test_insertions_replay_equals_eager():
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    n, count = 48, 24
    _, rot = _inputs(n, count, seed=3)
    inv = rot.transpose(1, 2).contiguous()
    slices = torch.from_numpy(synthetic.make_slices(count, n, seed=4)).cuda()
    vshape, sshape = (1, n, n, n), (count, 1, n, n)
    ws = fp.WindowedSinc(-1.0, 3.0 / n)
    grid = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grid_w = torch.zeros(grid.shape, dtype=torch.float32, device="cuda")
    grid_s = torch.zeros_like(grid)
    grid_sw = torch.zeros_like(grid_w)
    out = torch.empty((5, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    _, rot_out = _inputs(n, 5, seed=5)

    def step():
        fp.insert_central_slices_3d("h2hc", slices, None, sshape, grid, grid_w, vshape, None, inv, windowed_sinc=ws)
        fp.insert_central_slices_3d_scatter("h2hc", slices, None, sshape, grid_s, grid_sw, vshape, None, inv,
                                            windowed_sinc=ws)
        fp.insert_and_extract_central_slices_3d("h2h", slices, None, sshape, out, None, (5, 1, n, n), None, inv,
                                                None, rot_out, input_windowed_sinc=ws)

    step()
    torch.cuda.synchronize()
    refs = [t.clone() for t in (grid, grid_w, grid_s, grid_sw, out)]
    g = _capture(step)
    for _ in range(2):
        for t in (grid, grid_w, grid_s, grid_sw):
            t.zero_()
        out.fill_(7)
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(grid, refs[0]) and torch.equal(grid_w, refs[1])  # gather: deterministic
        assert _rel(grid_s, refs[2]) <= 1e-6 and _rel(grid_sw, refs[3]) <= 1e-6
        assert torch.equal(out, refs[4])


def test_one_shot_batch_launches_replay_equals_eager():
    """The serving loop's one-shot launches stage their request descriptors from host memory that is
    gone when the call returns; under capture they go in as kernel parameters, so every replay reads
    the descriptors of the capture (a plain memcpy node would read the freed host buffer)."""
    import torch
    from noa_b200 import synthetic
    from noa_b200.batch import (ExtractRequest, RasterizeRequest, extract_batch_launch, rasterize_batch_launch,
                                volume_pairs)
    n = 64
    vol, rot = _inputs(n, 1000, seed=7)
    # 1000 slices of 64 x 33 pixels: above 2^21 pixels, a grid of its own unless persistent_only; 9 slices:
    # the persistent kernel either way
    outs = [torch.empty((c, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda") for c in (1000, 9)]
    ereqs = [ExtractRequest(volume=vol, volume_shape=(1, n, n, n), slice=o, slice_shape=(o.shape[0], 1, n, n),
                            fwd_rotation=rot[:o.shape[0]].contiguous()) for o in outs]
    pairs = [volume_pairs(vol, (1, n, n, n))] * 2
    rreqs = []
    for i, count in enumerate((20, 7, 33)):
        rreqs.append(RasterizeRequest(
            slice=torch.from_numpy(synthetic.make_slices(count, n, seed=20 + i)).cuda(), slice_shape=(count, 1, n, n),
            volume=torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda"), volume_shape=(1, n, n, n),
            volume_weight=torch.zeros((1, n, n, n // 2 + 1), dtype=torch.float32, device="cuda"),
            fwd_rotation=rot[i * 40:i * 40 + count].contiguous()))

    for persistent_only in (False, True):
        def step():
            extract_batch_launch("hc2h", ereqs, pairs, persistent_only=persistent_only)
            rasterize_batch_launch("h2hc", rreqs)

        for r in rreqs:
            r.volume.zero_()
            r.volume_weight.zero_()
        step()
        torch.cuda.synchronize()
        refs = [o.clone() for o in outs] + [t.clone() for r in rreqs for t in (r.volume, r.volume_weight)]
        g = _capture(step)
        for _ in range(2):
            for o in outs:
                o.fill_(7)
            for r in rreqs:
                r.volume.zero_()
                r.volume_weight.zero_()
            g.replay()
            torch.cuda.synchronize()
            for o, ref in zip(outs, refs):
                assert torch.equal(o, ref)
            got = [t for r in rreqs for t in (r.volume, r.volume_weight)]
            for t, ref in zip(got, refs[len(outs):]):
                assert _rel(t, ref) <= 1e-6


def test_batch_runs_capture_and_creation_refuses_inside_a_capture():
    """A batch's runs may be captured (inside a capture a run issues the batch's launch sequence into it);
    its creation, which uploads, may autotune and synchronizes, is refused inside a capture without
    breaking it."""
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200.batch import ExtractBatch, ExtractRequest
    n, count = 64, 300
    vol, rot = _inputs(n, count, seed=11)
    out = torch.empty((count, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    req = [ExtractRequest(volume=vol, volume_shape=(1, n, n, n), slice=out, slice_shape=(count, 1, n, n),
                          fwd_rotation=rot)]
    batch = ExtractBatch("hc2h", req, interp="linear", autotune=False)
    batch.run()
    torch.cuda.synchronize()
    ref = out.clone()
    g = _capture(batch.run)
    for _ in range(2):
        out.fill_(7)
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g2 = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g2, stream=side, capture_error_mode="thread_local"):
        with pytest.raises(fp.NoaB200Error):
            ExtractBatch("hc2h", req, interp="linear", autotune=False)
    torch.cuda.synchronize()
    batch.close()
