"""The serving loop on the GPU: every request's result is the same alone and in the mix.

Extractions served in shared persistent launches (through the volumes' pair copies) must be
bit-identical to nb_extract_central_slices_3d on the request alone; insertions, rasterized
concurrently with other work, must match a lone rasterization within the atomic-insertion tolerance
(relative L2 <= 1e-4: only the order of the float reductions differs).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from noa_b200 import fourier_project as fp  # noqa: E402
from noa_b200 import synthetic  # noqa: E402
from noa_b200.serve import CudaExecutor, ProjectionServer, Request, latency_summary, run_stream  # noqa: E402

INSERT_TOL = 1e-4


def _rel_l2(a, b):
    a = a.to(torch.complex128) if a.is_complex() else a.to(torch.float64)
    b = b.to(a.dtype)
    den = torch.linalg.vector_norm(b).item()
    return torch.linalg.vector_norm(a - b).item() / (den if den else 1.0)


@pytest.mark.gpu
def test_served_results_match_alone():
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    boxes = [32, 48, 64]
    ex = CudaExecutor(dev, insert_streams=2)
    server = ProjectionServer(ex, int(2e9), max_batch_slices=300, max_inflight_batches=2, keep_outputs=True)
    vols = {}
    for vid, n in enumerate(boxes):
        vols[vid] = torch.from_numpy(synthetic.make_volume(n, seed=10 + vid)).to(dev)
        server.add_volume(vid, vols[vid], (1, n, n, n))
    reqs = []
    for i in range(30):
        vid = int(rng.integers(len(boxes)))
        n = boxes[vid]
        k = int(rng.integers(5, 120))
        rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(k, seed=100 + i)))
        if i % 2:
            rot = rot.pin_memory()
        else:
            rot = rot.to(dev)
        kind = "insert" if rng.random() < 0.35 else "extract"
        slices = None
        if kind == "insert":
            slices = torch.from_numpy(synthetic.make_slices(k, n, seed=200 + i)).to(dev)
        reqs.append(Request(kind, vid, rot, slices, arrival=(i // 6) * 2e-3))  # bursts of 6
    torch.cuda.synchronize()
    run_stream(server, reqs)
    ex.synchronize()
    assert all(r.error is None for r in reqs)
    n_extract = sum(r.kind == "extract" for r in reqs)
    assert server.stats.batches < n_extract  # some launches carried several requests
    for r in reqs:
        n = boxes[r.volume_id]
        k = r.n_slices
        rot = r.rotations.to(dev)
        if r.kind == "extract":
            alone = torch.empty((k, 1, n, n // 2 + 1), dtype=torch.complex64, device=dev)
            fp.extract_central_slices_3d("hc2h", vols[r.volume_id], None, (1, n, n, n), alone, None,
                                         (k, 1, n, n), None, rot)
            torch.cuda.synchronize()
            assert torch.equal(alone, r.output), f"request {r.rid}"
        else:
            v = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device=dev)
            w = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.float32, device=dev)
            fp.rasterize_central_slices_3d("h2hc", r.slices, None, (k, 1, n, n), v, w, (1, n, n, n), None, rot)
            torch.cuda.synchronize()
            assert _rel_l2(r.output[0], v) <= INSERT_TOL, f"request {r.rid}"
            assert _rel_l2(r.output[1], w) <= INSERT_TOL, f"request {r.rid}"
    lat = latency_summary(reqs)
    assert lat["n"] == len(reqs) and lat["p99_ms"] >= lat["p50_ms"] > 0


@pytest.mark.gpu
def test_batch_launch_with_pairs_matches_per_call():
    from noa_b200 import batch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    calls, pairs, outs = [], [], []
    for i, n in enumerate((40, 64, 33)):
        vol = torch.from_numpy(synthetic.make_volume(n, seed=i)).to(dev)
        k = 7 + 5 * i
        rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(k, seed=50 + i)).to(dev))
        out = torch.empty((k, 1, n, n // 2 + 1), dtype=torch.complex64, device=dev)
        calls.append(batch.ExtractRequest(volume=vol, volume_shape=(1, n, n, n), slice=out,
                                          slice_shape=(k, 1, n, n), fwd_rotation=rot))
        pairs.append(batch.volume_pairs(vol, (1, n, n, n)) if i != 1 else None)
        outs.append(out)
    batch.extract_batch_launch("hc2h", calls, pairs)
    torch.cuda.synchronize()
    for c, out in zip(calls, outs):
        alone = torch.empty_like(out)
        fp.extract_central_slices_3d("hc2h", c.volume, None, c.volume_shape, alone, None, c.slice_shape, None,
                                     c.fwd_rotation)
        torch.cuda.synchronize()
        assert torch.equal(alone, out)
