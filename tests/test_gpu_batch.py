"""GPU: batched extraction (one persistent kernel in a CUDA graph) gives the per-call results bit for
bit, for uneven volumes and slice counts, with and without autotuning, and on graph replay."""
import numpy as np
import pytest

from cases import rel_l2

pytestmark = pytest.mark.gpu


def _requests(seed=0, out_dt="c32"):
    import torch
    from noa_b200 import synthetic
    from noa_b200.batch import ExtractRequest
    reqs, specs = [], []
    for i, (n, count) in enumerate([(32, 7), (48, 30), (64, 3), (40, 12), (32, 1), (64, 19)]):
        vol = torch.from_numpy(synthetic.make_volume(n, seed=seed + i)).cuda()
        rot = torch.from_numpy(synthetic.random_rotations(count, seed=seed + 50 + i)).cuda()
        dt = torch.complex64 if out_dt == "c32" else torch.float32
        out = torch.full((count, 1, n, n // 2 + 1), 7, dtype=dt, device="cuda")
        reqs.append(ExtractRequest(volume=vol, volume_shape=(1, n, n, n), slice=out, slice_shape=(count, 1, n, n),
                                   fwd_rotation=rot))
        specs.append((vol, rot, n, count, dt))
    return reqs, specs


@pytest.mark.parametrize("interp", ["linear", "lanczos8", "cubic"])
@pytest.mark.parametrize("autotune", [False, True])
def test_batch_matches_per_call(interp, autotune, tmp_path, monkeypatch):
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200.batch import ExtractBatch
    monkeypatch.setenv("NB_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    reqs, specs = _requests()
    batch = ExtractBatch("hc2h", reqs, interp=interp, autotune=autotune)
    for _ in range(2):  # graph replay gives the same result
        for r in reqs:
            r.slice.fill_(3)
        batch.run()
        torch.cuda.synchronize()
        for r, (vol, rot, n, count, dt) in zip(reqs, specs):
            ref = torch.zeros((count, 1, n, n // 2 + 1), dtype=dt, device="cuda")
            fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), ref, None, (count, 1, n, n), None, rot,
                                         interp=interp)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(r.slice.cpu().numpy(), ref.cpu().numpy())
    info = batch.info()
    assert info["n_requests"] == 6 and info["n_items"] > 0
    if autotune:
        assert info["tuned_ms"] > 0 or info["from_cache"]
    batch.close()


def test_batch_against_oracle_and_cache_reuse(tmp_path, monkeypatch):
    import torch
    from oracle.oracle import Call, FpOracle
    from noa_b200.batch import ExtractBatch
    monkeypatch.setenv("NB_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    reqs, specs = _requests(seed=11, out_dt="f32")
    ExtractBatch("hc2h", reqs, interp="lanczos8", autotune=True).run()
    torch.cuda.synchronize()
    second = ExtractBatch("hc2h", reqs, interp="lanczos8", autotune=True)
    assert second.info()["from_cache"]
    for r, (vol, rot, n, count, dt) in zip(reqs, specs):
        call = Call(func="extract", remap="hc2h", inp=vol.cpu().numpy(), in_shape=(1, n, n, n),
                    out=np.zeros((count, 1, n, n // 2 + 1), np.float32), out_shape=(count, 1, n, n),
                    rot=rot.cpu().numpy(), interp=6)
        FpOracle().run(call, 8)
        assert rel_l2(r.slice.cpu().numpy(), call.out) <= 1e-5


def test_batch_rejects_mixed_types():
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200.batch import ExtractBatch
    reqs, _ = _requests()
    n, count = 32, 7
    reqs[0].slice = torch.zeros((count, 1, n, n // 2 + 1), dtype=torch.float32, device="cuda")
    with pytest.raises(fp.NoaB200Error):
        ExtractBatch("hc2h", reqs, interp="linear", autotune=False)


def _large_requests(spec, seed=0):
    import torch
    from noa_b200 import synthetic
    from noa_b200.batch import ExtractRequest
    reqs, vols = [], {}
    for i, (n, count) in enumerate(spec):
        if n not in vols:
            vols[n] = torch.from_numpy(synthetic.make_volume(n, seed=seed + n)).cuda()
        rot = torch.from_numpy(synthetic.random_rotations(count, seed=seed + 70 + i)).cuda()
        out = torch.full((count, 1, n, n // 2 + 1), 7, dtype=torch.complex64, device="cuda")
        reqs.append(ExtractRequest(volume=vols[n], volume_shape=(1, n, n, n), slice=out,
                                   slice_shape=(count, 1, n, n), fwd_rotation=rot))
    return reqs, vols


def _per_call_equal(reqs, interp):
    import torch
    from noa_b200 import fourier_project as fp
    for r in reqs:
        count, n = r.slice_shape[0], r.slice_shape[2]
        ref = torch.zeros((count, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        fp.extract_central_slices_3d("hc2h", r.volume, None, r.volume_shape, ref, None, r.slice_shape, None,
                                     r.fwd_rotation, interp=interp)
        torch.cuda.synchronize()
        assert torch.equal(r.slice, ref)


# Enough items that the persistent kernel claims several consecutive items at a time (more than
# 2 x 64 per CTA), so runs cross slice and request boundaries inside one claim.
LARGE = [(128, 1500), (96, 2000), (112, 1201), (64, 903), (128, 700), (80, 1000), (112, 37)]


@pytest.mark.parametrize("interp", ["linear", "cubic"])
def test_batch_long_claims_match_per_call(interp, tmp_path, monkeypatch):
    import torch
    from noa_b200.batch import ExtractBatch
    monkeypatch.setenv("NB_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    # LINEAR batches read pair copies, whose items are 64 x 16 pixels: 4x the slices for as many claims
    reqs, _ = _large_requests([(n, 4 * c) for n, c in LARGE] if interp == "linear" else LARGE)
    batch = ExtractBatch("hc2h", reqs, interp=interp, autotune=False, persistent_only=True)
    info = batch.info()
    assert info["n_items"] // (info["grid"] * 64) >= 2 and info["n_direct"] == 0, info
    batch.run()
    torch.cuda.synchronize()
    _per_call_equal(reqs, interp)
    batch.close()


def test_batch_direct_grids_match_per_call(tmp_path, monkeypatch):
    """A LINEAR batch whose large requests run as grids of their own on graph branches (while the
    other volumes' pair copies are made) and whose small ones go through the persistent kernel: both
    bit-identical to the per-call entry point, over two replays."""
    import torch
    from noa_b200.batch import ExtractBatch
    monkeypatch.setenv("NB_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    # 2^16 output pixels: 32 slices of 64 x 33 reach it, 20 do not; the 112^3 volume is read by too
    # few pixels for a pair copy (generic LINEAR path, in the persistent kernel)
    spec = [(128, 1009), (64, 3980), (64, 20), (64, 32), (112, 5), (128, 300)]
    reqs, _ = _large_requests(spec, seed=9)
    batch = ExtractBatch("hc2h", reqs, interp="linear", autotune=True)
    info = batch.info()
    assert info["n_direct"] == 4 and info["n_requests"] == len(spec) and info["n_items"] > 0, info
    for _ in range(2):
        for r in reqs:
            r.slice.fill_(7)
        batch.run()
        torch.cuda.synchronize()
        _per_call_equal(reqs, "linear")
    batch.close()
    # every request direct: no persistent kernel in the graph
    reqs, _ = _large_requests([(128, 1009), (128, 1100)], seed=10)
    batch = ExtractBatch("hc2h", reqs, interp="linear", autotune=False)
    assert batch.info()["n_direct"] == 2 and batch.info()["n_items"] == 0
    batch.run()
    torch.cuda.synchronize()
    _per_call_equal(reqs, "linear")
    batch.close()


def test_resident_pairs_long_claims_match_per_call():
    import torch
    from noa_b200.batch import extract_batch_launch, volume_pairs
    # pair-copy items are 64 x 16 pixels: more slices for the same number of claims
    reqs, vols = _large_requests([(n, 4 * c) for n, c in LARGE], seed=5)
    pairs = {n: volume_pairs(v, (1, n, n, n)) for n, v in vols.items()}
    extract_batch_launch("hc2h", reqs, [pairs[r.slice_shape[2]] for r in reqs], persistent_only=True)
    torch.cuda.synchronize()
    _per_call_equal(reqs, "linear")
    # the same requests, those of at least 2^21 output pixels as grids of their own
    for r in reqs:
        r.slice.fill_(7)
    extract_batch_launch("hc2h", reqs, [pairs[r.slice_shape[2]] for r in reqs])
    torch.cuda.synchronize()
    _per_call_equal(reqs, "linear")


def test_linear_batch_pair_copies_follow_volume_updates(tmp_path, monkeypatch):
    """LINEAR batches read pair copies that the graph rebuilds at every run: a volume changed between
    runs is seen, and results stay those of the per-call entry point."""
    import torch
    from noa_b200.batch import ExtractBatch
    monkeypatch.setenv("NB_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    reqs, vols = _large_requests([(64, 300), (96, 150), (64, 40)], seed=9)
    batch = ExtractBatch("hc2h", reqs, interp="linear", autotune=True)
    batch.run()
    torch.cuda.synchronize()
    _per_call_equal(reqs, "linear")
    for v in vols.values():
        v.mul_(-0.5).add_(0.25)
    for r in reqs:
        r.slice.fill_(3)
    batch.run()
    torch.cuda.synchronize()
    _per_call_equal(reqs, "linear")
    batch.close()


def test_linear_batch_scaled_and_curved_match_per_call(tmp_path, monkeypatch):
    """Scaled requests and the Ewald curvature go through the batch's pair copies too (coordinates by
    the same slice2grid): results are the per-call ones, bit for bit."""
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    from noa_b200.batch import ExtractBatch
    monkeypatch.setenv("NB_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    reqs, _ = _large_requests([(64, 300), (48, 400)], seed=13)
    for i, r in enumerate(reqs):
        count = r.slice_shape[0]
        sc = synthetic.scale_matrices(count, (1.0, 1.0), seed=80 + i, jitter=0.05).astype(np.float32)
        r.inv_scaling = torch.from_numpy(sc).cuda()
    ews = (45.0, 60.0)
    batch = ExtractBatch("hc2h", reqs, interp="linear", ews_radius=ews, autotune=False)
    batch.run()
    torch.cuda.synchronize()
    for r in reqs:
        count, n = r.slice_shape[0], r.slice_shape[2]
        ref = torch.zeros((count, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        fp.extract_central_slices_3d("hc2h", r.volume, None, r.volume_shape, ref, None, r.slice_shape, r.inv_scaling,
                                     r.fwd_rotation, interp="linear", ews_radius=ews)
        torch.cuda.synchronize()
        assert torch.equal(r.slice, ref)
    batch.close()


# ---------------------------------------------------------------------------------------------------
# Batched rasterization: each request of one launch equals its own per-call rasterization (the same
# terms; the atomic summation order may differ) and the oracle within the rasterization bar.
# ---------------------------------------------------------------------------------------------------
def _raster_requests(out_dt="c32", weights=True, counts=((32, 10), (48, 3), (64, 25), (40, 7)), seed=30):
    import torch
    from noa_b200 import synthetic
    from noa_b200.batch import RasterizeRequest
    reqs = []
    for i, (n, count) in enumerate(counts):
        sl = synthetic.make_slices(count, n, seed=seed + i)
        if out_dt == "f32":
            sl = np.ascontiguousarray(sl.real)
        rot = synthetic.random_rotations(count, seed=seed + 20 + i)
        dt = torch.complex64 if out_dt == "c32" else torch.float32
        reqs.append(RasterizeRequest(
            slice=torch.from_numpy(sl).cuda(), slice_shape=(count, 1, n, n),
            volume=torch.zeros((1, n, n, n // 2 + 1), dtype=dt, device="cuda"), volume_shape=(1, n, n, n),
            volume_weight=torch.zeros((1, n, n, n // 2 + 1), dtype=torch.float32, device="cuda") if weights else None,
            fwd_rotation=torch.from_numpy(rot).cuda()))
    return reqs


@pytest.mark.parametrize("out_dt,weights", [("c32", True), ("c32", False), ("f32", True)])
def test_rasterize_batch_matches_per_call_and_oracle(out_dt, weights):
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200.batch import rasterize_batch_launch
    from oracle.oracle import Call, FpOracle
    reqs = _raster_requests(out_dt, weights)
    rasterize_batch_launch("h2hc", reqs)
    torch.cuda.synchronize()
    for r in reqs:
        v = torch.zeros_like(r.volume)
        w = torch.zeros_like(r.volume_weight) if weights else None
        fp.rasterize_central_slices_3d("h2hc", r.slice, None, r.slice_shape, v, w, r.volume_shape, None,
                                       r.fwd_rotation)
        torch.cuda.synchronize()
        assert rel_l2(r.volume.cpu().numpy(), v.cpu().numpy()) <= 1e-6
        call = Call(func="rasterize", remap="h2hc", inp=r.slice.cpu().numpy(), in_shape=r.slice_shape,
                    out=np.zeros(tuple(r.volume.shape), np.complex64 if out_dt == "c32" else np.float32),
                    out_shape=r.volume_shape, rot=r.fwd_rotation.cpu().numpy(),
                    out_w=np.zeros(tuple(r.volume.shape), np.float32) if weights else None)
        FpOracle().run(call, 4)
        assert rel_l2(r.volume.cpu().numpy(), call.out) <= 1e-4
        if weights:
            assert rel_l2(w.cpu().numpy(), r.volume_weight.cpu().numpy()) <= 1e-6
            assert rel_l2(r.volume_weight.cpu().numpy(), call.out_w) <= 1e-4


def test_rasterize_batch_rejects_shared_grids_and_mixed_types():
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200.batch import rasterize_batch_launch
    reqs = _raster_requests(counts=((32, 3), (32, 4)))
    reqs[1].volume = reqs[0].volume  # both requests would add into the same grid
    with pytest.raises(fp.NoaB200Error) as e:
        rasterize_batch_launch("h2hc", reqs)
    assert e.value.code == fp.NB_ERROR_INVALID and "disjoint" in str(e.value)
    reqs = _raster_requests(counts=((32, 3), (32, 4)))
    reqs[1].volume_weight = None
    with pytest.raises(fp.NoaB200Error) as e:
        rasterize_batch_launch("h2hc", reqs)
    assert e.value.code == fp.NB_ERROR_INVALID
    torch.cuda.synchronize()
