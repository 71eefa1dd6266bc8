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
