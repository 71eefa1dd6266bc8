"""GPU: the paths a call takes when the library cannot allocate its scratch memory.

``nb_set_scratch_limit`` caps the size of one allocation the library makes on its own, and an
allocation above the cap fails exactly as an out-of-memory one does. With it these tests drive, on
purpose, what only a full device would otherwise reach, and check each against the oracle (the C
restatement pinned to noa's CPU path) and against the unconstrained path:

  extraction without the pair copy        -> the generic kernel reads the volume (bit-identical)
  rasterization without the padded grid   -> unpadded scratch, or reductions into the caller's grids
  scatter insertion without its grid      -> the gather form (bit-identical to it)
  one-shot batched launch, batch creation -> NB_ERROR_OOM when the descriptors cannot be allocated;
                                             LINEAR batches without pair copies read the volumes
  the static-scratch rasterization        -> allocates nothing, so the cap does not change it

noa reports a failed allocation as a noa::Exception (base/Error.hpp:115-168, runtime/cuda/Error.hpp);
this library's counterpart is the NB_ERROR_OOM status, or a slower path with the same results where one
exists.
"""
import numpy as np
import pytest

from cases import build, clone, default_case, rel_l2
from oracle.oracle import FpOracle

pytestmark = pytest.mark.gpu


@pytest.fixture
def cap():
    """Sets a scratch cap for the test and removes it afterwards, whatever happens."""
    from noa_b200 import fourier_project as fp
    yield fp.set_scratch_limit
    fp.set_scratch_limit(None)


def _oracle(call):
    ref = clone(call)
    assert FpOracle().run(ref, 8) == 0
    return ref


def test_limit_is_reported_and_removed(cap):
    from noa_b200 import fourier_project as fp
    assert fp.scratch_limit() is None
    cap(12345)
    assert fp.scratch_limit() == 12345
    cap(None)
    assert fp.scratch_limit() is None
    with pytest.raises(fp.NoaB200Error) as e:
        fp.set_scratch_limit(0, device=4096)
    assert e.value.code == fp.NB_ERROR_INVALID


@pytest.mark.parametrize("remap", ["hc2h", "h2hc"])
def test_extract_without_pair_copy(cap, remap):
    import gpu_run
    call = build(default_case("extract", n=64, nslices=64, remap=remap, seed=701))  # pair path when uncapped
    ref = _oracle(call)
    fast, _ = gpu_run.run(clone(call))
    cap(0)
    slow, _ = gpu_run.run(clone(call))
    assert rel_l2(slow, ref.out) <= 1e-5
    np.testing.assert_array_equal(slow, fast)


@pytest.mark.parametrize("in_dt,out_dt,out_w,limit", [
    ("c32", "c32", True, 0), ("c32", "c32", True, 2_500_000), ("c32", "c32", False, 0),
    ("c32", "f32", True, 1_250_000), ("f32", "f32", True, 0)],
    ids=["c32-w-direct", "c32-w-unpadded", "c32-direct", "c32f32-w-unpadded", "f32-w-direct"])
def test_rasterize_without_padded_accumulator(cap, in_dt, out_dt, out_w, limit):
    """At 64^3 with weights the padded accumulator is 2.9 MB (1.45 MB for real values) and the unpadded
    one 2.2 MB (1.1 MB), so these caps take the unpadded scratch, and a 0 cap the reductions straight
    into the caller's grids."""
    import gpu_run
    call = build(default_case("rasterize", n=64, nslices=24, remap="h2hc", in_dt=in_dt, out_dt=out_dt,
                              out_w=out_w, seed=702))
    ref = _oracle(call)
    cap(limit)
    out, got_w = gpu_run.run(clone(call))
    assert rel_l2(out, ref.out) <= 1e-4
    if out_w:
        assert rel_l2(got_w, ref.out_w) <= 1e-4


def test_scatter_insert_without_accumulator_is_the_gather_form(cap):
    import gpu_run
    call = build(default_case("insert", n=40, nslices=30, out_w=True, sinc=(-1.0, 6 / 40), remap="hc2hc",
                              seed=703))
    ref = _oracle(call)
    from noa_b200 import fourier_project as fp
    gather, gather_w = gpu_run.run(clone(call))
    cap(0)
    before = fp.scratch_refusals()
    out, out_w = gpu_run.run(clone(call), scatter=True)
    assert fp.scratch_refusals() == before + 1  # the refused accumulator is counted
    np.testing.assert_array_equal(out, gather)
    np.testing.assert_array_equal(out_w, gather_w)
    assert rel_l2(out, ref.out) <= 1e-5


def _batch_requests():
    import torch
    from noa_b200 import synthetic
    from noa_b200.batch import ExtractRequest
    reqs, specs = [], []
    for i, (n, count) in enumerate([(64, 300), (48, 9)]):
        vol = torch.from_numpy(synthetic.make_volume(n, seed=710 + i)).cuda()
        rot = torch.from_numpy(synthetic.random_rotations(count, seed=720 + i)).cuda()
        out = torch.zeros((count, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        reqs.append(ExtractRequest(volume=vol, volume_shape=(1, n, n, n), slice=out, slice_shape=(count, 1, n, n),
                                   fwd_rotation=rot))
        specs.append((vol, rot, n, count))
    return reqs, specs


def test_batch_out_of_memory_is_reported(cap):
    from noa_b200 import batch
    from noa_b200 import fourier_project as fp
    reqs, _ = _batch_requests()
    cap(0)
    with pytest.raises(fp.NoaB200Error) as e:
        batch.extract_batch_launch("hc2h", reqs)
    assert e.value.code == fp.NB_ERROR_OOM
    with pytest.raises(fp.NoaB200Error) as e:
        batch.ExtractBatch("hc2h", reqs, autotune=False)
    assert e.value.code == fp.NB_ERROR_OOM


def test_batch_without_pair_copies_matches_per_call(cap):
    """A 1 MB cap leaves room for the descriptors but not for the 64^3 pair copy (2.2 MB)."""
    import torch
    from noa_b200 import batch
    from noa_b200 import fourier_project as fp
    reqs, specs = _batch_requests()
    cap(1 << 20)
    b = batch.ExtractBatch("hc2h", reqs, autotune=False)
    b.run()
    torch.cuda.synchronize()
    cap(None)
    for r, (vol, rot, n, count) in zip(reqs, specs):
        ref = torch.zeros((count, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), ref, None, (count, 1, n, n), None, rot)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(r.slice.cpu().numpy(), ref.cpu().numpy())
    b.close()


def test_static_scratch_rasterization_ignores_the_cap(cap):
    import torch
    from noa_b200 import fourier_project as fp
    call = build(default_case("rasterize", n=32, nslices=12, remap="h2hc", out_w=True, seed=704))
    ref = _oracle(call)
    cap(0)
    n = 32
    out = torch.zeros(call.out.shape, dtype=torch.complex64, device="cuda")
    out_w = torch.zeros(call.out_w.shape, dtype=torch.float32, device="cuda")
    fp.rasterize_central_slices_3d_static_scratch("h2hc", torch.from_numpy(call.inp).cuda(), None,
                                                  (12, 1, n, n), out, out_w, (1, n, n, n), None,
                                                  torch.from_numpy(call.rot).cuda())
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref.out) <= 1e-4
    assert rel_l2(out_w.cpu().numpy(), ref.out_w) <= 1e-4
