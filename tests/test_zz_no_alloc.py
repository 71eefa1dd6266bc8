"""The allocation-free rasterization entry point against the regular one (GPU, through the C ABI).

nb_rasterize_central_slices_3d_static_scratch exists for callers that cannot let the library allocate
device memory at call time; it keeps its accumulator in a fixed 64 MiB array of the library's device
code (reserved on a GPU by its first call there, under CUDA's default lazy module loading). It must
give the regular entry point's results (rasterization tolerance: relative L2 1e-4), also on a second
call in a row, which shows that the shared array is cleared between calls, and up to the largest
volume the array holds; one stored column more per row is refused. This file is collected last on
purpose.
"""
import numpy as np
import pytest

from cases import build, default_case, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _run(entry, call, vol, volw):
    import torch
    from noa_b200 import fourier_project as fp
    slices = torch.from_numpy(call.inp).cuda()
    rot = fp.pack_rotations(torch.from_numpy(call.rot).cuda())  # noa's Mat33 layout, made before the call
    getattr(fp, entry)(call.remap, slices, None, call.in_shape, vol, volw, call.out_shape, None, rot,
                       fftfreq_cutoff=call.cutoff)


@pytest.mark.parametrize("dts", [("c32", "c32"), ("c32", "f32"), ("f32", "f32")])
@pytest.mark.parametrize("weights", [True, False])
def test_static_scratch_matches_regular_entry_point_twice(dts, weights):
    import torch
    n = 64
    first = build(default_case("rasterize", remap="h2hc", n=n, nslices=48, in_dt=dts[0], out_dt=dts[1],
                               out_w=weights, seed=900))
    second = build(default_case("rasterize", remap="h2hc", n=n, nslices=48, in_dt=dts[0], out_dt=dts[1],
                                out_w=weights, seed=901))
    dt = torch.complex64 if dts[1] == "c32" else torch.float32
    shape = (1, n, n, n // 2 + 1)
    ref_v = torch.zeros(shape, dtype=dt, device="cuda")
    ref_w = torch.zeros(shape, dtype=torch.float32, device="cuda") if weights else None
    new_v = torch.zeros(shape, dtype=dt, device="cuda")
    new_w = torch.zeros(shape, dtype=torch.float32, device="cuda") if weights else None
    for call in (first, second):
        _run("rasterize_central_slices_3d", call, ref_v, ref_w)
        _run("rasterize_central_slices_3d_static_scratch", call, new_v, new_w)
        torch.cuda.synchronize()
        assert rel_l2(new_v.cpu().numpy(), ref_v.cpu().numpy()) <= TOL
        if weights:
            assert rel_l2(new_w.cpu().numpy(), ref_w.cpu().numpy()) <= TOL


def test_static_scratch_rejects_volumes_beyond_its_capacity():
    import torch
    from noa_b200 import fourier_project as fp
    n = 256  # 256 x 256 x 129 complex voxels need 135 MB of accumulator, more than 64 MiB
    call = build(default_case("rasterize", remap="h2hc", n=16, nslices=2, seed=902))
    slices = torch.zeros((2, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    vol = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    volw = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.float32, device="cuda")
    rot = fp.pack_rotations(torch.from_numpy(call.rot).cuda())
    with pytest.raises(fp.NoaB200Error) as e:
        fp.rasterize_central_slices_3d_static_scratch("h2hc", slices, None, (2, 1, n, n), vol, volw, (1, n, n, n),
                                                      None, rot)
    assert e.value.code == fp.NB_ERROR_INVALID and "static scratch" in str(e.value)


@pytest.mark.parametrize("cplx", [False, True], ids=["real", "complex"])
def test_static_scratch_at_its_capacity_and_just_beyond(cplx):
    """With weights the array holds 8,388,608 real (8 bytes each) or 4,194,304 complex (16 bytes) rfft
    voxels. The largest accepted grids here are exactly that: 256 x 256 x 128 (real) and 128 x 256 x 128
    (complex), logical width 254. Widening the logical width to 256 (129 stored columns) goes beyond."""
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    d = 128 if cplx else 256
    h, w = 256, 254
    assert d * h * (w // 2 + 1) * (16 if cplx else 8) == 64 << 20
    dt = torch.complex64 if cplx else torch.float32
    b = 4
    rng = np.random.default_rng(903)
    vals = rng.standard_normal((b, 1, h, w // 2 + 1)).astype(np.float32)
    if cplx:
        vals = (vals + 1j * rng.standard_normal(vals.shape)).astype(np.complex64)
    slices = torch.from_numpy(vals).cuda()
    rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(b, seed=904)).cuda())
    shape = (1, d, h, w // 2 + 1)
    outs = []
    for entry in ("rasterize_central_slices_3d", "rasterize_central_slices_3d_static_scratch"):
        v = torch.zeros(shape, dtype=dt, device="cuda")
        vw = torch.zeros(shape, dtype=torch.float32, device="cuda")
        getattr(fp, entry)("h2hc", slices, None, (b, 1, h, w), v, vw, (1, d, h, w), None, rot)
        torch.cuda.synchronize()
        outs.append((v.cpu().numpy(), vw.cpu().numpy()))
    assert np.abs(outs[0][1]).sum() > 0
    assert rel_l2(outs[1][0], outs[0][0]) <= TOL
    assert rel_l2(outs[1][1], outs[0][1]) <= TOL

    w2 = 256  # one more stored column per row: beyond the array
    big = torch.zeros((1, d, h, w2 // 2 + 1), dtype=dt, device="cuda")
    bigw = torch.zeros((1, d, h, w2 // 2 + 1), dtype=torch.float32, device="cuda")
    sl2 = torch.zeros((b, 1, h, w2 // 2 + 1), dtype=dt, device="cuda")
    with pytest.raises(fp.NoaB200Error) as e:
        fp.rasterize_central_slices_3d_static_scratch("h2hc", sl2, None, (b, 1, h, w2), big, bigw, (1, d, h, w2),
                                                      None, rot)
    assert e.value.code == fp.NB_ERROR_INVALID and "static scratch" in str(e.value)
