"""Known-answer identities of noa's own xform tests, on the CUDA path (no golden data needed).

* rasterize: hc2hc == hc2h then remap h2hc, h2hc == h2h then remap h2hc
  (TestXformFourierInsertRasterize.cpp:72-120, linspace slices, rotations about y by 2i degrees,
  cutoff 0.45, abs 5e-5);
* rasterize: the weight grid of real slices given as their own weights equals the value grid
  (TestXformFourierInsertRasterize.cpp:122-152);
* extract: hc2hc == hc2h then remap h2hc (TestXformFourierExtract.cpp:116-153, linspace volume);
* insert_and_extract: hc2hc == hc2h then remap h2hc, and the weights of real inputs given as their own
  weights equal the values (TestXformFourierInsertInterpolateExtract.cpp:89-182, input windowed sinc
  0.01, cutoff 0.8);
* Mat33 == quaternion for the same rotations (TestXformFourierInsertInterpolateExtract.cpp:231-285
  compares the two rotation types), within rounding of the two rotate() forms.

noa checks these with allclose_abs_safe at 5e-5; the same check is used here, and the identities are
asserted bit for bit where the GPU path makes them exact (extraction remaps only move pixels; a value
and its weight ride in one reduction).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rfft(shape):
    return tuple(shape[:-1]) + (shape[-1] // 2 + 1,)


def _linspace(shape, start, stop, dtype):
    """noa::linspace over an array: values start..stop (endpoint included) in memory order."""
    n = int(np.prod(shape))
    v = np.linspace(start, stop, n, endpoint=True).reshape(shape)
    return v.astype(np.complex64) if dtype == "c32" else v.astype(np.float32)


def _rot_y(degrees):
    """Rotations about the y axis (euler2matrix({0, a, 0}, "zyx")), acting on (z, y, x) vectors."""
    out = []
    for d in degrees:
        a = np.deg2rad(d)
        c, s = np.cos(a), np.sin(a)
        out.append([[c, 0.0, -s], [0.0, 1.0, 0.0], [s, 0.0, c]])
    return np.asarray(out, dtype=np.float32)


def _h2hc(t, axes):
    """noa::fft::remap("h2hc"): fftshift of the non-redundant layout along the given full axes."""
    import torch
    return torch.fft.fftshift(t, dim=axes)


def _abs_close(a, b, eps=5e-5):
    """noa's test::allclose_abs_safe (tests/Utils.hpp:331-355): per real and imaginary component,
    |a - b| <= eps, or |a - b| <= max(|a|, |b|) * eps."""
    import torch
    if a.is_complex():
        a, b = torch.view_as_real(a), torch.view_as_real(b)
    d = (a - b).abs()
    ok = torch.isfinite(d) & ((d <= eps) | (d <= torch.maximum(a.abs(), b.abs()) * eps))
    assert bool(ok.all()), (d.max().item(), int((~ok).sum()))


@pytest.mark.parametrize("dtype", ["f32", "c32"])
def test_rasterize_remaps(dtype):
    import torch
    from noa_b200 import fourier_project as fp
    sshape, gshape = (20, 1, 64, 64), (1, 128, 128, 128)
    tdt = torch.complex64 if dtype == "c32" else torch.float32
    slices = torch.from_numpy(_linspace(_rfft(sshape), 1, 10, dtype)).cuda()
    rot = torch.from_numpy(_rot_y([2 * i for i in range(sshape[0])])).cuda()
    grids = [torch.zeros(_rfft(gshape), dtype=tdt, device="cuda") for _ in range(2)]
    for centered_in in (True, False):
        for g in grids:
            g.zero_()
        src = "hc" if centered_in else "h"
        fp.rasterize_central_slices_3d(f"{src}2hc", slices, None, sshape, grids[0], None, gshape, None, rot,
                                       fftfreq_cutoff=0.45)
        fp.rasterize_central_slices_3d(f"{src}2h", slices, None, sshape, grids[1], None, gshape, None, rot,
                                       fftfreq_cutoff=0.45)
        torch.cuda.synchronize()
        assert grids[0].abs().max().item() > 1.0  # something was rasterized
        _abs_close(grids[0], _h2hc(grids[1], (1, 2)))


def test_rasterize_weights_equal_values_of_real_slices():
    import torch
    from noa_b200 import fourier_project as fp
    sshape, gshape = (20, 1, 64, 64), (1, 64, 64, 64)
    rng = np.random.default_rng(3)
    slices = torch.from_numpy(rng.uniform(-10, 10, _rfft(sshape)).astype(np.float32)).cuda()
    rot = torch.from_numpy(_rot_y([2 * i for i in range(sshape[0])])).cuda()
    grid = torch.zeros(_rfft(gshape), dtype=torch.float32, device="cuda")
    grid_w = torch.zeros_like(grid)
    fp.rasterize_central_slices_3d("hc2hc", slices, slices.clone(), sshape, grid, grid_w, gshape, None, rot,
                                   fftfreq_cutoff=0.45)
    torch.cuda.synchronize()
    # value and weight ride in the same reduction (one element per tap): equal bit for bit
    assert torch.equal(grid, grid_w)
    assert grid.abs().max().item() > 1.0


@pytest.mark.parametrize("dtype", ["f32", "c32"])
def test_extract_remap(dtype):
    import torch
    from noa_b200 import fourier_project as fp
    sshape, gshape = (20, 1, 128, 128), (1, 128, 128, 128)
    tdt = torch.complex64 if dtype == "c32" else torch.float32
    grid = torch.from_numpy(_linspace(_rfft(gshape), -50, 50, dtype)).cuda()
    rot = torch.from_numpy(_rot_y([2 * i for i in range(sshape[0])])).cuda()
    out = [torch.full(_rfft(sshape), 7, dtype=tdt, device="cuda") for _ in range(2)]
    fp.extract_central_slices_3d("hc2hc", grid, None, gshape, out[0], None, sshape, None, rot, fftfreq_cutoff=0.45)
    fp.extract_central_slices_3d("hc2h", grid, None, gshape, out[1], None, sshape, None, rot, fftfreq_cutoff=0.45)
    torch.cuda.synchronize()
    # the remap only moves output pixels: the same interpolation per pixel, bit for bit
    assert torch.equal(out[0], _h2hc(out[1], (2,)))


def _ie_rotations(n_in, n_out):
    inv_in = _rot_y([-2 * i for i in range(n_in)])
    fwd_out = _rot_y([2 * i + 1 for i in range(n_out)])
    return inv_in, fwd_out


@pytest.mark.parametrize("dtype", ["f32", "c32"])
def test_insert_and_extract_remap(dtype):
    import torch
    from noa_b200 import fourier_project as fp
    ishape, oshape = (20, 1, 256, 256), (5, 1, 256, 256)
    tdt = torch.complex64 if dtype == "c32" else torch.float32
    inp = torch.from_numpy(_linspace(_rfft(ishape), -50, 50, dtype)).cuda()
    inv_in, fwd_out = (torch.from_numpy(r).cuda() for r in _ie_rotations(ishape[0], oshape[0]))
    out = [torch.full(_rfft(oshape), 7, dtype=tdt, device="cuda") for _ in range(2)]
    ws = fp.WindowedSinc(0.01)
    for remap, o in zip(("hc2hc", "hc2h"), out):
        fp.insert_and_extract_central_slices_3d(remap, inp, None, ishape, o, None, oshape, None, inv_in, None, fwd_out,
                                                input_windowed_sinc=ws, fftfreq_cutoff=0.8)
    torch.cuda.synchronize()
    assert out[0].abs().max().item() > 1.0
    _abs_close(out[0], _h2hc(out[1], (2,)))


def test_insert_and_extract_weights_equal_values_of_real_inputs():
    import torch
    from noa_b200 import fourier_project as fp
    ishape, oshape = (20, 1, 256, 256), (5, 1, 256, 256)
    rng = np.random.default_rng(4)
    inp = torch.from_numpy(rng.uniform(-10, 10, _rfft(ishape)).astype(np.float32)).cuda()
    inv_in, fwd_out = (torch.from_numpy(r).cuda() for r in _ie_rotations(ishape[0], oshape[0]))
    out = torch.full(_rfft(oshape), 7, dtype=torch.float32, device="cuda")
    out_w = torch.full_like(out, 7)
    fp.insert_and_extract_central_slices_3d("hc2hc", inp, inp.clone(), ishape, out, out_w, oshape, None, inv_in, None,
                                            fwd_out, input_windowed_sinc=fp.WindowedSinc(0.01), fftfreq_cutoff=0.8)
    torch.cuda.synchronize()
    assert out.abs().max().item() > 1.0
    _abs_close(out, out_w)


def test_mat33_and_quaternion_rotations_agree():
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    n, count = 64, 32
    vol = torch.from_numpy(synthetic.make_volume(n, seed=5)).cuda()
    q = synthetic.random_quaternions(count, seed=6)
    mats = torch.from_numpy(synthetic.quaternion_to_matrix(q).astype(np.float32)).cuda()
    quats = torch.from_numpy(q.astype(np.float32)).cuda()
    outs = []
    # cutoff 0.45: no pixel lies within rounding of the cutoff sphere (|(v, u)|^2 = 829.44 has no
    # integer solution), so both rotation forms keep the same pixels
    for rot in (mats, quats):
        o = torch.empty((count, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), o, None, (count, 1, n, n), None, rot,
                                     fftfreq_cutoff=0.45)
        outs.append(o)
    grids = []
    for rot in (mats, quats):
        g = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        fp.rasterize_central_slices_3d("h2hc", outs[0], None, (count, 1, n, n), g, None, (1, n, n, n), None, rot,
                                       fftfreq_cutoff=0.45)
        grids.append(g)
    torch.cuda.synchronize()
    for a, b in ((outs[0], outs[1]), (grids[0], grids[1])):
        rel = ((a - b).abs().pow(2).sum() / b.abs().pow(2).sum()).sqrt().item()
        assert rel <= 1e-5, rel


def test_extract_and_rasterize_are_adjoint():
    """<extract(V), S> == <V, rasterize(S)> for the trilinear pair (an identity the scope adds to noa's
    tests): real V and S, forward rotations shared, hc2h / h2hc layouts, cutoff 0.45. The rasterizer's
    extra taps on the redundant x == 0 plane (FourierProject.hpp:347-372) have no counterpart in the
    extraction, so V is zero on that plane, which makes them drop out of <V, rasterize(S)>; the Friedel
    flips of both sides are the same reflection for real data."""
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    n, count = 96, 24
    rng = np.random.default_rng(8)
    v = rng.uniform(0.0, 1.0, (1, n, n, n // 2 + 1)).astype(np.float32)
    v[..., 0] = 0.0
    s = rng.uniform(0.0, 1.0, (count, 1, n, n // 2 + 1)).astype(np.float32)
    rot = torch.from_numpy(synthetic.quaternion_to_matrix(synthetic.random_quaternions(count, seed=9))
                           .astype(np.float32)).cuda()
    vol, slices = torch.from_numpy(v).cuda(), torch.from_numpy(s).cuda()
    ext = torch.empty_like(slices)
    fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), ext, None, (count, 1, n, n), None, rot,
                                 fftfreq_cutoff=0.45)
    grid = torch.zeros_like(vol)
    fp.rasterize_central_slices_3d("h2hc", slices, None, (count, 1, n, n), grid, None, (1, n, n, n), None, rot,
                                   fftfreq_cutoff=0.45)
    torch.cuda.synchronize()
    lhs = float((ext.double() * slices.double()).sum())
    rhs = float((vol.double() * grid.double()).sum())
    assert lhs > 1e3
    assert abs(lhs - rhs) <= 1e-5 * lhs, (lhs, rhs)
