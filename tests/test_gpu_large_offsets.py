"""GPU: arrays whose element offsets need 64 bits.

An array whose last element lies 2^31 or more elements past its first takes the kernels' 64-bit index
paths (the generic extraction kernel's Idx = int64, the pair copy's 64-bit source offsets, the 64-bit
output offsets of every store). Here a 64^3 rfft volume (and grid) is laid out with a depth stride of
35,000,000 elements inside one 17.6 GB allocation, so it spans 2.2 G elements while holding 135 k, and
every call on it must equal, bit for bit (extraction) or to 1e-6 (rasterization, atomic order), the
same call on a contiguous copy.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 64
DEPTH_STRIDE = 35_000_000  # 63 x 35e6 = 2.2e9 >= 2^31 - 1


def _wide_view(buf):
    import torch
    wp = N // 2 + 1
    return torch.as_strided(buf, (1, N, N, wp), (N * DEPTH_STRIDE, DEPTH_STRIDE, wp, 1))


@pytest.fixture(scope="module")
def big_buffer():
    import torch
    wp = N // 2 + 1
    span = (N - 1) * DEPTH_STRIDE + (N - 1) * wp + wp
    buf = torch.empty(span, dtype=torch.complex64, device="cuda")
    yield buf
    del buf
    torch.cuda.empty_cache()


@pytest.mark.parametrize("count", [8, 400], ids=["generic", "pair_copy"])
def test_extract_from_a_volume_spanning_2_31_elements(big_buffer, count):
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    compact = torch.from_numpy(synthetic.make_volume(N, seed=31)).cuda()
    wide = _wide_view(big_buffer)
    wide.copy_(compact)
    assert (wide.shape[1] - 1) * wide.stride(1) >= 2 ** 31 - 1
    rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(count, seed=32)).cuda())
    outs = []
    for vol in (wide, compact):
        o = torch.full((count, 1, N, N // 2 + 1), 7, dtype=torch.complex64, device="cuda")
        fp.extract_central_slices_3d("hc2h", vol, None, (1, N, N, N), o, None, (count, 1, N, N), None, rot)
        outs.append(o)
    torch.cuda.synchronize()
    assert outs[1].abs().max().item() > 0
    assert torch.equal(outs[0], outs[1])


def test_rasterize_into_a_grid_spanning_2_31_elements(big_buffer):
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    count = 40
    slices = torch.from_numpy(synthetic.make_slices(count, N, seed=33)).cuda()
    rot = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(count, seed=34)).cuda())
    wide = _wide_view(big_buffer)
    wide.zero_()
    compact = torch.zeros((1, N, N, N // 2 + 1), dtype=torch.complex64, device="cuda")
    for grid in (wide, compact):
        fp.rasterize_central_slices_3d("h2hc", slices, None, (count, 1, N, N), grid, None, (1, N, N, N), None, rot)
    torch.cuda.synchronize()
    got = wide.contiguous()
    rel = float(((got - compact).abs().pow(2).sum() / compact.abs().pow(2).sum()).sqrt())
    assert compact.abs().max().item() > 0 and rel <= 1e-6, rel
