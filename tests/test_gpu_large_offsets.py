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


def _wide_slices(buf, count):
    """count slices of N x (N/2+1) whose rows lie 35 M elements apart (the slices interleaved along x,
    batch stride N/2+1): offsets within one slice need 64 bits."""
    import torch
    wp = N // 2 + 1
    assert count * wp <= DEPTH_STRIDE
    return torch.as_strided(buf, (count, 1, N, wp), (wp, wp, DEPTH_STRIDE, 1))


def test_insertions_from_slices_spanning_2_31_elements(big_buffer):
    import torch
    from noa_b200 import fourier_project as fp
    from noa_b200 import synthetic
    count = 24
    compact = torch.from_numpy(synthetic.make_slices(count, N, seed=35)).cuda()
    wide = _wide_slices(big_buffer, count)
    wide.copy_(compact)
    assert (wide.shape[2] - 1) * wide.stride(2) >= 2 ** 31 - 1
    rot = torch.from_numpy(synthetic.random_rotations(count, seed=36)).cuda()
    inv = fp.pack_rotations(rot.transpose(1, 2).contiguous())
    fwd = fp.pack_rotations(rot)
    rot_out = fp.pack_rotations(torch.from_numpy(synthetic.random_rotations(5, seed=37)).cuda())
    ws = fp.WindowedSinc(-1.0, 3.0 / N)
    res = {}
    for name, sl in (("wide", wide), ("compact", compact)):
        g = torch.zeros((1, N, N, N // 2 + 1), dtype=torch.complex64, device="cuda")
        gs = torch.zeros_like(g)
        gr = torch.zeros_like(g)
        o = torch.full((5, 1, N, N // 2 + 1), 7, dtype=torch.complex64, device="cuda")
        fp.insert_central_slices_3d("h2hc", sl, None, (count, 1, N, N), g, None, (1, N, N, N), None, inv,
                                    windowed_sinc=ws)
        fp.insert_central_slices_3d_scatter("h2hc", sl, None, (count, 1, N, N), gs, None, (1, N, N, N), None, inv,
                                            windowed_sinc=ws)
        fp.rasterize_central_slices_3d("h2hc", sl, None, (count, 1, N, N), gr, None, (1, N, N, N), None, fwd)
        fp.insert_and_extract_central_slices_3d("h2h", sl, None, (count, 1, N, N), o, None, (5, 1, N, N), None, inv,
                                                None, rot_out, input_windowed_sinc=ws)
        res[name] = (g, gs, gr, o)
    torch.cuda.synchronize()
    (g, gs, gr, o), (g2, gs2, gr2, o2) = res["wide"], res["compact"]
    assert g2.abs().max().item() > 0 and o2.abs().max().item() > 0
    assert torch.equal(g, g2) and torch.equal(o, o2)  # deterministic gathers: bit for bit
    for a, b in ((gs, gs2), (gr, gr2)):  # atomic scatters: summation order only
        rel = float(((a - b).abs().pow(2).sum() / b.abs().pow(2).sum()).sqrt())
        assert rel <= 1e-6, rel
