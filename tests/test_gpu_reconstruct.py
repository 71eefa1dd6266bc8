"""Gridding correction and the reconstruction steps on the GPU.

* nb_fourier_interpolation_correction against the oracle (f32; factors differ only through sinf):
  maximum relative error 1e-5.
* reconstruct() (spectrum pass + cuFFT c2r + correction) against a plain PyTorch fp32 chain of the same
  operations (division, ifftshift, irfftn, fftshift, division by sinc^2): relative L2 1e-5.
"""
import numpy as np
import pytest

from oracle.oracle import gridding_correction

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from noa_b200 import fourier_project as fp  # noqa: E402
from noa_b200.reconstruct import reconstruct  # noqa: E402


@pytest.mark.parametrize("shape", [(1, 16, 16, 16), (2, 9, 12, 7), (1, 1, 20, 20), (1, 64, 64, 64)])
@pytest.mark.parametrize("post", [True, False])
def test_gridding_matches_oracle(shape, post):
    rng = np.random.default_rng(sum(shape) + post)
    inp = rng.standard_normal(shape).astype(np.float32)
    ref = np.zeros(shape, dtype=np.float32)
    assert gridding_correction(inp, ref, post_correction=post) == 0
    x = torch.from_numpy(inp).cuda()
    out = torch.empty_like(x)
    fp.fourier_interpolation_correction(x, out, "linear", post)
    fp.fourier_interpolation_correction(x, x, "linear", post)  # in place
    torch.cuda.synchronize()
    for got in (out, x):
        g = got.cpu().numpy()
        assert np.max(np.abs(g - ref) / np.maximum(np.abs(ref), 1e-6)) < 1e-5


def test_gridding_broadcast_constant_and_errors():
    shape = (1, 12, 10, 8)
    out = torch.empty(shape, dtype=torch.float32, device="cuda")
    fp.fourier_interpolation_correction(3.0, out, "linear", True)
    ref = np.zeros(shape, dtype=np.float32)
    assert gridding_correction(3.0, ref, post_correction=True) == 0
    assert np.allclose(out.cpu().numpy(), ref, rtol=1e-5)
    row = torch.randn((1, 1, 1, 8), device="cuda")
    fp.fourier_interpolation_correction(row, out, "linear", False)
    ref2 = np.zeros(shape, dtype=np.float32)
    assert gridding_correction(np.broadcast_to(row.cpu().numpy(), shape).copy(), ref2, post_correction=False) == 0
    assert np.allclose(out.cpu().numpy(), ref2, rtol=1e-5, atol=1e-7)
    with pytest.raises(fp.NoaB200Error) as e:
        fp.fourier_interpolation_correction(out, out, "cubic", True)
    assert e.value.code == fp.NB_ERROR_INVALID


def _torch_reconstruct(values, weights, n, thr, centered):
    spec = values / torch.clamp(weights, min=thr)
    if centered:
        spec = torch.fft.ifftshift(spec, dim=(1, 2))
    real = torch.fft.irfftn(spec[0], s=(n, n, n), norm="backward")
    real = torch.fft.fftshift(real)
    idx = torch.arange(n, device=values.device, dtype=torch.float64)
    d = (idx - n // 2 if n % 2 == 0 else idx - n / 2) / n
    r = torch.sqrt(d[:, None, None] ** 2 + d[None, :, None] ** 2 + d[None, None, :] ** 2)
    x = np.pi * r
    sinc = torch.where(x == 0, torch.ones_like(x), torch.sin(x) / x)
    return (real.to(torch.float64) / sinc ** 2)[None]


@pytest.mark.parametrize("n,centered", [(32, True), (48, False), (64, True)])
def test_reconstruct_matches_torch_chain(n, centered):
    g = torch.Generator(device="cuda")
    g.manual_seed(n)
    wp = n // 2 + 1
    values = torch.complex(torch.randn((1, n, n, wp), generator=g, device="cuda"),
                           torch.randn((1, n, n, wp), generator=g, device="cuda"))
    weights = torch.rand((1, n, n, wp), generator=g, device="cuda") * 3
    got = reconstruct(values, weights, (1, n, n, n), centered=centered, weight_threshold=0.5)
    ref = _torch_reconstruct(values, weights, n, 0.5, centered)
    err = (torch.linalg.vector_norm(got.to(torch.float64) - ref) / torch.linalg.vector_norm(ref)).item()
    assert err <= 1e-5, err
