"""Argument errors of the entry points beyond the four drop-in functions (GPU, no kernel runs on bad
arguments): each returns NB_ERROR_INVALID / NB_ERROR_UNSUPPORTED with a message, like the per-call ABI."""
import ctypes as C

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from noa_b200 import batch  # noqa: E402
from noa_b200 import fourier_project as fp  # noqa: E402
from noa_b200 import reconstruct  # noqa: E402


def _code(fn, *a, **k):
    with pytest.raises(fp.NoaB200Error) as e:
        fn(*a, **k)
    assert str(e.value)
    return e.value.code


def test_volume_pairs_errors():
    n = 16
    vol = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    real = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.float32, device="cuda")
    assert _code(batch.volume_pairs, real, (1, n, n, n)) == fp.NB_ERROR_INVALID
    assert _code(batch.volume_pairs, vol, (1, n, n, 2 * n)) == fp.NB_ERROR_INVALID       # shape mismatch
    lib = fp.lib()
    batch._setup(lib)
    keep = []
    arr = fp.as_nb_array(vol, keep)
    small = torch.empty(16, dtype=torch.uint8, device="cuda")
    code = lib.nb_volume_pairs(C.byref(arr), fp._shape((1, n, n, n)), small.data_ptr(), 16,
                               fp._stream_ptr(None))
    assert code == fp.NB_ERROR_INVALID
    stacked = torch.zeros((2, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    assert _code(batch.volume_pairs, stacked, (2, n, n, n)) == fp.NB_ERROR_INVALID


def test_batch_launch_errors():
    n, k = 16, 3
    vol = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    rot = fp.pack_rotations(torch.eye(3).repeat(k, 1, 1).cuda())
    out_c = torch.empty((k, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    out_r = torch.empty((k, 1, n, n // 2 + 1), dtype=torch.float32, device="cuda")
    mk = lambda o: batch.ExtractRequest(volume=vol, volume_shape=(1, n, n, n), slice=o, slice_shape=(k, 1, n, n),
                                        fwd_rotation=rot)
    # value types must agree across the batch
    assert _code(batch.extract_batch_launch, "hc2h", [mk(out_c), mk(out_r)]) == fp.NB_ERROR_INVALID
    # a pair copy too small for its volume
    tiny = torch.empty(64, dtype=torch.uint8, device="cuda")
    assert _code(batch.extract_batch_launch, "hc2h", [mk(out_c)], [tiny]) == fp.NB_ERROR_INVALID
    # per-request checks of the drop-in (wrong slice shape)
    bad = batch.ExtractRequest(volume=vol, volume_shape=(1, n, n, n), slice=out_c, slice_shape=(k, 1, n, 2 * n),
                               fwd_rotation=rot)
    assert _code(batch.extract_batch_launch, "hc2h", [bad]) == fp.NB_ERROR_INVALID


def test_scatter_insert_rejects_what_the_gather_form_rejects():
    n, k = 16, 2
    sl = torch.zeros((k, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grid = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    rot = torch.eye(3).repeat(k, 1, 1).cuda()
    for fn in (fp.insert_central_slices_3d, fp.insert_central_slices_3d_scatter):
        assert _code(fn, "hc2hc", sl, None, (k, 1, n, n), grid, None, (1, n, n, 2 * n), None, rot) == \
            fp.NB_ERROR_INVALID
        f64 = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex128, device="cuda")
        assert _code(fn, "hc2hc", sl, None, (k, 1, n, n), f64, None, (1, n, n, n), None, rot) == \
            fp.NB_ERROR_UNSUPPORTED


def test_gridding_and_spectrum_errors():
    n = 8
    x = torch.zeros((1, n, n, n), dtype=torch.float32, device="cuda")
    assert _code(fp.fourier_interpolation_correction, x, torch.zeros((1, n, n, n + 1), device="cuda")) == \
        fp.NB_ERROR_INVALID                                                   # cannot broadcast
    assert _code(fp.fourier_interpolation_correction, x.double(), x) == fp.NB_ERROR_UNSUPPORTED
    v = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    w = torch.ones((1, n, n, n // 2 + 1), dtype=torch.float32, device="cuda")
    out = torch.empty_like(v)
    assert _code(reconstruct.reconstruction_spectrum, v, w, (1, n, n, n), v) == fp.NB_ERROR_INVALID   # overlap
    strided = torch.empty((1, n, n, n + 2), dtype=torch.complex64, device="cuda")[..., : n // 2 + 1]
    assert _code(reconstruct.reconstruction_spectrum, v, w, (1, n, n, n), strided) == fp.NB_ERROR_INVALID
    assert _code(reconstruct.reconstruction_spectrum, v, v, (1, n, n, n), out) == fp.NB_ERROR_INVALID  # c32 weights
    reconstruct.reconstruction_spectrum(v, None, (1, n, n, n), out)           # no weights: fine
    torch.cuda.synchronize()
