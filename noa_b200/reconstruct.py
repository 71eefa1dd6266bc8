"""The reconstruction steps after insertion: spectrum normalization + remap + centering (one pass),
the c2r inverse FFT, and the LINEAR gridding correction (one pass, in place).

    volume = reconstruct(values, weights, (1, n, n, n))

``values`` / ``weights``: the inserted rfft grids, (1, D, H, W/2+1) complex64 / float32 CUDA tensors,
centered ("hc", what rasterize/insert with remap ``*2hc`` produce) unless ``centered=False``. Returns the
real-space volume (1, D, H, W) float32 with its origin at (D/2, H/2, W/2), divided by sinc^2 of the
trilinear gridding kernel (noa::xform::fourier_interpolation_correction). The inverse FFT is cuFFT
(through torch.fft) with the "backward" normalization (1 / (D H W)).
"""
from __future__ import annotations

import ctypes as C

from . import fourier_project as fp


def _setup(lib):
    if getattr(lib, "_nb_reconstruct_ready", False):
        return
    lib.nb_reconstruction_spectrum.argtypes = [C.POINTER(fp.NbArray), C.POINTER(fp.NbArray), C.POINTER(C.c_int64),
                                               C.c_int32, C.c_double, C.POINTER(fp.NbArray), C.c_void_p]
    lib.nb_reconstruction_spectrum.restype = C.c_int
    lib._nb_reconstruct_ready = True


def reconstruction_spectrum(values, weights, volume_shape, output, *, centered=True, weight_threshold=1.0,
                            stream=None) -> None:
    """nb_reconstruction_spectrum: output = values / max(weights, threshold), non-centered, phase-shifted
    so that the c2r puts the origin at the center."""
    lib = fp.lib()
    _setup(lib)
    keep = []
    fp._check(lib.nb_reconstruction_spectrum(
        fp._ref(fp.as_nb_array(values, keep)), fp._ref(fp.as_nb_array(weights, keep)), fp._shape(volume_shape),
        int(bool(centered)), float(weight_threshold), fp._ref(fp.as_nb_array(output, keep)),
        fp._stream_ptr(stream)))


def reconstruct(values, weights, volume_shape, *, centered=True, weight_threshold=1.0, correct=True,
                stream=None):
    torch = fp._torch()
    _, d, h, w = (int(x) for x in volume_shape)
    s = stream or torch.cuda.current_stream()
    with torch.cuda.stream(s):
        spec = torch.empty((1, d, h, w // 2 + 1), dtype=torch.complex64, device=values.device)
        reconstruction_spectrum(values, weights, volume_shape, spec, centered=centered,
                                weight_threshold=weight_threshold, stream=s)
        real = torch.fft.irfftn(spec[0], s=(d, h, w), norm="backward")[None].contiguous()
        if correct:
            fp.fourier_interpolation_correction(real, real, "linear", True, stream=s)
    return real
