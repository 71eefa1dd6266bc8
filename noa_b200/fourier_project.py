"""Python host API of noa_b200: noa's central-slice functions on CUDA tensors, through the C ABI.

Mirrors noa::xform (noa/xform/FourierProject.hpp): same function names, argument order and meaning
(BDHW logical shapes, rfft physical arrays, remaps "h2h" / "h2hc" / "hc2h" / "hc2hc", option names),
and the same error behaviour (an invalid call raises before anything runs). Arrays are torch CUDA
tensors (complex64 / float32 values, float32 weights); every call is asynchronous on the given CUDA
stream (default: torch's current stream).

There is no CPU fallback: if the CUDA library is missing, importing the functions raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libnoa_b200.so")

NB_OK = 0
NB_ERROR_INVALID = -1
NB_ERROR_UNSUPPORTED = -2
NB_ERROR_CUDA = -3
NB_ERROR_OOM = -4
NB_ERROR_TIMEOUT = -5  # reserved (no kernel waits on the device)

REMAPS = {"h2h": 0, "h2hc": 8, "hc2h": 4, "hc2hc": 12}
INTERPS = {"nearest": 0, "linear": 1, "cubic": 2, "cubic_bspline": 3, "lanczos4": 4, "lanczos6": 5,
           "lanczos8": 6, "nearest_fast": 100, "linear_fast": 101, "cubic_fast": 102,
           "cubic_bspline_fast": 103, "lanczos4_fast": 104, "lanczos6_fast": 105, "lanczos8_fast": 106}
DTYPE_F32, DTYPE_C32, DTYPE_F64, DTYPE_C64 = 1, 2, 3, 4
XFORM_NONE, XFORM_MAT22, XFORM_MAT33, XFORM_QUAT = 0, 1, 2, 3


class NbArray(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int32), ("is_value", C.c_int32),
                ("shape", C.c_int64 * 4), ("strides", C.c_int64 * 4), ("value", C.c_double * 2)]


class NbTransform(C.Structure):
    _fields_ = [("data", C.c_void_p), ("kind", C.c_int32), ("count", C.c_int64), ("value", C.c_double * 9)]


class NbOptions(C.Structure):
    _fields_ = [("interp", C.c_int32), ("fftfreq_cutoff", C.c_double), ("target_shape", C.c_int64 * 4),
                ("ews_radius", C.c_double * 2), ("fftfreq_sinc", C.c_double),
                ("fftfreq_blackman", C.c_double), ("w_fftfreq_sinc", C.c_double),
                ("w_fftfreq_blackman", C.c_double), ("add_to_output", C.c_int32),
                ("correct_weights", C.c_int32)]


class NoaB200Error(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


_lib_handle = None


def lib() -> C.CDLL:
    """The loaded CUDA library. Raises if it was not built (python -m noa_b200.build)."""
    global _lib_handle
    if _lib_handle is None:
        if not os.path.exists(_LIB_PATH):
            raise NoaB200Error(NB_ERROR_CUDA, f"{_LIB_PATH} is missing: build it with `python -m noa_b200.build`")
        h = C.CDLL(_LIB_PATH)
        P = C.POINTER
        arr, xf, opt = P(NbArray), P(NbTransform), P(NbOptions)
        shape = P(C.c_int64)
        h.nb_rasterize_central_slices_3d.argtypes = [C.c_int32, arr, arr, shape, arr, arr, shape, xf, xf, opt, C.c_void_p]
        h.nb_rasterize_central_slices_3d_static_scratch.argtypes = [C.c_int32, arr, arr, shape, arr, arr, shape, xf, xf,
                                                                   opt, C.c_void_p]
        h.nb_insert_central_slices_3d.argtypes = [C.c_int32, arr, arr, shape, arr, arr, shape, xf, xf, opt, C.c_void_p]
        h.nb_insert_central_slices_3d_scatter.argtypes = [C.c_int32, arr, arr, shape, arr, arr, shape, xf, xf, opt,
                                                          C.c_void_p]
        h.nb_extract_central_slices_3d.argtypes = [C.c_int32, arr, arr, shape, arr, arr, shape, xf, xf, opt, C.c_void_p]
        h.nb_insert_and_extract_central_slices_3d.argtypes = [C.c_int32, arr, arr, shape, arr, arr, shape,
                                                               xf, xf, xf, xf, opt, C.c_void_p]
        for f in ("nb_rasterize_central_slices_3d", "nb_rasterize_central_slices_3d_static_scratch",
                  "nb_insert_central_slices_3d", "nb_insert_central_slices_3d_scatter",
                  "nb_extract_central_slices_3d", "nb_insert_and_extract_central_slices_3d"):
            getattr(h, f).restype = C.c_int
        h.nb_fourier_interpolation_correction.argtypes = [arr, arr, C.c_int32, C.c_int32, C.c_void_p]
        h.nb_fourier_interpolation_correction.restype = C.c_int
        h.nb_last_error.restype = C.c_char_p
        h.nb_version.restype = C.c_char_p
        h.nb_options_default.argtypes = [opt]
        h.nb_set_scratch_limit.argtypes = [C.c_int32, C.c_int64]
        h.nb_set_scratch_limit.restype = C.c_int
        h.nb_scratch_refusals.argtypes = [C.c_int32]
        h.nb_scratch_refusals.restype = C.c_int64
        h.nb_scratch_limit.argtypes = [C.c_int32]
        h.nb_scratch_limit.restype = C.c_int64
        _lib_handle = h
    return _lib_handle


def library_path() -> str:
    return _LIB_PATH


# ---------------------------------------------------------------------------------------------------
# Argument marshalling.
# ---------------------------------------------------------------------------------------------------
def _torch():
    import torch
    return torch


_DTYPES: dict = {}


def _dtype_code(t) -> int:
    if not _DTYPES:
        torch = _torch()
        _DTYPES.update({torch.float32: DTYPE_F32, torch.complex64: DTYPE_C32,
                        torch.float64: DTYPE_F64, torch.complex128: DTYPE_C64})
    return _DTYPES[t.dtype]


def as_nb_array(t, keep: list) -> NbArray | None:
    """A torch tensor (4-D, physical rfft shape), a Python scalar (constant input) or None."""
    if t is None:
        return None
    a = NbArray()
    if isinstance(t, (int, float, complex)):
        a.is_value = 1
        a.dtype = DTYPE_C32 if isinstance(t, complex) else DTYPE_F32
        a.value[0] = float(np.real(t))
        a.value[1] = float(np.imag(t))
        return a
    shape = t.shape
    if len(shape) != 4:
        raise NoaB200Error(NB_ERROR_INVALID, f"expected a 4-D (BDHW) tensor, got shape {tuple(shape)}")
    a.data = t.data_ptr()
    a.dtype = _dtype_code(t)
    a.shape[:] = shape
    a.strides[:] = t.stride()
    keep.append(t)
    return a


def pack_rotations(m):
    """Matrices (n,3,3) -> noa's Mat33<f32> layout (n,12) (rows padded to the type's 48-byte size)."""
    torch = _torch()
    if isinstance(m, np.ndarray):
        m = torch.from_numpy(np.ascontiguousarray(m))
    m = m.to(torch.float32)
    p = torch.zeros((m.shape[0], 12), dtype=torch.float32, device=m.device)
    p[:, :9] = m.reshape(m.shape[0], 9)
    return p


def as_nb_transform(x, rotation: bool, keep: list) -> NbTransform | None:
    """None (Empty), a single matrix/quaternion (numpy/tuple, passed inline), or a CUDA tensor:
    (n,12) packed Mat33, (n,3,3) Mat33 (packed here), (n,4) quaternions z,y,x,w, (n,2,2) Mat22."""
    t = NbTransform()
    if x is None:
        if rotation:
            raise NoaB200Error(NB_ERROR_INVALID, "rotation should not be empty")
        t.kind = XFORM_NONE
        return t
    torch = _torch()
    if not isinstance(x, torch.Tensor):
        v = np.asarray(x, dtype=np.float64)
        if v.shape == (3, 3):
            t.kind = XFORM_MAT33
        elif v.shape == (4,):
            t.kind = XFORM_QUAT
        elif v.shape == (2, 2):
            t.kind = XFORM_MAT22
        else:
            raise NoaB200Error(NB_ERROR_INVALID, f"unexpected transform shape {v.shape}")
        t.count = 1
        for i, e in enumerate(v.ravel()):
            t.value[i] = float(e)
        return t
    if x.dim() == 3 and tuple(x.shape[1:]) == (3, 3):
        x = pack_rotations(x)
    x = x.contiguous()
    if x.dim() == 2 and x.shape[1] == 12:
        t.kind = XFORM_MAT33
    elif x.dim() == 2 and x.shape[1] == 4:
        t.kind = XFORM_QUAT
    elif x.dim() == 3 and tuple(x.shape[1:]) == (2, 2):
        t.kind = XFORM_MAT22
    else:
        raise NoaB200Error(NB_ERROR_INVALID, f"unexpected transform tensor shape {tuple(x.shape)}")
    if x.dtype != torch.float32:
        raise NoaB200Error(NB_ERROR_UNSUPPORTED, "transforms should be float32")
    t.data = x.data_ptr()
    t.count = x.shape[0]
    keep.append(x)
    return t


@dataclass
class WindowedSinc:
    """noa::xform::WindowedSinc (FourierProject.hpp:1703-1718)."""
    fftfreq_sinc: float = -1.0
    fftfreq_blackman: float = -1.0


_DEFAULT_OPTIONS: list = []
_NO_WINDOW = WindowedSinc()


def _default_options() -> NbOptions:
    """The library's default options (nb_options_default), fetched once."""
    if not _DEFAULT_OPTIONS:
        o = NbOptions()
        lib().nb_options_default(C.byref(o))
        _DEFAULT_OPTIONS.append(o)
    return _DEFAULT_OPTIONS[0]


def _options(interp="linear", fftfreq_cutoff=0.5, target_shape=None, ews_radius=(0.0, 0.0),
             windowed_sinc: WindowedSinc | None = None, w_windowed_sinc: WindowedSinc | None = None,
             add_to_output=False, correct_weights=False) -> NbOptions:
    o = NbOptions.from_buffer_copy(_default_options())
    o.interp = INTERPS[interp] if isinstance(interp, str) else int(interp)
    o.fftfreq_cutoff = float(fftfreq_cutoff)
    if target_shape is not None:
        for i in range(4):
            o.target_shape[i] = int(target_shape[i])
    if isinstance(ews_radius, (int, float)) or np.isscalar(ews_radius):
        ews_radius = (ews_radius, ews_radius)
    o.ews_radius[0], o.ews_radius[1] = float(ews_radius[0]), float(ews_radius[1])
    ws = windowed_sinc or _NO_WINDOW
    wws = w_windowed_sinc or _NO_WINDOW
    o.fftfreq_sinc, o.fftfreq_blackman = float(ws.fftfreq_sinc), float(ws.fftfreq_blackman)
    o.w_fftfreq_sinc, o.w_fftfreq_blackman = float(wws.fftfreq_sinc), float(wws.fftfreq_blackman)
    o.add_to_output = int(bool(add_to_output))
    o.correct_weights = int(bool(correct_weights))
    return o


def _stream_ptr(stream) -> int | None:
    torch = _torch()
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _check(code: int) -> None:
    if code != NB_OK:
        raise NoaB200Error(code, lib().nb_last_error().decode(errors="replace"))


_I64x4 = C.c_int64 * 4


def _shape(s) -> C.Array:
    return _I64x4(*map(int, s))


def _ref(x):
    return C.byref(x) if x is not None else None


# ---------------------------------------------------------------------------------------------------
# noa::xform API.
# ---------------------------------------------------------------------------------------------------
def rasterize_central_slices_3d(remap: str, slice, slice_weight, slice_shape, volume, volume_weight,
                                volume_shape, inv_scaling, fwd_rotation, *, fftfreq_cutoff=0.5,
                                target_shape=None, ews_radius=(0.0, 0.0), stream=None) -> None:
    """noa::xform::rasterize_central_slices_3d (FourierProject.hpp:1653-1692): trilinear insertion (+=)."""
    keep = []
    o = _options(fftfreq_cutoff=fftfreq_cutoff, target_shape=target_shape, ews_radius=ews_radius)
    _check(lib().nb_rasterize_central_slices_3d(
        REMAPS[remap], _ref(as_nb_array(slice, keep)), _ref(as_nb_array(slice_weight, keep)), _shape(slice_shape),
        _ref(as_nb_array(volume, keep)), _ref(as_nb_array(volume_weight, keep)), _shape(volume_shape),
        _ref(as_nb_transform(inv_scaling, False, keep)), _ref(as_nb_transform(fwd_rotation, True, keep)),
        C.byref(o), _stream_ptr(stream)))


def rasterize_central_slices_3d_static_scratch(remap: str, slice, slice_weight, slice_shape, volume, volume_weight,
                                               volume_shape, inv_scaling, fwd_rotation, *, fftfreq_cutoff=0.5,
                                               target_shape=None, ews_radius=(0.0, 0.0), stream=None) -> None:
    """rasterize_central_slices_3d without any device allocation (no counterpart in the reference).

    For callers that cannot let the library allocate device memory at call time. The accumulator is a
    64 MiB array reserved per GPU when the library loads: with weights, volumes up to 4,194,304 rfft
    voxels (complex) are accepted, larger ones raise. Calls share that array, so calls that overlap on
    the GPU must be ordered; the first call on a device should come before any stream capture."""
    keep = []
    o = _options(fftfreq_cutoff=fftfreq_cutoff, target_shape=target_shape, ews_radius=ews_radius)
    _check(lib().nb_rasterize_central_slices_3d_static_scratch(
        REMAPS[remap], _ref(as_nb_array(slice, keep)), _ref(as_nb_array(slice_weight, keep)), _shape(slice_shape),
        _ref(as_nb_array(volume, keep)), _ref(as_nb_array(volume_weight, keep)), _shape(volume_shape),
        _ref(as_nb_transform(inv_scaling, False, keep)), _ref(as_nb_transform(fwd_rotation, True, keep)),
        C.byref(o), _stream_ptr(stream)))


def insert_central_slices_3d(remap: str, slice, slice_weight, slice_shape, volume, volume_weight, volume_shape,
                             fwd_scaling, inv_rotation, *, interp="linear", windowed_sinc=None,
                             fftfreq_cutoff=0.5, target_shape=None, ews_radius=(0.0, 0.0), stream=None) -> None:
    """noa::xform::insert_central_slices_3d (FourierProject.hpp:1770-1815): windowed-sinc gather (+=)."""
    keep = []
    o = _options(interp=interp, fftfreq_cutoff=fftfreq_cutoff, target_shape=target_shape,
                 ews_radius=ews_radius, windowed_sinc=windowed_sinc)
    _check(lib().nb_insert_central_slices_3d(
        REMAPS[remap], _ref(as_nb_array(slice, keep)), _ref(as_nb_array(slice_weight, keep)), _shape(slice_shape),
        _ref(as_nb_array(volume, keep)), _ref(as_nb_array(volume_weight, keep)), _shape(volume_shape),
        _ref(as_nb_transform(fwd_scaling, False, keep)), _ref(as_nb_transform(inv_rotation, True, keep)),
        C.byref(o), _stream_ptr(stream)))


def insert_central_slices_3d_scatter(remap: str, slice, slice_weight, slice_shape, volume, volume_weight,
                                     volume_shape, fwd_scaling, inv_rotation, *, interp="linear",
                                     windowed_sinc=None, fftfreq_cutoff=0.5, target_shape=None,
                                     ews_radius=(0.0, 0.0), stream=None) -> None:
    """Slice-major atomic scatter form of ``insert_central_slices_3d``: the same terms, summed over the
    slices in an unspecified order (no counterpart in the reference; see fourier_project.h)."""
    keep = []
    o = _options(interp=interp, fftfreq_cutoff=fftfreq_cutoff, target_shape=target_shape,
                 ews_radius=ews_radius, windowed_sinc=windowed_sinc)
    _check(lib().nb_insert_central_slices_3d_scatter(
        REMAPS[remap], _ref(as_nb_array(slice, keep)), _ref(as_nb_array(slice_weight, keep)), _shape(slice_shape),
        _ref(as_nb_array(volume, keep)), _ref(as_nb_array(volume_weight, keep)), _shape(volume_shape),
        _ref(as_nb_transform(fwd_scaling, False, keep)), _ref(as_nb_transform(inv_rotation, True, keep)),
        C.byref(o), _stream_ptr(stream)))


def fourier_interpolation_correction(input, output, interp="linear", post_correction=True, *, stream=None) -> None:
    """noa::xform::fourier_interpolation_correction (FourierProject.hpp:2062-2087): divides (post) or
    multiplies (pre) the real-space ``input`` by sinc^2(pi r) into ``output`` (4-D float32 CUDA tensors,
    ``input`` broadcastable or a float; in place allowed). LINEAR only, as in the reference."""
    keep = []
    _check(lib().nb_fourier_interpolation_correction(
        _ref(as_nb_array(input, keep)), _ref(as_nb_array(output, keep)),
        INTERPS[interp] if isinstance(interp, str) else int(interp), int(bool(post_correction)),
        _stream_ptr(stream)))


def extract_central_slices_3d(remap: str, volume, volume_weight, volume_shape, slice, slice_weight, slice_shape,
                              inv_scaling, fwd_rotation, *, interp="linear", w_windowed_sinc=None,
                              fftfreq_cutoff=0.5, target_shape=None, ews_radius=(0.0, 0.0), stream=None) -> None:
    """noa::xform::extract_central_slices_3d (FourierProject.hpp:1869-1914)."""
    keep = []
    o = _options(interp=interp, fftfreq_cutoff=fftfreq_cutoff, target_shape=target_shape,
                 ews_radius=ews_radius, w_windowed_sinc=w_windowed_sinc)
    _check(lib().nb_extract_central_slices_3d(
        REMAPS[remap], _ref(as_nb_array(volume, keep)), _ref(as_nb_array(volume_weight, keep)), _shape(volume_shape),
        _ref(as_nb_array(slice, keep)), _ref(as_nb_array(slice_weight, keep)), _shape(slice_shape),
        _ref(as_nb_transform(inv_scaling, False, keep)), _ref(as_nb_transform(fwd_rotation, True, keep)),
        C.byref(o), _stream_ptr(stream)))


def insert_and_extract_central_slices_3d(remap: str, input_slice, input_weight, input_slice_shape, output_slice,
                                         output_weight, output_slice_shape, input_fwd_scaling, input_inv_rotation,
                                         output_inv_scaling, output_fwd_rotation, *, interp="linear",
                                         input_windowed_sinc=None, w_windowed_sinc=None, add_to_output=False,
                                         correct_weights=False, fftfreq_cutoff=0.5, ews_radius=(0.0, 0.0),
                                         stream=None) -> None:
    """noa::xform::insert_and_extract_central_slices_3d (FourierProject.hpp:1987-2049)."""
    keep = []
    o = _options(interp=interp, fftfreq_cutoff=fftfreq_cutoff, ews_radius=ews_radius,
                 windowed_sinc=input_windowed_sinc, w_windowed_sinc=w_windowed_sinc,
                 add_to_output=add_to_output, correct_weights=correct_weights)
    _check(lib().nb_insert_and_extract_central_slices_3d(
        REMAPS[remap], _ref(as_nb_array(input_slice, keep)), _ref(as_nb_array(input_weight, keep)),
        _shape(input_slice_shape),
        _ref(as_nb_array(output_slice, keep)), _ref(as_nb_array(output_weight, keep)), _shape(output_slice_shape),
        _ref(as_nb_transform(input_fwd_scaling, False, keep)), _ref(as_nb_transform(input_inv_rotation, True, keep)),
        _ref(as_nb_transform(output_inv_scaling, False, keep)), _ref(as_nb_transform(output_fwd_rotation, True, keep)),
        C.byref(o), _stream_ptr(stream)))


def version() -> str:
    return lib().nb_version().decode()


def _device_index(device) -> int:
    if device is None:
        return _torch().cuda.current_device()
    if isinstance(device, int):
        return device
    d = _torch().device(device)
    return d.index if d.index is not None else _torch().cuda.current_device()


def set_scratch_limit(nbytes: int | None, device=None) -> None:
    """Caps the size of any one device allocation the library makes on its own on ``device`` (default:
    the current CUDA device): the fast paths' scratch (pair copies, padded accumulators) and batch
    buffers. Calls then take their paths without that memory, with the same results; batched launches
    that cannot allocate their descriptors raise NB_ERROR_OOM. ``None`` removes the cap."""
    _check(lib().nb_set_scratch_limit(_device_index(device), -1 if nbytes is None else int(nbytes)))


def scratch_limit(device=None) -> int | None:
    """The cap set with ``set_scratch_limit`` (None when there is none)."""
    v = int(lib().nb_scratch_limit(_device_index(device)))
    return None if v < 0 else v


def scratch_refusals(device=None) -> int:
    """How many of the library's own allocations on ``device`` were refused since it loaded (above the
    cap or out of memory), each sending a call down its path without that memory."""
    return int(lib().nb_scratch_refusals(_device_index(device)))
