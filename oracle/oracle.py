"""ORACLE TEST INFRASTRUCTURE — parity checkers for the CUDA path; never the product.

Two CPU implementations of noa's Fourier central-slice path, both callable on numpy arrays:

* ``fp``  — oracle/libfp_oracle.so, the plain-C restatement in oracle/fp_oracle_impl.h (f32 and the
  FP64 oracle). Always buildable (``make -C oracle fp``).
* ``ref`` — oracle/_ref/libnoa_ref.so, the reference's own CPU (OpenMP) path compiled from its sources
  (``make -C oracle ref``). Present only where it was built.
* ``ref_cuda`` — oracle/_ref/libnoa_ref_cuda.so (``make -C oracle ref-cuda``): noa's CUDA backend and the
  reference-side binding, to pass a noa GPU Texture through the binding (GPU tests only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FP_LIB = os.path.join(HERE, "libfp_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libnoa_ref.so")

REMAPS = {"h2h": 0, "h2hc": 8, "hc2h": 4, "hc2hc": 12}
INTERPS = {"nearest": 0, "linear": 1, "cubic": 2, "cubic_bspline": 3,
           "lanczos4": 4, "lanczos6": 5, "lanczos8": 6}
FUNCS = ("rasterize", "insert", "extract", "insert_extract")


class FpoArray(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int32), ("is_value", C.c_int32),
                ("shape", C.c_int64 * 4), ("strides", C.c_int64 * 4), ("value", C.c_double * 2)]


class FpoTransform(C.Structure):
    _fields_ = [("data", C.c_void_p), ("kind", C.c_int32), ("count", C.c_int64),
                ("value", C.c_double * 9)]


class FpoOptions(C.Structure):
    _fields_ = [("interp", C.c_int32), ("fftfreq_cutoff", C.c_double), ("target_shape", C.c_int64 * 4),
                ("ews_radius", C.c_double * 2), ("fftfreq_sinc", C.c_double),
                ("fftfreq_blackman", C.c_double), ("w_fftfreq_sinc", C.c_double),
                ("w_fftfreq_blackman", C.c_double), ("add_to_output", C.c_int32),
                ("correct_weights", C.c_int32)]


class RefArray(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("shape", C.c_int64 * 4), ("strides", C.c_int64 * 4)]


class RefOptions(C.Structure):
    _fields_ = [("remap", C.c_int32), ("interp", C.c_int32), ("fftfreq_cutoff", C.c_double),
                ("target_shape", C.c_int64 * 4), ("ews_radius", C.c_double * 2),
                ("sinc", C.c_double * 2), ("w_sinc", C.c_double * 2),
                ("add_to_output", C.c_int32), ("correct_weights", C.c_int32)]


@dataclass
class Call:
    """One call of a Fourier-projection function on host numpy arrays (BDHW, rfft physical shapes).

    ``inp``/``out`` hold values (complex64/float32, or complex128/float64 for the FP64 oracle);
    weights are real arrays or None. ``scale``/``rot`` are per-slice arrays, shape (n,2,2) and (n,3,3)
    for matrices or (n,4) z,y,x,w for quaternions. For insert_extract, ``scale2``/``rot2`` are the
    output transforms. ``inp_value`` replaces ``inp`` by a constant (rasterize/insert_extract)."""
    func: str
    remap: str
    inp: np.ndarray | None
    in_shape: tuple
    out: np.ndarray
    out_shape: tuple
    rot: np.ndarray
    inp_w: np.ndarray | None = None
    out_w: np.ndarray | None = None
    scale: np.ndarray | None = None
    rot2: np.ndarray | None = None
    scale2: np.ndarray | None = None
    interp: int = 1
    cutoff: float = 0.5
    target: tuple = (0, 0, 0, 0)
    ews: tuple = (0.0, 0.0)
    sinc: tuple = (-1.0, -1.0)
    w_sinc: tuple = (-1.0, -1.0)
    add_to_output: bool = False
    correct_weights: bool = False
    inp_value: complex | float | None = None
    inp_value_shape: tuple | None = None
    keep: list = field(default_factory=list)


def _is_f64(a: np.ndarray) -> bool:
    return a.dtype in (np.float64, np.complex128)


def _fpo_array(a, keep, value=None, value_shape=None, complex_value=True):
    s = FpoArray()
    if value is not None:
        s.is_value = 1
        s.dtype = 2 if complex_value else 1
        s.value[0] = float(np.real(value))
        s.value[1] = float(np.imag(value))
        for i in range(4):
            s.shape[i] = value_shape[i]
            s.strides[i] = 0
        return s
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"] or True
    s.data = a.ctypes.data
    s.dtype = 2 if np.iscomplexobj(a) else 1
    for i in range(4):
        s.shape[i] = a.shape[i]
        s.strides[i] = a.strides[i] // a.itemsize
    keep.append(a)
    return s


def pack_transforms(a: np.ndarray) -> np.ndarray:
    """Per-slice transforms in noa's memory layout: Mat22 (n,2,2) and quaternions (n,4) are dense;
    Mat33 (n,3,3) rows are padded to the type's 16-byte alignment (12 floats or 10 doubles each)."""
    a = np.ascontiguousarray(a)
    if a.ndim == 3 and a.shape[1:] == (3, 3):
        stride = 12 if a.dtype == np.float32 else 10
        p = np.zeros((a.shape[0], stride), dtype=a.dtype)
        p[:, :9] = a.reshape(a.shape[0], 9)
        return p
    return a


def _fpo_transform(a, kind_hint, keep):
    t = FpoTransform()
    if a is None:
        t.kind = 0
        return t
    if a.ndim == 3 and a.shape[1:] == (2, 2):
        t.kind = 1
    elif a.ndim == 3 and a.shape[1:] == (3, 3):
        t.kind = 2
    else:
        assert a.ndim == 2 and a.shape[1] == 4
        t.kind = 3
    t.count = a.shape[0]
    p = pack_transforms(a)
    keep.append(p)
    t.data = p.ctypes.data
    return t


def _options(c: Call) -> FpoOptions:
    o = FpoOptions()
    o.interp = c.interp
    o.fftfreq_cutoff = c.cutoff
    for i in range(4):
        o.target_shape[i] = c.target[i]
    o.ews_radius[0], o.ews_radius[1] = c.ews
    o.fftfreq_sinc, o.fftfreq_blackman = c.sinc
    o.w_fftfreq_sinc, o.w_fftfreq_blackman = c.w_sinc
    o.add_to_output = int(c.add_to_output)
    o.correct_weights = int(c.correct_weights)
    return o


class _Lib:
    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle)")
        self.lib = C.CDLL(path)


class FpOracle(_Lib):
    """The C restatement. ``run(call, threads)`` writes into call.out / call.out_w in place."""

    def __init__(self):
        super().__init__(FP_LIB)

    def run(self, c: Call, threads: int = 1) -> int:
        keep = []
        f64 = _is_f64(c.out)
        fn = getattr(self.lib, f"fpo_{c.func}_{'f64' if f64 else 'f32'}")
        inp = _fpo_array(c.inp, keep, c.inp_value, c.inp_value_shape,
                         complex_value=np.iscomplexobj(c.out) or isinstance(c.inp_value, complex))
        args = [C.c_int32(REMAPS[c.remap]),
                C.byref(inp), C.byref(_fpo_array(c.inp_w, keep)) if c.inp_w is not None else None,
                (C.c_int64 * 4)(*c.in_shape),
                C.byref(_fpo_array(c.out, keep)),
                C.byref(_fpo_array(c.out_w, keep)) if c.out_w is not None else None,
                (C.c_int64 * 4)(*c.out_shape)]
        t = [_fpo_transform(c.scale, 1, keep), _fpo_transform(c.rot, 2, keep),
             _fpo_transform(c.scale2, 1, keep), _fpo_transform(c.rot2, 2, keep)]
        keep.extend(t)
        args += [C.byref(t[0]), C.byref(t[1]), C.byref(t[2]), C.byref(t[3]) if c.rot2 is not None else None]
        opts = _options(c)
        args += [C.byref(opts), C.c_int(threads)]
        return fn(*args)


def gridding_correction(inp, out: np.ndarray, interp: int = 1, post_correction: bool = True,
                        threads: int = 1) -> int:
    """fpo_gridding_correction_{f32,f64} on host arrays (``inp`` an array or a float constant)."""
    lib = FpOracle().lib
    keep = []
    f64 = out.dtype == np.float64
    fn = getattr(lib, f"fpo_gridding_correction_{'f64' if f64 else 'f32'}")
    if isinstance(inp, (int, float)):
        a = _fpo_array(None, keep, value=float(inp), value_shape=out.shape, complex_value=False)
    else:
        a = _fpo_array(inp, keep)
    o = _fpo_array(out, keep)
    return fn(C.byref(a), C.byref(o), C.c_int32(interp), C.c_int32(int(post_correction)), C.c_int(threads))


COMBOS = {("c32", "c32"): 0, ("f32", "f32"): 1, ("c32", "f32"): 2, ("c64", "c64"): 3, ("f64", "f64"): 4}
_DT = {np.dtype(np.complex64): "c32", np.dtype(np.float32): "f32",
       np.dtype(np.complex128): "c64", np.dtype(np.float64): "f64"}


class RefLib(_Lib):
    """noa's own CPU path (oracle/_ref). Same Call description; constant inputs are not supported."""

    def __init__(self):
        super().__init__(REF_LIB)

    def available_combo(self, c: Call) -> bool:
        return (_DT[c.inp.dtype], _DT[c.out.dtype]) in COMBOS

    def run(self, c: Call, threads: int = 1) -> tuple[int, str]:
        combo = COMBOS[(_DT[c.inp.dtype], _DT[c.out.dtype])]
        suffix = ["c32c32", "f32f32", "c32f32", "c64c64", "f64f64"][combo]
        fn = getattr(self.lib, f"noaref_{c.func}_{suffix}")
        keep = []

        def arr(a):
            if a is None:
                return None
            s = RefArray()
            s.ptr = a.ctypes.data
            for i in range(4):
                s.shape[i] = a.shape[i]
                s.strides[i] = a.strides[i] // a.itemsize
            keep.append(s)
            return C.byref(s)

        def tr(a):
            if a is None:
                return None
            p = pack_transforms(a)
            keep.append(p)
            return C.c_void_p(p.ctypes.data)

        rot_kind = 1 if c.rot.ndim == 2 else 0
        o = RefOptions()
        o.remap = REMAPS[c.remap]
        o.interp = c.interp
        o.fftfreq_cutoff = c.cutoff
        for i in range(4):
            o.target_shape[i] = c.target[i]
        o.ews_radius[0], o.ews_radius[1] = c.ews
        o.sinc[0], o.sinc[1] = c.sinc
        o.w_sinc[0], o.w_sinc[1] = c.w_sinc
        o.add_to_output = int(c.add_to_output)
        o.correct_weights = int(c.correct_weights)
        err = C.create_string_buffer(512)
        status = fn(arr(c.inp), arr(c.inp_w), (C.c_int64 * 4)(*c.in_shape),
                    arr(c.out), arr(c.out_w), (C.c_int64 * 4)(*c.out_shape),
                    tr(c.scale), tr(c.rot), tr(c.scale2), tr(c.rot2), C.c_int(rot_kind),
                    C.byref(o), C.c_int(threads), err, C.c_int(512))
        return status, err.value.decode(errors="replace")


def ref_gridding_correction(inp: np.ndarray, out: np.ndarray, post_correction: bool = True,
                            threads: int = 1) -> tuple[int, str]:
    """The reference's own fourier_interpolation_correction (oracle/_ref, built with the one-expression
    patch described in oracle/ref_gridding.cpp) on host arrays of the same precision."""
    lib = RefLib().lib
    fn = getattr(lib, f"noaref_gridding_correction_{'f64' if out.dtype == np.float64 else 'f32'}")
    keep = []

    def arr(a):
        r = RefArray()
        r.ptr = a.ctypes.data
        for i in range(4):
            r.shape[i] = a.shape[i]
            r.strides[i] = a.strides[i] // a.itemsize
        keep.append(a)
        return r

    a_in, a_out = arr(inp), arr(out)
    err = C.create_string_buffer(512)
    status = fn(C.byref(a_in), C.byref(a_out), C.c_int32(int(post_correction)), C.c_int(threads), err, C.c_int(512))
    return status, err.value.decode(errors="replace")


REF_CUDA_LIB = os.path.join(HERE, "_ref", "libnoa_ref_cuda.so")


def ref_texture_extract(volume: np.ndarray, rotations: np.ndarray, interp: int = 1) -> tuple:
    """Through noa's own CUDA backend (oracle/_ref/libnoa_ref_cuda.so, GPU only): builds a noa
    Texture<c32> of `volume` ((1, n, n, n/2+1) complex64, hc layout) and runs the reference-side binding's
    extract<HC2H> with it and with the plain device array. Returns (from_texture, from_array)."""
    lib = C.CDLL(REF_CUDA_LIB)
    n = volume.shape[1]
    count = rotations.shape[0]
    vol = np.ascontiguousarray(volume, dtype=np.complex64)
    rot = np.ascontiguousarray(pack_transforms(rotations.astype(np.float32)))
    a = np.zeros((count, 1, n, n // 2 + 1), np.complex64)
    b = np.zeros_like(a)
    err = C.create_string_buffer(512)
    status = lib.noaref_texture_extract(C.c_void_p(vol.ctypes.data), C.c_int64(n), C.c_void_p(rot.ctypes.data),
                                        C.c_int64(count), C.c_int32(interp), C.c_void_p(a.ctypes.data),
                                        C.c_void_p(b.ctypes.data), err, C.c_int(512))
    if status != 0:
        raise RuntimeError(err.value.decode(errors="replace"))
    return a, b


def ref_cuda_available() -> bool:
    return os.path.exists(REF_CUDA_LIB)


def fp_available() -> bool:
    return os.path.exists(FP_LIB)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)
