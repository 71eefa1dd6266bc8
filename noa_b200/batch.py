"""Batched extraction and rasterization (Python side of include/noa_b200/batch.h).

``ExtractBatch`` takes a list of extract_central_slices_3d calls — any mix of volumes, box sizes and
slice counts — and runs them as one CUDA graph: one persistent work-queue kernel, with large LINEAR
requests read through pair copies as grids of their own on parallel branches. Build it once, then
``run()`` it as often as needed; the tensors it was given must stay alive and unchanged in shape.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import fourier_project as fp


class NbExtractRequest(C.Structure):
    _fields_ = [("volume", C.POINTER(fp.NbArray)), ("volume_weight", C.POINTER(fp.NbArray)),
                ("volume_shape", C.c_int64 * 4), ("slice", C.POINTER(fp.NbArray)),
                ("slice_weight", C.POINTER(fp.NbArray)), ("slice_shape", C.c_int64 * 4),
                ("inv_scaling", C.POINTER(fp.NbTransform)), ("fwd_rotation", C.POINTER(fp.NbTransform))]


class NbExtractRequestEx(C.Structure):
    _fields_ = [("call", NbExtractRequest), ("volume_pairs", C.c_void_p), ("volume_pairs_bytes", C.c_int64)]


class NbBatchInfo(C.Structure):
    _fields_ = [("n_requests", C.c_int64), ("n_items", C.c_int64), ("tile_h", C.c_int32), ("tile_w", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("grid", C.c_int32), ("tuned_ms", C.c_double),
                ("from_cache", C.c_int32), ("min_ctas", C.c_int32), ("n_direct", C.c_int32)]


NB_BATCH_AUTOTUNE = 1
NB_BATCH_PERSISTENT_ONLY = 2


@dataclass
class ExtractRequest:
    """The arguments of one extract_central_slices_3d call."""
    volume: object
    volume_shape: tuple
    slice: object
    slice_shape: tuple
    fwd_rotation: object
    inv_scaling: object = None
    volume_weight: object = None
    slice_weight: object = None


def _setup(lib):
    if getattr(lib, "_nb_batch_ready", False):
        return
    lib.nb_extract_batch_create.argtypes = [C.c_int32, C.POINTER(NbExtractRequest), C.c_int64,
                                            C.POINTER(fp.NbOptions), C.c_int32, C.c_void_p,
                                            C.POINTER(C.c_void_p)]
    lib.nb_extract_batch_create.restype = C.c_int
    lib.nb_extract_batch_run.argtypes = [C.c_void_p, C.c_void_p]
    lib.nb_extract_batch_run.restype = C.c_int
    lib.nb_extract_batch_info.argtypes = [C.c_void_p, C.POINTER(NbBatchInfo)]
    lib.nb_extract_batch_info.restype = C.c_int
    lib.nb_extract_batch_destroy.argtypes = [C.c_void_p]
    lib.nb_extract_batch_destroy.restype = C.c_int
    lib.nb_volume_pairs_bytes.argtypes = [C.POINTER(C.c_int64)]
    lib.nb_volume_pairs_bytes.restype = C.c_int64
    lib.nb_volume_pairs.argtypes = [C.POINTER(fp.NbArray), C.POINTER(C.c_int64), C.c_void_p, C.c_int64, C.c_void_p]
    lib.nb_volume_pairs.restype = C.c_int
    lib.nb_extract_batch_launch.argtypes = [C.c_int32, C.POINTER(NbExtractRequestEx), C.c_int64,
                                            C.POINTER(fp.NbOptions), C.c_void_p]
    lib.nb_extract_batch_launch.restype = C.c_int
    lib.nb_extract_batch_launch_ex.argtypes = [C.c_int32, C.POINTER(NbExtractRequestEx), C.c_int64,
                                               C.POINTER(fp.NbOptions), C.c_int32, C.c_void_p]
    lib.nb_extract_batch_launch_ex.restype = C.c_int
    lib.nb_rasterize_batch_launch.argtypes = [C.c_int32, C.POINTER(NbRasterizeRequest), C.c_int64,
                                              C.POINTER(fp.NbOptions), C.c_void_p]
    lib.nb_rasterize_batch_launch.restype = C.c_int
    lib._nb_batch_ready = True


class NbRasterizeRequest(C.Structure):
    _fields_ = [("slice", C.POINTER(fp.NbArray)), ("slice_weight", C.POINTER(fp.NbArray)),
                ("slice_shape", C.c_int64 * 4), ("volume", C.POINTER(fp.NbArray)),
                ("volume_weight", C.POINTER(fp.NbArray)), ("volume_shape", C.c_int64 * 4),
                ("inv_scaling", C.POINTER(fp.NbTransform)), ("fwd_rotation", C.POINTER(fp.NbTransform))]


@dataclass
class RasterizeRequest:
    """The arguments of one rasterize_central_slices_3d call (each request owns its output grids)."""
    slice: object
    slice_shape: tuple
    volume: object
    volume_shape: tuple
    fwd_rotation: object
    volume_weight: object = None
    slice_weight: object = None
    inv_scaling: object = None


def rasterize_batch_launch(remap: str, requests: list[RasterizeRequest], *, fftfreq_cutoff=0.5,
                           target_shape=None, ews_radius=(0.0, 0.0), stream=None) -> None:
    """Enqueues many rasterize_central_slices_3d calls, each into its own grids, as one scatter launch
    and one finalize launch on ``stream`` (nb_rasterize_batch_launch)."""
    lib = fp.lib()
    _setup(lib)
    keep = []
    reqs = (NbRasterizeRequest * len(requests))()
    for i, r in enumerate(requests):
        q = reqs[i]
        arrays = [fp.as_nb_array(t, keep) for t in (r.slice, r.slice_weight, r.volume, r.volume_weight)]
        keep.extend(a for a in arrays if a is not None)
        q.slice = C.pointer(arrays[0])
        q.slice_weight = C.pointer(arrays[1]) if arrays[1] is not None else None
        q.volume = C.pointer(arrays[2])
        q.volume_weight = C.pointer(arrays[3]) if arrays[3] is not None else None
        for k in range(4):
            q.slice_shape[k] = int(r.slice_shape[k])
            q.volume_shape[k] = int(r.volume_shape[k])
        sc = fp.as_nb_transform(r.inv_scaling, False, keep)
        rot = fp.as_nb_transform(r.fwd_rotation, True, keep)
        keep.extend([sc, rot])
        q.inv_scaling = C.pointer(sc)
        q.fwd_rotation = C.pointer(rot)
    opts = fp._options(fftfreq_cutoff=fftfreq_cutoff, target_shape=target_shape, ews_radius=ews_radius)
    fp._check(lib.nb_rasterize_batch_launch(fp.REMAPS[remap], reqs, len(requests), C.byref(opts),
                                            fp._stream_ptr(stream)))


def _fill_request(q: NbExtractRequest, r: ExtractRequest, keep: list) -> None:
    arrays = [fp.as_nb_array(t, keep) for t in (r.volume, r.volume_weight, r.slice, r.slice_weight)]
    keep.extend(a for a in arrays if a is not None)
    q.volume = C.pointer(arrays[0])
    q.volume_weight = C.pointer(arrays[1]) if arrays[1] is not None else None
    q.slice = C.pointer(arrays[2])
    q.slice_weight = C.pointer(arrays[3]) if arrays[3] is not None else None
    for k in range(4):
        q.volume_shape[k] = int(r.volume_shape[k])
        q.slice_shape[k] = int(r.slice_shape[k])
    sc = fp.as_nb_transform(r.inv_scaling, False, keep)
    rot = fp.as_nb_transform(r.fwd_rotation, True, keep)
    keep.extend([sc, rot])
    q.inv_scaling = C.pointer(sc)
    q.fwd_rotation = C.pointer(rot)


def volume_pairs(volume, volume_shape, stream=None):
    """The pair copy of one c32 rfft volume (1, D, H, W/2+1) for LINEAR extraction, as a uint8 device
    tensor. Extractions given it (``extract_batch_launch``) read 4 aligned 16-byte pairs per pixel."""
    torch = fp._torch()
    lib = fp.lib()
    _setup(lib)
    shape = (C.c_int64 * 4)(*[int(x) for x in volume_shape])
    nbytes = lib.nb_volume_pairs_bytes(shape)
    if nbytes <= 0:
        raise fp.NoaB200Error(fp.NB_ERROR_INVALID, f"bad volume shape {tuple(volume_shape)}")
    pairs = torch.empty(int(nbytes), dtype=torch.uint8, device=volume.device)
    keep = []
    arr = fp.as_nb_array(volume, keep)
    fp._check(lib.nb_volume_pairs(C.byref(arr), shape, pairs.data_ptr(), nbytes, fp._stream_ptr(stream)))
    return pairs


def extract_batch_launch(remap: str, requests: list[ExtractRequest], pairs: list | None = None, *,
                         interp="linear", fftfreq_cutoff=0.5, w_windowed_sinc=None, ews_radius=(0.0, 0.0),
                         persistent_only=False, stream=None) -> None:
    """Enqueues many extract_central_slices_3d calls on ``stream`` (no graph, no autotuning): requests
    of at least 2^21 output pixels read through their pair copy as grids of their own, the others as
    ONE persistent launch (every request, with ``persistent_only``). ``pairs[i]`` is an optional
    ``volume_pairs`` copy of request i's volume."""
    lib = fp.lib()
    _setup(lib)
    keep = []
    reqs = (NbExtractRequestEx * len(requests))()
    for i, r in enumerate(requests):
        _fill_request(reqs[i].call, r, keep)
        p = pairs[i] if pairs is not None else None
        if p is not None:
            reqs[i].volume_pairs = p.data_ptr()
            reqs[i].volume_pairs_bytes = p.numel() * p.element_size()
    opts = fp._options(interp=interp, fftfreq_cutoff=fftfreq_cutoff, ews_radius=ews_radius,
                       w_windowed_sinc=w_windowed_sinc)
    fp._check(lib.nb_extract_batch_launch_ex(fp.REMAPS[remap], reqs, len(requests), C.byref(opts),
                                             NB_BATCH_PERSISTENT_ONLY if persistent_only else 0,
                                             fp._stream_ptr(stream)))


class ExtractBatch:
    """A captured batch of extractions. ``autotune=True`` times tile shapes and CTAs per SM on this
    batch (once per workload key; the choice is cached) before capturing the launch. LINEAR requests
    of at least 2^23 output pixels read through a pair copy run as grids of their own inside the
    graph, unless ``persistent_only=True``."""

    def __init__(self, remap: str, requests: list[ExtractRequest], *, interp="linear", fftfreq_cutoff=0.5,
                 w_windowed_sinc=None, ews_radius=(0.0, 0.0), autotune=True, persistent_only=False, stream=None):
        lib = fp.lib()
        _setup(lib)
        self._lib = lib
        self._handle = None
        self._keep = []
        reqs = (NbExtractRequest * len(requests))()
        for i, r in enumerate(requests):
            _fill_request(reqs[i], r, self._keep)
        self._keep.append(reqs)
        opts = fp._options(interp=interp, fftfreq_cutoff=fftfreq_cutoff, ews_radius=ews_radius,
                           w_windowed_sinc=w_windowed_sinc)
        handle = C.c_void_p()
        code = lib.nb_extract_batch_create(fp.REMAPS[remap], reqs, len(requests), C.byref(opts),
                                           (NB_BATCH_AUTOTUNE if autotune else 0) |
                                           (NB_BATCH_PERSISTENT_ONLY if persistent_only else 0), fp._stream_ptr(stream),
                                           C.byref(handle))
        fp._check(code)
        self._handle = handle

    def run(self, stream=None) -> None:
        fp._check(self._lib.nb_extract_batch_run(self._handle, fp._stream_ptr(stream)))

    def info(self) -> dict:
        i = NbBatchInfo()
        fp._check(self._lib.nb_extract_batch_info(self._handle, C.byref(i)))
        return {"n_requests": i.n_requests, "n_items": i.n_items, "tile": (i.tile_h, i.tile_w),
                "blocks_per_sm": i.blocks_per_sm, "grid": i.grid, "tuned_ms": i.tuned_ms,
                "from_cache": bool(i.from_cache), "min_ctas": i.min_ctas, "n_direct": i.n_direct}

    def close(self) -> None:
        if getattr(self, "_handle", None):
            self._lib.nb_extract_batch_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
