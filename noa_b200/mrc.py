"""MRC2014 files for resident volumes and slice stacks (host side, numpy).

The format is the public MRC2014 one (https://www.ccpem.ac.uk/mrc_format/mrc2014.php): a 1024-byte
header of 56 32-bit words followed by 10 80-byte labels, an optional extended header, then the data,
x fastest. Shapes follow noa's BDHW convention: a volume is (1, D, H, W) with space group 1, a stack of
2-D images (B, 1, H, W) with space group 0, a stack of volumes (B, D, H, W) with space group 401 and
mz = D sections per volume. Supported modes: 0 (int8), 1 (int16), 2 (float32), 4 (complex64, e.g. an
rfft volume stored with its physical width), 6 (uint16), 12 (float16).

    write(path, array, pixel_size=(1, 1, 1))     # array: 2-D, 3-D or 4-D (BDHW) numpy array
    data, header = read(path)                    # data in BDHW, header: dict of the fields used
"""
from __future__ import annotations

import struct

import numpy as np

HEADER_BYTES = 1024
_MODES = {0: np.int8, 1: np.int16, 2: np.float32, 4: np.complex64, 6: np.uint16, 12: np.float16}
_DTYPE_TO_MODE = {np.dtype(v): k for k, v in _MODES.items()}


def _bdhw(a: np.ndarray) -> np.ndarray:
    if a.ndim == 2:
        return a[None, None]
    if a.ndim == 3:
        return a[None]
    if a.ndim == 4:
        return a
    raise ValueError(f"expected a 2-D, 3-D or 4-D array, got {a.ndim}-D")


def write(path: str, array, pixel_size=(1.0, 1.0, 1.0), label: str = "noa_b200") -> None:
    """Writes ``array`` (BDHW, or DHW / HW) little-endian. ``pixel_size`` is (d, h, w) in Angstrom."""
    a = _bdhw(np.ascontiguousarray(np.asarray(array)))
    mode = _DTYPE_TO_MODE.get(a.dtype)
    if mode is None:
        raise ValueError(f"no MRC mode for dtype {a.dtype}")
    b, d, h, w = a.shape
    if b > 1 and d > 1:
        nz, mz, ispg = b * d, d, 401
    elif b > 1:
        nz, mz, ispg = b, 1, 0
    else:
        nz, mz, ispg = d, d, 1
    nx, ny = w, h
    mx, my = w, h
    pd, ph, pw = (float(p) for p in pixel_size)
    mag = np.abs(a) if np.iscomplexobj(a) else a.astype(np.float64)
    stats = (float(mag.min()), float(mag.max()), float(mag.mean()), float(mag.std())) if a.size else (0, 0, 0, 0)
    hdr = bytearray(HEADER_BYTES)
    struct.pack_into("<3i", hdr, 0, nx, ny, nz)
    struct.pack_into("<i", hdr, 12, mode)
    struct.pack_into("<3i", hdr, 16, 0, 0, 0)                       # nxstart, nystart, nzstart
    struct.pack_into("<3i", hdr, 28, mx, my, mz)
    struct.pack_into("<3f", hdr, 40, pw * mx, ph * my, pd * mz)     # cell dimensions (x, y, z)
    struct.pack_into("<3f", hdr, 52, 90.0, 90.0, 90.0)
    struct.pack_into("<3i", hdr, 64, 1, 2, 3)                       # mapc, mapr, maps
    struct.pack_into("<3f", hdr, 76, stats[0], stats[1], stats[2])  # dmin, dmax, dmean
    struct.pack_into("<i", hdr, 88, ispg)
    struct.pack_into("<i", hdr, 92, 0)                              # no extended header
    hdr[104:108] = b"\0\0\0\0"                                      # exttyp
    struct.pack_into("<i", hdr, 108, 20140)                         # nversion
    hdr[208:212] = b"MAP "
    hdr[212:216] = bytes([68, 68, 0, 0])                            # little-endian machine stamp
    struct.pack_into("<f", hdr, 216, stats[3])                      # rms
    struct.pack_into("<i", hdr, 220, 1)                             # nlabl
    lab = label.encode("ascii", "replace")[:80]
    hdr[224:224 + len(lab)] = lab
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes())


def read_header(path: str) -> dict:
    with open(path, "rb") as f:
        raw = f.read(HEADER_BYTES)
    if len(raw) < HEADER_BYTES:
        raise ValueError(f"{path}: shorter than the 1024-byte MRC header")
    stamp = raw[212:216]
    if stamp[0] == 68 and stamp[1] in (65, 68):
        e = "<"
    elif stamp[0] == 17 and stamp[1] == 17:
        e = ">"
    else:
        raise ValueError(f"{path}: unrecognised machine stamp {list(stamp)}")
    nx, ny, nz, mode = struct.unpack_from(e + "4i", raw, 0)
    mx, my, mz = struct.unpack_from(e + "3i", raw, 28)
    cx, cy, cz = struct.unpack_from(e + "3f", raw, 40)
    ispg, nsymbt = struct.unpack_from(e + "2i", raw, 88)
    if min(nx, ny, nz) <= 0:
        raise ValueError(f"{path}: invalid shape nx,ny,nz = {nx},{ny},{nz}")
    if mode not in _MODES:
        raise ValueError(f"{path}: unsupported mode {mode}")
    if nz > 1 and ispg >= 401 and mz > 0 and nz % mz == 0:
        shape = (nz // mz, mz, ny, nx)
    elif nz > 1 and ispg == 0:
        shape = (nz, 1, ny, nx)
    else:
        shape = (1, nz, ny, nx)
    spacing = tuple(c / m if m > 0 else 0.0 for c, m in ((cz, mz), (cy, my), (cx, mx)))
    return {"shape": shape, "mode": mode, "dtype": np.dtype(_MODES[mode]).newbyteorder(e),
            "pixel_size": spacing, "space_group": ispg, "extended_bytes": nsymbt, "endian": e}


def read(path: str) -> tuple[np.ndarray, dict]:
    """Returns (data in BDHW, native byte order; header fields)."""
    h = read_header(path)
    count = int(np.prod(h["shape"]))
    with open(path, "rb") as f:
        f.seek(HEADER_BYTES + h["extended_bytes"])
        data = np.fromfile(f, dtype=h["dtype"], count=count)
    if data.size != count:
        raise ValueError(f"{path}: expected {count} elements, found {data.size}")
    return data.astype(h["dtype"].newbyteorder("="), copy=False).reshape(h["shape"]), h
