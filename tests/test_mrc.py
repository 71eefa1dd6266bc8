"""MRC2014 files (noa_b200.mrc): round trips of volumes, image stacks and volume stacks, the header
fields the format defines, and big-endian files."""
import struct

import numpy as np
import pytest

from noa_b200 import mrc


@pytest.mark.parametrize("shape,dtype", [((1, 12, 10, 8), np.float32), ((5, 1, 9, 7), np.float32),
                                         ((3, 4, 6, 5), np.float16), ((1, 16, 16, 9), np.complex64),
                                         ((2, 1, 4, 4), np.int16)])
def test_round_trip(tmp_path, shape, dtype):
    rng = np.random.default_rng(0)
    a = rng.standard_normal(shape) * 10
    if np.issubdtype(dtype, np.complexfloating):
        a = a + 1j * rng.standard_normal(shape)
    a = a.astype(dtype)
    p = str(tmp_path / "x.mrc")
    mrc.write(p, a, pixel_size=(1.5, 2.0, 2.5))
    b, h = mrc.read(p)
    assert b.shape == shape and b.dtype == np.dtype(dtype)
    assert np.array_equal(a, b)
    assert h["pixel_size"] == pytest.approx((1.5, 2.0, 2.5))


def test_header_fields(tmp_path):
    a = np.zeros((1, 6, 5, 4), np.float32)
    a[0, 1, 2, 3] = 2.0
    p = str(tmp_path / "v.mrc")
    mrc.write(p, a)
    raw = open(p, "rb").read()
    assert len(raw) == 1024 + a.nbytes
    assert struct.unpack_from("<4i", raw, 0) == (4, 5, 6, 2)        # nx, ny, nz, mode
    assert struct.unpack_from("<3i", raw, 28) == (4, 5, 6)          # mx, my, mz
    assert struct.unpack_from("<3i", raw, 64) == (1, 2, 3)          # axis order
    assert struct.unpack_from("<i", raw, 88)[0] == 1                # volume
    assert raw[208:212] == b"MAP " and raw[212:214] == bytes([68, 68])
    dmin, dmax, dmean = struct.unpack_from("<3f", raw, 76)
    assert (dmin, dmax) == (0.0, 2.0) and dmean == pytest.approx(2.0 / a.size)


def test_big_endian_file(tmp_path):
    a = np.arange(24, dtype=np.float32).reshape(1, 2, 3, 4)
    p = str(tmp_path / "le.mrc")
    mrc.write(p, a)
    raw = bytearray(open(p, "rb").read())
    # Rewrite as big-endian: swap the header words the reader uses and the data, set the stamp.
    for off in list(range(0, 96, 4)) + [216, 220]:
        raw[off:off + 4] = raw[off:off + 4][::-1]
    raw[212:216] = bytes([17, 17, 0, 0])
    raw[1024:] = a.astype(">f4").tobytes()
    q = str(tmp_path / "be.mrc")
    open(q, "wb").write(bytes(raw))
    b, h = mrc.read(q)
    assert h["endian"] == ">" and np.array_equal(a, b)


def test_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.mrc"
    p.write_bytes(b"\0" * 100)
    with pytest.raises(ValueError):
        mrc.read(str(p))
    p.write_bytes(b"\0" * 1024)
    with pytest.raises(ValueError):
        mrc.read(str(p))
    with pytest.raises(ValueError):
        mrc.write(str(tmp_path / "x.mrc"), np.zeros((2, 2), np.float64))
