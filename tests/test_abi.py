"""CPU tests of the drop-in boundary: the C-ABI library loads, exports every entry point its public
header declares, and rejects invalid calls on the host (no GPU needed for these paths)."""
import ctypes as C
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "noa_b200", "*.h")))


def declared_symbols():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        names.update(re.findall(r"^NB_API\s+[\w\s\*]+?\b(nb_\w+)\s*\(", src, flags=re.M))
    return sorted(names)


def _lib():
    from noa_b200 import fourier_project as fp
    if not os.path.exists(fp.library_path()):
        pytest.skip("noa_b200 library not built (python -m noa_b200.build)")
    return fp.lib()


def test_headers_declare_entry_points():
    syms = declared_symbols()
    for name in ("nb_extract_central_slices_3d", "nb_rasterize_central_slices_3d",
                 "nb_insert_central_slices_3d", "nb_insert_and_extract_central_slices_3d", "nb_last_error"):
        assert name in syms


def test_library_exports_every_declared_symbol():
    lib = _lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_defaults():
    from noa_b200 import fourier_project as fp
    lib = _lib()
    assert lib.nb_version().decode().count(".") == 2
    o = fp.NbOptions()
    lib.nb_options_default(C.byref(o))
    assert o.interp == 1 and o.fftfreq_cutoff == 0.5
    assert o.fftfreq_sinc == -1 and o.fftfreq_blackman == -1
    assert o.w_fftfreq_sinc == -1 and o.w_fftfreq_blackman == -1
    assert list(o.target_shape) == [0, 0, 0, 0]


def _args(fp):
    a = fp.NbArray()
    a.dtype = fp.DTYPE_C32
    a.data = 0x1000
    shape = (C.c_int64 * 4)(1, 16, 16, 16)
    t = fp.NbTransform()
    t.kind = fp.XFORM_MAT33
    t.count = 1
    o = fp.NbOptions()
    _lib().nb_options_default(C.byref(o))
    return a, shape, t, o


def test_rejects_bad_remap_on_host():
    from noa_b200 import fourier_project as fp
    lib = _lib()
    a, shape, t, o = _args(fp)
    rc = lib.nb_extract_central_slices_3d(3, C.byref(a), None, shape, C.byref(a), None, shape,
                                          None, C.byref(t), C.byref(o), None)
    assert rc == fp.NB_ERROR_INVALID
    assert "remap" in lib.nb_last_error().decode()


def test_rejects_null_options_and_shapes():
    from noa_b200 import fourier_project as fp
    lib = _lib()
    a, shape, t, o = _args(fp)
    assert lib.nb_rasterize_central_slices_3d(0, C.byref(a), None, shape, C.byref(a), None, shape,
                                              None, C.byref(t), None, None) == fp.NB_ERROR_INVALID
    bad = (C.c_int64 * 4)(1, 0, 16, 16)
    assert lib.nb_insert_central_slices_3d(0, C.byref(a), None, bad, C.byref(a), None, shape,
                                           None, C.byref(t), C.byref(o), None) == fp.NB_ERROR_INVALID
    assert "Empty" in lib.nb_last_error().decode()


def test_rejects_bad_interp_on_host():
    from noa_b200 import fourier_project as fp
    lib = _lib()
    a, shape, t, o = _args(fp)
    o.interp = 7
    rc = lib.nb_extract_central_slices_3d(4, C.byref(a), None, shape, C.byref(a), None, shape,
                                          None, C.byref(t), C.byref(o), None)
    assert rc == fp.NB_ERROR_INVALID and "interpolation" in lib.nb_last_error().decode()


def test_python_api_raises():
    from noa_b200 import fourier_project as fp
    _lib()
    with pytest.raises(fp.NoaB200Error):
        fp.as_nb_transform(None, True, [])
