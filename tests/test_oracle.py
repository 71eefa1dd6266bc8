"""CPU tests: the C restatement (oracle/libfp_oracle.so) is pinned to the reference's own CPU path.

* against the committed golden fixtures (outputs of noa's CPU path, tests/golden/make_golden.py), bit
  for bit — runs wherever the oracle is built;
* against the reference library itself (oracle/_ref), on every pinning case, when it was built here.
"""
import glob
import json
import os

import numpy as np
import pytest

from cases import build, case_id, clone, pin_cases, rel_l2
from oracle.oracle import Call, FpOracle, RefLib, fp_available, ref_available

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "g*.npz")))
GOLDEN_GRIDDING = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "h*_gridding.npz")))

pytestmark = pytest.mark.skipif(not fp_available(), reason="oracle not built (make -C oracle fp)")


def _call_from_fixture(path):
    z = np.load(path)
    c = json.loads(str(z["meta"]))
    call = build(c)  # rebuilds the same seeded inputs; the fixture's arrays are checked against them
    for name in ("inp", "inp_w", "rot", "scale", "rot2", "scale2"):
        if name in z:
            np.testing.assert_array_equal(getattr(call, name), z[name], err_msg=f"{name} generator drift")
    call.out = z["out_init"].copy()
    if "out_w_init" in z:
        call.out_w = z["out_w_init"].copy()
    return c, call, z


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_reference_golden(path):
    c, call, z = _call_from_fixture(path)
    assert FpOracle().run(call, 1) == 0
    np.testing.assert_array_equal(call.out, z["out"], err_msg=case_id(c))
    if "out_w" in z:
        np.testing.assert_array_equal(call.out_w, z["out_w"], err_msg=case_id(c))


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 60


@pytest.mark.skipif(not ref_available(), reason="reference CPU path not built (make -C oracle ref)")
@pytest.mark.parametrize("case", pin_cases(), ids=case_id)
def test_oracle_matches_reference_library(case):
    call = build(case)
    a, b = clone(call), clone(call)
    assert FpOracle().run(a, 1) == 0
    status, err = RefLib().run(b, 1)
    assert status == 0, err
    np.testing.assert_array_equal(a.out, b.out)
    if a.out_w is not None:
        np.testing.assert_array_equal(a.out_w, b.out_w)


def test_oracle_threads_deterministic():
    """The gather forms are parallel over outputs; the result does not depend on the thread count."""
    for func in ("extract", "insert", "insert_extract"):
        call = build(dict(pin_cases()[0], func=func, n=20, nslices=5, nout=3, sinc=(0.02, 0.06)))
        a, b = clone(call), clone(call)
        FpOracle().run(a, 1)
        FpOracle().run(b, 4)
        np.testing.assert_array_equal(a.out, b.out)


def test_oracle_fp64_close_to_fp32():
    """The FP64 oracle (same algorithm in double) agrees with the f32 path to single precision.
    The cutoff is kept off the lattice points of the 0.5 sphere, where f32 and f64 may decide a
    pixel's in/out test differently."""
    from cases import default_case
    c32 = build(default_case("extract", n=32, nslices=8, seed=7, cutoff=0.45))
    c64 = build(default_case("extract", n=32, nslices=8, seed=7, in_dt="c64", out_dt="c64", cutoff=0.45))
    c64.inp = c32.inp.astype(np.complex128)
    c64.rot = c32.rot.astype(np.float64)
    FpOracle().run(c32, 2)
    FpOracle().run(c64, 2)
    assert rel_l2(c32.out, c64.out) < 1e-5


def test_oracle_rejects_bad_interp():
    from cases import default_case
    call = build(default_case("extract", n=16, nslices=2))
    call.interp = 42
    assert FpOracle().run(call, 1) != 0


def test_known_answer_identity_extract():
    """Identity rotation, hc2hc, LINEAR: the extracted central slice is the volume's z=0 plane inside
    the cutoff and 0 outside (FourierProject.hpp:647-656)."""
    from noa_b200 import synthetic
    n = 16
    vol = synthetic.make_volume(n, seed=3)
    out = np.zeros((1, 1, n, n // 2 + 1), np.complex64)
    call = Call(func="extract", remap="hc2hc", inp=vol, in_shape=(1, n, n, n), out=out, out_shape=(1, 1, n, n),
                rot=np.eye(3, dtype=np.float32)[None])
    FpOracle().run(call, 1)
    f = synthetic.slice_fftfreq_norm((n, n), centered=True)
    expected = np.where(f <= 0.5, vol[0, n // 2], 0)
    np.testing.assert_allclose(call.out[0, 0], expected, rtol=0, atol=0)


# ---------------------------------------------------------------------------------------------------
# Gridding correction. As published, the reference's GriddingCorrection does not compile
# (FourierProject.hpp:1034 hands Vec::from_vec the single bool of `l_shape != 1`); oracle/_ref builds it
# with that expression written per element (oracle/ref_gridding.cpp), and the oracle is pinned bit for
# bit to that build: to its fixtures (h*_gridding.npz) and, where it was built, to the library itself.
# The numpy restatement of the documented formula below is an independent check.
# ---------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("path", GOLDEN_GRIDDING, ids=[os.path.basename(p) for p in GOLDEN_GRIDDING])
def test_oracle_gridding_matches_reference_golden(path):
    from oracle.oracle import gridding_correction
    z = np.load(path)
    c = json.loads(str(z["meta"]))
    shape = tuple(c["shape"])
    inp = z["inp"]
    src = np.broadcast_to(inp, shape) if c["broadcast"] else inp
    out = np.zeros(shape, dtype=inp.dtype)
    assert gridding_correction(src, out, post_correction=c["post"]) == 0
    np.testing.assert_array_equal(out, z["out"])


def test_gridding_fixtures_present():
    assert len(GOLDEN_GRIDDING) >= 7


@pytest.mark.skipif(not ref_available(), reason="reference CPU path not built (make -C oracle ref)")
@pytest.mark.parametrize("shape", [(1, 32, 32, 32), (1, 33, 31, 17), (2, 5, 1, 40), (1, 64, 64, 1)])
@pytest.mark.parametrize("post", [True, False])
def test_oracle_gridding_matches_reference_library(shape, post):
    from oracle.oracle import gridding_correction, ref_gridding_correction
    rng = np.random.default_rng(sum(shape) + post)
    for dt in (np.float32, np.float64):
        inp = rng.standard_normal(shape).astype(dt)
        a, b = np.zeros(shape, dt), np.zeros(shape, dt)
        assert gridding_correction(inp, a, post_correction=post) == 0
        status, err = ref_gridding_correction(inp, b, post_correction=post, threads=4)
        assert status == 0, err
        np.testing.assert_array_equal(a, b)

def _numpy_gridding(inp, shape, post):
    b, d, h, w = shape
    half = np.array([s / 2 if s != 1 else 0.0 for s in (d, h, w)])
    j, k, l = np.meshgrid(np.arange(d), np.arange(h), np.arange(w), indexing="ij")
    dist = np.stack([(j - half[0]) / d, (k - half[1]) / h, (l - half[2]) / w])
    x = np.pi * np.sqrt((dist ** 2).sum(0))
    with np.errstate(invalid="ignore", divide="ignore"):
        sinc = np.where(x == 0, 1.0, np.sin(x) / x)
    s2 = np.broadcast_to(sinc ** 2, shape)
    v = np.broadcast_to(np.asarray(inp, dtype=np.float64), shape)
    return v / s2 if post else v * s2


@pytest.mark.parametrize("shape", [(1, 16, 16, 16), (2, 9, 12, 7), (1, 1, 20, 20), (1, 24, 1, 1)])
@pytest.mark.parametrize("post", [True, False])
def test_oracle_gridding_matches_formula(shape, post):
    from oracle.oracle import gridding_correction
    rng = np.random.default_rng(sum(shape))
    inp = rng.standard_normal(shape)
    for dt, tol in ((np.float32, 2e-6), (np.float64, 1e-12)):
        out = np.zeros(shape, dtype=dt)
        assert gridding_correction(inp.astype(dt), out, post_correction=post) == 0
        ref = _numpy_gridding(inp.astype(dt).astype(np.float64), shape, post)
        assert np.max(np.abs(out - ref) / np.maximum(np.abs(ref), 1e-30)) < tol
    out = np.zeros(shape, dtype=np.float32)
    assert gridding_correction(2.5, out, post_correction=post) == 0
    assert np.allclose(out, _numpy_gridding(2.5, shape, post), rtol=2e-6)
    assert gridding_correction(inp.astype(np.float32), out, interp=2) == -2  # LINEAR only
