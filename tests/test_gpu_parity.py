"""GPU parity: the sm_100a kernels, called through the C ABI, against the oracle (the C restatement
pinned bit-exactly to noa's CPU path). Tolerances (relative L2 over the whole output):
  extract, insert (gather), insert_and_extract: 1e-5      rasterize (f32 atomics): 1e-4
"""
import numpy as np
import pytest

from cases import build, case_id, clone, default_case, pin_cases, rel_l2
from oracle.oracle import FpOracle

pytestmark = pytest.mark.gpu

TOL = {"extract": 1e-5, "insert": 1e-5, "insert_extract": 1e-5, "rasterize": 1e-4}


def _gpu_cases():
    cases = [c for c in pin_cases() if c["out_dt"] in ("c32", "f32")]
    extra = [
        default_case("extract", n=33, slice_n=33, seed=601),                      # odd sizes
        default_case("extract", n=64, nslices=16, remap="hc2h", seed=602),
        default_case("extract", n=48, slice_n=64, target=(1, 64, 64, 64), seed=603),
        default_case("extract", interp="lanczos8", n=40, seed=604, out_w=True, in_w=True),
        default_case("extract", interp="cubic_bspline", rot="quat", scale=True, seed=605),
        default_case("rasterize", n=64, nslices=16, remap="h2hc", out_w=True, seed=606),
        default_case("rasterize", n=48, slice_n=64, cutoff=0.45, seed=607),
        default_case("insert", n=32, nslices=24, out_w=True, sinc=(-1.0, 0.05), seed=608),
        default_case("insert", n=32, nslices=24, interp="lanczos6", seed=609),
        default_case("insert_extract", n=32, nslices=16, nout=6, sinc=(0.01, 0.03), out_w=True, seed=610),
        default_case("insert_extract", n=32, nslices=16, nout=6, sinc=(0.01, 0.03), interp="cubic", seed=611),
    ]
    return cases + extra


@pytest.mark.parametrize("case", _gpu_cases(), ids=case_id)
def test_gpu_matches_oracle(case):
    import gpu_run
    call = build(case)
    ref = clone(call)
    assert FpOracle().run(ref, 8) == 0
    out, out_w = gpu_run.run(clone(call))
    tol = TOL[case["func"]]
    err = rel_l2(out, ref.out)
    assert err <= tol, f"rel L2 {err:.3e} > {tol:g}"
    if ref.out_w is not None:
        errw = rel_l2(out_w, ref.out_w)
        assert errw <= tol, f"weights rel L2 {errw:.3e} > {tol:g}"


def _insert_cases():
    return [c for c in _gpu_cases() if c["func"] == "insert"] + [
        default_case("insert", n=40, nslices=60, out_w=True, sinc=(-1.0, 6 / 40), remap="hc2hc", seed=620),
        default_case("insert", n=33, nslices=30, out_w=True, in_w=True, sinc=(0.03, 0.1), remap="h2hc", seed=621),
        default_case("insert", n=32, nslices=20, in_dt="c32", out_dt="f32", sinc=(-1.0, 0.1), seed=622),
    ]


@pytest.mark.parametrize("case", _insert_cases(), ids=case_id)
def test_gpu_scatter_insert_matches_oracle(case):
    """The slice-major scatter form: the gather form's terms, summed in atomic order (tolerance 1e-5)."""
    import gpu_run
    call = build(case)
    ref = clone(call)
    assert FpOracle().run(ref, 8) == 0
    out, out_w = gpu_run.run(clone(call), scatter=True)
    err = rel_l2(out, ref.out)
    assert err <= TOL["insert"], f"rel L2 {err:.3e}"
    if ref.out_w is not None:
        assert rel_l2(out_w, ref.out_w) <= TOL["insert"]


def test_gpu_rejects_f64_values():
    import torch
    from noa_b200 import fourier_project as fp
    n = 16
    vol = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex128, device="cuda")
    out = torch.zeros((2, 1, n, n // 2 + 1), dtype=torch.complex128, device="cuda")
    rot = torch.eye(3).repeat(2, 1, 1).cuda()
    with pytest.raises(fp.NoaB200Error) as e:
        fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), out, None, (2, 1, n, n), None, rot)
    assert e.value.code == fp.NB_ERROR_UNSUPPORTED


def test_gpu_rejects_shape_mismatch_and_overlap():
    import torch
    from noa_b200 import fourier_project as fp
    n = 16
    vol = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    out = torch.zeros((2, 1, n, n // 2), dtype=torch.complex64, device="cuda")
    rot = torch.eye(3).repeat(2, 1, 1).cuda()
    with pytest.raises(fp.NoaB200Error) as e:
        fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n), out, None, (2, 1, n, n), None, rot)
    assert e.value.code == fp.NB_ERROR_INVALID
    big = torch.zeros((1, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    view_out = big[:, :2].permute(1, 0, 2, 3)  # overlaps the input below
    with pytest.raises(fp.NoaB200Error):
        fp.extract_central_slices_3d("hc2h", big, None, (1, n, n, n), view_out, None, (2, 1, n, n), None, rot)
    # A transform array with the wrong count.
    with pytest.raises(fp.NoaB200Error):
        fp.extract_central_slices_3d("hc2h", vol, None, (1, n, n, n),
                                     torch.zeros((3, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda"),
                                     None, (3, 1, n, n), None, rot)
    # Host memory is refused.
    with pytest.raises(fp.NoaB200Error):
        fp.extract_central_slices_3d("hc2h", vol.cpu(), None, (1, n, n, n), out, None, (2, 1, n, n), None, rot)


def test_gpu_strided_and_broadcast_inputs():
    """Non-contiguous outputs/inputs (noa Views with strides) and a single inline rotation."""
    import torch
    import gpu_run  # noqa: F401
    from noa_b200 import fourier_project as fp
    call = build(default_case("extract", n=32, nslices=4, seed=620))
    call.rot = np.repeat(call.rot[:1], 4, axis=0)
    ref = clone(call)
    FpOracle().run(ref, 4)
    n = 32
    vol = torch.from_numpy(call.inp).cuda()
    vol_padded = torch.zeros((1, n, n, n // 2 + 1 + 3), dtype=torch.complex64, device="cuda")
    vol_padded[..., : n // 2 + 1] = vol
    vol_view = vol_padded[..., : n // 2 + 1]
    out_t = torch.zeros((n, n // 2 + 1, 1, 4), dtype=torch.complex64, device="cuda").permute(3, 2, 0, 1)
    fp.extract_central_slices_3d("hc2h", vol_view, None, (1, n, n, n), out_t, None, (4, 1, n, n), None,
                                 call.rot[0].astype(np.float64))
    torch.cuda.synchronize()
    assert rel_l2(out_t.cpu().numpy(), ref.out) <= 1e-5


def test_gpu_constant_input_rasterize():
    """A constant slice value (noa's AllowValue inputs) against the oracle's constant input."""
    import gpu_run
    call = build(default_case("rasterize", n=32, nslices=6, out_w=True, seed=621))
    call.inp_value = complex(1.5, -0.25)
    call.inp_value_shape = (6, 1, 32, 17)
    ref = clone(call)
    FpOracle().run(ref, 1)
    out, out_w = gpu_run.run(clone(call))
    assert rel_l2(out, ref.out) <= 1e-4
    assert rel_l2(out_w, ref.out_w) <= 1e-4


@pytest.mark.parametrize("remap", ["h2h", "h2hc", "hc2h", "hc2hc"])
@pytest.mark.parametrize("out_dt", ["c32", "f32"])
def test_gpu_extract_pair_path(remap, out_dt):
    """Enough slices that extraction takes the pair-copy fast path (pixels >= 2 x voxels)."""
    import gpu_run
    call = build(default_case("extract", remap=remap, n=32, nslices=80, out_dt=out_dt, out_w=True, seed=640))
    ref = clone(call)
    FpOracle().run(ref, 8)
    out, out_w = gpu_run.run(clone(call))
    assert rel_l2(out, ref.out) <= 1e-5
    assert rel_l2(out_w, ref.out_w) <= 1e-5


def _generic_forced(call):
    """The same extraction through the generic kernel: input weights (which change only the output
    weights) keep a call off the pair copy."""
    c = clone(call)
    c.inp_w = np.ones(call.inp.shape, np.float32)
    return c


@pytest.mark.parametrize("variant", ["plain", "scaled", "ews"])
def test_gpu_extract_pair_path_bit_identical_to_generic(variant):
    """The pair path and the generic path give identical values, also with scaling and the Ewald
    curvature (which the pair kernels compute through the same slice2grid)."""
    import gpu_run
    kw = {"scaled": dict(scale=True), "ews": dict(ews=(45.0, 60.0))}.get(variant, {})
    call = build(default_case("extract", remap="hc2h", n=48, nslices=96, seed=641, **kw))
    a, _ = gpu_run.run(clone(call))
    b, _ = gpu_run.run(_generic_forced(call))
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("variant", ["scaled", "ews"])
def test_gpu_extract_pair_path_scaled_or_curved(variant):
    """Scaled and curved extractions through the pair copy, against the oracle."""
    import gpu_run
    kw = {"scaled": dict(scale=True), "ews": dict(ews=(45.0, 60.0))}[variant]
    call = build(default_case("extract", remap="h2hc", n=32, nslices=80, out_w=True, seed=644, **kw))
    ref = clone(call)
    FpOracle().run(ref, 8)
    out, out_w = gpu_run.run(clone(call))
    assert rel_l2(out, ref.out) <= 1e-5
    assert rel_l2(out_w, ref.out_w) <= 1e-5


@pytest.mark.parametrize("remap", ["h2h", "hc2hc"])
@pytest.mark.parametrize("out_dt", ["c32", "f32"])
def test_gpu_extract_pair_path_w_window(remap, out_dt):
    """The w-windowed extraction through the pair copy (5-sample window, enough slices)."""
    import gpu_run
    call = build(default_case("extract", remap=remap, n=32, nslices=80, out_dt=out_dt, out_w=True,
                              w_sinc=(1.5 / 32, 3.0 / 32), seed=642))
    ref = clone(call)
    FpOracle().run(ref, 8)
    out, out_w = gpu_run.run(clone(call))
    assert rel_l2(out, ref.out) <= 1e-5
    assert rel_l2(out_w, ref.out_w) <= 1e-5


def test_gpu_extract_pair_path_w_window_bit_identical_to_generic():
    """With the w-window too, the pair path and the generic path give identical bits."""
    import gpu_run
    call = build(default_case("extract", remap="hc2h", n=48, nslices=96, out_w=True, w_sinc=(2.0 / 48, 4.0 / 48),
                              seed=643))
    a, _ = gpu_run.run(clone(call))
    b, _ = gpu_run.run(_generic_forced(call))
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("out_w", [False, True])
@pytest.mark.parametrize("dts", [("c32", "c32"), ("c32", "f32"), ("f32", "f32")])
def test_gpu_rasterize_accumulator_paths(out_w, dts):
    """Rasterization through the interleaved scratch (weights) and straight into the grid (no weights),
    accumulating on top of existing grid contents."""
    import gpu_run
    call = build(default_case("rasterize", remap="h2hc", n=48, nslices=40, in_dt=dts[0], out_dt=dts[1],
                              out_w=out_w, in_w=out_w, seed=650))
    rng = np.random.default_rng(5)
    call.out[...] = rng.standard_normal(call.out.shape).astype(call.out.dtype)
    if out_w:
        call.out_w[...] = rng.uniform(0, 1, call.out_w.shape).astype(np.float32)
    ref = clone(call)
    FpOracle().run(ref, 1)
    out, ow = gpu_run.run(clone(call))
    assert rel_l2(out, ref.out) <= 1e-4
    if out_w:
        assert rel_l2(ow, ref.out_w) <= 1e-4
