"""Error of the device path against the FP64 oracle, per workload.

The FP64 oracle is the C restatement instantiated in double precision, fed the same f32 input values
upcast to f64 and the rotations as composed in f64 (before their cast to f32). Beside the device's
error, each case reports the error of the f32 oracle (which is bit-identical to noa's own f32 CPU
path) against the same FP64 result: the device's error should be that of single precision itself,
not more. The parity bar proper (1e-5 / 1e-4 against the f32 path) is in test_gpu_parity.py.

Two figures per case (printed; run with -s). "all" is the relative L2 over the whole output. It is
dominated by samples on the cutoff sphere: pixels such as (v, u) = (0, n/2) sit exactly at |f| = 0.5,
and whether a rotated copy passes |f|^2 <= 0.25 is decided by rounding, differently in f32 and f64
(an extracted pixel is then 0 in one and a full value in the other; a rasterized one adds or not).
"interior" excludes outputs within two voxels (or 1e-4 in |f|^2 for slice pixels) of that sphere and
is the error of the interpolation arithmetic itself: it must stay below the parity bar (1e-5 for
extraction, 1e-4 for insertion), and the device's "all" must equal the f32 path's (same decisions).

Workloads (seeded, synthetic; slice subsets keep the FP64 oracle within seconds):
  extract_64 / rasterize_64      the 64^3 extract-then-rasterize workload, 64 slices
  extract_256 / rasterize_256    256^3, 256 of the 4096 slices (LINEAR, hc2h / h2hc + weights, B=100)
  lanczos8_128 / lanczos8_192    LANCZOS8 extraction of 32 slices from boxes 128 and 192
  insert_sinc_128 (gather, scatter)  windowed-sinc insertion, half-width 6 voxels, 64 slices into 128^3
"""
import numpy as np
import pytest

from cases import clone, rel_l2
from noa_b200 import synthetic
from oracle.oracle import Call, FpOracle, INTERPS

pytestmark = pytest.mark.gpu

THREADS = 8


def _upcast(call: Call, rot64: np.ndarray) -> Call:
    c = clone(call)
    c.inp = call.inp.astype(np.complex128 if np.iscomplexobj(call.inp) else np.float64)
    c.out = np.zeros(call.out.shape, np.complex128 if np.iscomplexobj(call.out) else np.float64)
    c.out_w = None if call.out_w is None else np.zeros(call.out_w.shape, np.float64)
    c.rot = rot64
    return c


def _slice_interior(n, shape):
    f = synthetic.slice_fftfreq_norm((n, n), False)
    return np.broadcast_to(np.abs(f ** 2 - 0.25) > 1e-4, shape)


def _grid_interior(n, shape):
    f = synthetic.grid_fftfreq_norm((n, n, n), True)
    return np.broadcast_to(f < 0.5 - 2.0 / n, shape)


def _check(name, call, rot64, interior, bar, scatter=False):
    import gpu_run
    ref64 = _upcast(call, rot64)
    assert FpOracle().run(ref64, THREADS) == 0
    ref32 = clone(call)
    assert FpOracle().run(ref32, THREADS) == 0
    out, out_w = gpu_run.run(clone(call), scatter=scatter)
    pairs = [("values", out, ref32.out, ref64.out)]
    if call.out_w is not None:
        pairs.append(("weights", out_w, ref32.out_w, ref64.out_w))
    lines = []
    for what, dev, r32, r64 in pairs:
        e = {"device all": rel_l2(dev, r64), "f32 path all": rel_l2(r32, r64),
             "device interior": rel_l2(dev[interior], r64[interior]),
             "f32 path interior": rel_l2(r32[interior], r64[interior])}
        lines.append(f"{what}: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
        assert e["device interior"] <= bar, f"{name} {what}: interior rel L2 {e['device interior']:.3e}"
        assert e["device all"] <= 1.1 * e["f32 path all"] + 2 * bar, f"{name} {what}: {e}"
    print(f"\nFP64 {name}: " + "; ".join(lines))


def _extract_call(n, count, seed, interp="linear"):
    q = synthetic.random_quaternions(count, seed=seed)
    rot64 = synthetic.quaternion_to_matrix(q)
    vol = synthetic.make_volume(n, seed=0)
    call = Call(func="extract", remap="hc2h", inp=vol, in_shape=(1, n, n, n),
                out=np.zeros((count, 1, n, n // 2 + 1), np.complex64), out_shape=(count, 1, n, n),
                rot=rot64.astype(np.float32), interp=INTERPS[interp])
    return call, rot64


def _rasterize_call(n, count, seed):
    q = synthetic.random_quaternions(count, seed=seed)
    rot64 = synthetic.quaternion_to_matrix(q)
    sl = synthetic.make_slices(count, n, seed=seed + 1, bfactor=100.0)
    call = Call(func="rasterize", remap="h2hc", inp=sl, in_shape=(count, 1, n, n),
                out=np.zeros((1, n, n, n // 2 + 1), np.complex64), out_shape=(1, n, n, n),
                rot=rot64.astype(np.float32), out_w=np.zeros((1, n, n, n // 2 + 1), np.float32))
    return call, rot64


@pytest.mark.parametrize("n,count", [(64, 64), (256, 256)])
def test_extract_linear_fp64(n, count):
    call, rot64 = _extract_call(n, count, seed=2)
    _check(f"extract_{n}", call, rot64, _slice_interior(n, call.out.shape), 1e-5)


@pytest.mark.parametrize("n,count", [(64, 64), (256, 256)])
def test_rasterize_fp64(n, count):
    call, rot64 = _rasterize_call(n, count, seed=5)
    _check(f"rasterize_{n}", call, rot64, _grid_interior(n, call.out.shape), 1e-4)


@pytest.mark.parametrize("n", [128, 192])
def test_extract_lanczos8_fp64(n):
    call, rot64 = _extract_call(n, 32, seed=7, interp="lanczos8")
    _check(f"lanczos8_{n}", call, rot64, _slice_interior(n, call.out.shape), 1e-5)


@pytest.mark.parametrize("scatter", [False, True], ids=["gather", "scatter"])
def test_insert_windowed_sinc_fp64(scatter):
    n, count = 128, 64
    q = synthetic.random_quaternions(count, seed=11)
    inv64 = np.transpose(synthetic.quaternion_to_matrix(q), (0, 2, 1))
    sl = synthetic.make_slices(count, n, seed=12, bfactor=150.0)
    call = Call(func="insert", remap="h2hc", inp=sl, in_shape=(count, 1, n, n),
                out=np.zeros((1, n, n, n // 2 + 1), np.complex64), out_shape=(1, n, n, n),
                rot=inv64.astype(np.float32), out_w=np.zeros((1, n, n, n // 2 + 1), np.float32),
                sinc=(-1.0, 6.0 / n))
    _check(f"insert_sinc_{n}_{'scatter' if scatter else 'gather'}", call, inv64,
           _grid_interior(n, call.out.shape), 1e-4, scatter)
