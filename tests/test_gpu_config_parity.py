"""GPU parity at the measured workloads' own sizes, through the C ABI, against the f32 oracle (the C
restatement pinned bit-exactly to noa's CPU path).

The parity suites in test_gpu_parity.py and test_gpu_random.py run small volumes; these run the
sizes the benchmark numbers are quoted on, where the 32-bit offset paths, the pair copy, the padded
accumulator and the launch shapes meet full-size inputs:

  extract 256^3, 4096 slices of 256x129, LINEAR, hc2h, cutoff 0.5                      <= 1e-5
  rasterize 4096 slices of 256x129 (B = 100 envelope) into 256^3 + f32 weights, h2hc   <= 1e-4
  LANCZOS8 extraction of 32 slices from boxes 256 and 384, per call and batched        <= 1e-5
  windowed-sinc insertion (half-width 6 voxels) into 512^3 + weights, hc2hc, a 16-slice subset,
      gather form <= 1e-5, scatter form (atomic sum order) <= 1e-4

Tolerances are relative L2 over the whole output. Inputs are seeded and synthetic, generated as the
benchmark generates them.
"""
import os

import numpy as np
import pytest

from cases import clone
from noa_b200 import synthetic
from oracle.oracle import Call, FpOracle, INTERPS

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def rel_l2(a: np.ndarray, b: np.ndarray, chunk: int = 1 << 24) -> float:
    """Relative L2 of a against b, accumulated in float64 over chunks (outputs here reach 1 GB)."""
    a, b = a.reshape(-1), b.reshape(-1)
    num = den = 0.0
    for i in range(0, a.size, chunk):
        x = a[i:i + chunk].astype(np.complex128 if np.iscomplexobj(a) else np.float64)
        y = b[i:i + chunk].astype(x.dtype)
        num += float(np.sum(np.abs(x - y) ** 2))
        den += float(np.sum(np.abs(y) ** 2))
    return float(np.sqrt(num / den)) if den > 0 else float(np.sqrt(num))


def _oracle(call: Call) -> Call:
    ref = clone(call)
    assert FpOracle().run(ref, THREADS) == 0
    return ref


def test_extract_256_4096_slices():
    import gpu_run
    n, b = 256, 4096
    call = Call(func="extract", remap="hc2h", inp=synthetic.make_volume(n, seed=0), in_shape=(1, n, n, n),
                out=np.zeros((b, 1, n, n // 2 + 1), np.complex64), out_shape=(b, 1, n, n),
                rot=synthetic.random_rotations(b, seed=2), cutoff=0.5)
    ref = _oracle(call)
    out, _ = gpu_run.run(clone(call))
    err = rel_l2(out, ref.out)
    print(f"\nextract 256^3 x 4096: rel L2 {err:.3e}")
    assert err <= 1e-5


def test_rasterize_256_4096_slices_with_weights():
    import gpu_run
    n, b = 256, 4096
    call = Call(func="rasterize", remap="h2hc", inp=synthetic.make_slices(b, n, seed=1, bfactor=100.0),
                in_shape=(b, 1, n, n), out=np.zeros((1, n, n, n // 2 + 1), np.complex64), out_shape=(1, n, n, n),
                rot=synthetic.random_rotations(b, seed=3), out_w=np.zeros((1, n, n, n // 2 + 1), np.float32),
                cutoff=0.5)
    ref = _oracle(call)
    out, out_w = gpu_run.run(clone(call))
    ev, ew = rel_l2(out, ref.out), rel_l2(out_w, ref.out_w)
    print(f"\nrasterize 256^3 x 4096: rel L2 values {ev:.3e}, weights {ew:.3e}")
    assert ev <= 1e-4 and ew <= 1e-4


@pytest.mark.parametrize("n", [256, 384])
def test_lanczos8_extract_per_call_and_batched(n):
    import torch
    import gpu_run
    from noa_b200 import batch
    b = 32
    vol = synthetic.make_volume(n, seed=n)
    rot = synthetic.random_rotations(b, seed=n + 1)
    call = Call(func="extract", remap="hc2h", inp=vol, in_shape=(1, n, n, n),
                out=np.zeros((b, 1, n, n // 2 + 1), np.complex64), out_shape=(b, 1, n, n), rot=rot,
                interp=INTERPS["lanczos8"], cutoff=0.5)
    ref = _oracle(call)
    out, _ = gpu_run.run(clone(call))
    err = rel_l2(out, ref.out)

    # The same extraction as one request of a batched launch, beside a second request of another box.
    vt = torch.from_numpy(vol).cuda()
    rt = torch.from_numpy(rot).cuda()
    m = 128
    other = torch.from_numpy(synthetic.make_volume(m, seed=5)).cuda()
    o1 = torch.zeros((b, 1, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    o2 = torch.zeros((7, 1, m, m // 2 + 1), dtype=torch.complex64, device="cuda")
    reqs = [batch.ExtractRequest(volume=vt, volume_shape=(1, n, n, n), slice=o1, slice_shape=(b, 1, n, n),
                                 fwd_rotation=rt),
            batch.ExtractRequest(volume=other, volume_shape=(1, m, m, m), slice=o2, slice_shape=(7, 1, m, m),
                                 fwd_rotation=torch.from_numpy(synthetic.random_rotations(7, seed=6)).cuda())]
    batch.extract_batch_launch("hc2h", reqs, interp="lanczos8")
    torch.cuda.synchronize()
    errb = rel_l2(o1.cpu().numpy(), ref.out)
    print(f"\nLANCZOS8 {n}^3 x {b}: rel L2 per call {err:.3e}, batched {errb:.3e}")
    assert err <= 1e-5 and errb <= 1e-5


@pytest.mark.parametrize("scatter", [False, True], ids=["gather", "scatter"])
def test_windowed_sinc_insert_512_subset(scatter):
    import gpu_run
    n, b = 512, 16
    wp = n // 2 + 1
    # 16 slices generated as the 512^3 x 20,000 workload's are (B = 150, centered slices).
    q = synthetic.random_quaternions(b, seed=16)
    inv = np.ascontiguousarray(np.transpose(synthetic.quaternion_to_matrix(q), (0, 2, 1))).astype(np.float32)
    call = Call(func="insert", remap="hc2hc", inp=synthetic.make_slices(b, n, seed=15, bfactor=150.0, centered=True),
                in_shape=(b, 1, n, n), out=np.zeros((1, n, n, wp), np.complex64), out_shape=(1, n, n, n),
                rot=inv, out_w=np.zeros((1, n, n, wp), np.float32), interp=INTERPS["linear"], cutoff=0.5,
                sinc=(-1.0, 6.0 / n))
    ref = _oracle(call)
    out, out_w = gpu_run.run(clone(call), scatter=scatter)
    ev, ew = rel_l2(out, ref.out), rel_l2(out_w, ref.out_w)
    tol = 1e-4 if scatter else 1e-5
    print(f"\ninsert 512^3 x {b} ({'scatter' if scatter else 'gather'}): rel L2 values {ev:.3e}, weights {ew:.3e}")
    assert ev <= tol and ew <= tol
