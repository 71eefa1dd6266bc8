"""Seeded random parity cases: GPU (C ABI) against the oracle over the option space — every function,
remap and interpolation, odd and even sizes, complex and real data, weights in and out, Mat33 or quaternion rotations,
scaling, EWS, target shapes, cutoffs — beyond the hand-picked cases of test_gpu_parity.py. Insertions also run the scatter form.

Tolerances as in test_gpu_parity: relative L2 <= 1e-5 (1e-4 for rasterization).
"""
import numpy as np
import pytest

from cases import build, case_id, clone, default_case, rel_l2
from oracle.oracle import FpOracle, INTERPS

pytestmark = pytest.mark.gpu

TOL = {"extract": 1e-5, "insert": 1e-5, "insert_extract": 1e-5, "rasterize": 1e-4}
REMAPS = ["h2h", "h2hc", "hc2h", "hc2hc"]


def _random_case(i: int) -> dict:
    rng = np.random.default_rng(10_000 + i)
    func = ["extract", "rasterize", "insert", "insert_extract"][i % 4]
    n = int(rng.choice([16, 17, 20, 24, 25]))
    c = dict(remap=str(rng.choice(REMAPS)), n=n, nslices=int(rng.integers(1, 7)), seed=20_000 + i,
             rot=str(rng.choice(["mat33", "quat"])), scale=bool(rng.random() < 0.3),
             cutoff=float(rng.choice([0.5, 0.45, 0.35])), in_w=bool(rng.random() < 0.3),
             out_w=bool(rng.random() < 0.6))
    c["in_dt"], c["out_dt"] = [("c32", "c32"), ("c32", "c32"), ("c32", "f32"), ("f32", "f32")][int(rng.integers(4))]
    if func != "rasterize":
        c["interp"] = str(rng.choice(list(INTERPS)))
    if rng.random() < 0.25:
        c["ews"] = (float(rng.uniform(30, 80)), float(rng.uniform(30, 80)))
    if func == "extract":
        if rng.random() < 0.3:
            t = int(rng.choice([n + 4, n + 8]))
            c["target"] = (1, t, t, t)
        if rng.random() < 0.3:
            c["slice_n"] = int(rng.choice([n - 2, n + 3]))
    if func == "rasterize":
        c["n"] = c["n"] + (c["n"] % 2)  # the u-bound deviation: even sizes, cutoff <= 0.5
    if func == "insert":
        c["sinc"] = (float(rng.choice([-1.0, 0.04])), float(rng.uniform(0.06, 0.15)))
    if func == "insert_extract":
        c["nout"] = int(rng.integers(1, 4))
        c["sinc"] = (0.02, float(rng.uniform(0.05, 0.1)))
        c["add"] = bool(rng.random() < 0.3)
        c["correct"] = (not c["add"]) and bool(rng.random() < 0.3)
    return default_case(func, **c)


CASES = [_random_case(i) for i in range(48)]


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_random_case_matches_oracle(case):
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
    if case["func"] == "insert":
        out, out_w = gpu_run.run(clone(call), scatter=True)
        err = rel_l2(out, ref.out)
        assert err <= tol, f"scatter form: rel L2 {err:.3e} > {tol:g}"
        if ref.out_w is not None:
            assert rel_l2(out_w, ref.out_w) <= tol
