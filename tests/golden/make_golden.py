"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own CPU path.

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture (one .npz per case) holds a case description, its seeded inputs and the outputs of
noa's extract/rasterize/insert/insert_and_extract (compiled from the reference sources into
oracle/_ref/libnoa_ref.so, run single-threaded). tests/test_oracle.py checks the C restatement
(oracle/libfp_oracle.so) against these fixtures bit for bit, so the pin holds wherever the reference
sources are absent. The h*_gridding fixtures come from the reference's fourier_interpolation_correction,
built with the one-expression patch that lets its GriddingCorrection compile (oracle/ref_gridding.cpp).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from cases import build, clone, pin_cases, case_id  # noqa: E402
from oracle.oracle import RefLib, ref_gridding_correction  # noqa: E402


def golden_cases() -> list[dict]:
    cases = pin_cases()
    keep = []
    for i, c in enumerate(cases):
        grid_case = c["seed"] < 100 or 200 <= c["seed"] < 201 or 243 <= c["seed"] < 250 or 357 <= c["seed"] < 380 or 480 <= c["seed"] < 490
        # The remap x interp grids: keep one in two; every option case is kept.
        if grid_case and i % 2:
            continue
        keep.append(c)
    return keep


# Gridding correction (fourier_interpolation_correction): shapes with even, odd and size-1 dimensions,
# a batch, and an input broadcast along the batch; f32 and f64, post- and pre-correction.
GRIDDING_CASES = [
    ((1, 16, 16, 16), None, "f32", True), ((1, 16, 16, 16), None, "f64", False),
    ((2, 9, 12, 7), None, "f32", False), ((2, 9, 12, 7), None, "f64", True),
    ((1, 1, 20, 21), None, "f32", True), ((1, 24, 1, 1), None, "f32", False),
    ((3, 10, 8, 6), (1, 10, 8, 6), "f32", True),
]


def write_gridding(ref_gridding) -> int:
    for k, (shape, in_shape, dt, post) in enumerate(GRIDDING_CASES):
        rng = np.random.default_rng(500 + k)
        typ = np.float32 if dt == "f32" else np.float64
        inp = rng.standard_normal(in_shape or shape).astype(typ)
        src = np.broadcast_to(inp, shape) if in_shape else inp
        out = np.zeros(shape, dtype=typ)
        status, err = ref_gridding(np.ascontiguousarray(src) if in_shape is None else src, out, post)
        assert status == 0, err
        meta = json.dumps({"func": "gridding", "shape": list(shape), "dtype": dt, "post": post,
                           "broadcast": in_shape is not None})
        np.savez_compressed(os.path.join(HERE, f"h{k:03d}_gridding.npz"), meta=np.array(meta), inp=inp, out=out)
    return len(GRIDDING_CASES)


def main() -> None:
    ref = RefLib()
    for f in os.listdir(HERE):
        if f.endswith(".npz"):
            os.remove(os.path.join(HERE, f))
    print("wrote", write_gridding(ref_gridding_correction), "gridding fixtures")
    for k, c in enumerate(golden_cases()):
        call = build(c)
        out = clone(call)
        status, err = ref.run(out, 1)
        assert status == 0, (case_id(c), err)
        arrays = {"out": out.out, "out_init": call.out}
        for name in ("inp", "inp_w", "rot", "scale", "rot2", "scale2"):
            v = getattr(call, name)
            if v is not None:
                arrays[name] = v
        if out.out_w is not None:
            arrays["out_w"] = out.out_w
            arrays["out_w_init"] = call.out_w
        meta = json.dumps({k2: (list(v) if isinstance(v, tuple) else v) for k2, v in c.items()})
        np.savez_compressed(os.path.join(HERE, f"g{k:03d}_{c['func']}.npz"), meta=np.array(meta), **arrays)
    print("wrote", len(golden_cases()), "fixtures")


if __name__ == "__main__":
    main()
