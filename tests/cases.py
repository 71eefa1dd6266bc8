"""Parity-case construction shared by the CPU (oracle pinning) and GPU (kernel parity) tests.

A case is a small dict; ``build(case)`` turns it into an ``oracle.Call`` with seeded host inputs.
Sizes are kept small enough for the C oracle (and the reference's CPU path) to finish in seconds.
"""
from __future__ import annotations

import copy
import itertools
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle.oracle import Call, INTERPS  # noqa: E402
from noa_b200 import synthetic  # noqa: E402

_CDT = {"c32": np.complex64, "f32": np.float32, "c64": np.complex128, "f64": np.float64}


def _rfft(shape4):
    b, d, h, w = shape4
    return (b, d, h, w // 2 + 1)


def _values(rng, shape, dt):
    if dt in ("c32", "c64"):
        v = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    else:
        v = rng.standard_normal(shape)
    return v.astype(_CDT[dt])


def _real_dt(dt):
    return np.float64 if dt in ("c64", "f64") else np.float32


def default_case(func: str, **kw) -> dict:
    c = dict(func=func, remap="hc2h", interp="linear", n=32, nslices=6, nout=4,
             in_dt="c32", out_dt="c32", in_w=False, out_w=False, rot="mat33", scale=False,
             cutoff=0.5, target=(0, 0, 0, 0), ews=(0.0, 0.0), sinc=(-1.0, -1.0), w_sinc=(-1.0, -1.0),
             add=False, correct=False, seed=0, slice_n=None, out_n=None)
    c.update(kw)
    return c


def build(case: dict) -> Call:
    """Seeded inputs for one case. Volumes are (1, n, n, n); slices (nslices, 1, slice_n, slice_n)."""
    c = case
    rng = np.random.default_rng(c["seed"])
    n = c["n"]
    sn = c["slice_n"] or n
    f64 = c["out_dt"] in ("c64", "f64")
    rdt = np.float64 if f64 else np.float32
    func = c["func"]
    if func in ("rasterize", "insert"):
        in_shape = (c["nslices"], 1, sn, sn)
        out_shape = (1, n, n, n)
        nrot = c["nslices"]
    elif func == "extract":
        in_shape = (1, n, n, n)
        out_shape = (c["nslices"], 1, sn, sn)
        nrot = c["nslices"]
    else:
        on = c["out_n"] or sn
        in_shape = (c["nslices"], 1, sn, sn)
        out_shape = (c["nout"], 1, on, on)
        nrot = c["nslices"]
    inp = _values(rng, _rfft(in_shape), c["in_dt"])
    out = np.zeros(_rfft(out_shape), dtype=_CDT[c["out_dt"]])
    if func == "insert_extract" and c["add"]:
        out[...] = _values(rng, out.shape, c["out_dt"])
    inp_w = rng.uniform(0.5, 2.0, size=_rfft(in_shape)).astype(rdt) if c["in_w"] else None
    out_w = np.zeros(_rfft(out_shape), dtype=rdt) if c["out_w"] else None
    if out_w is not None and func == "insert_extract" and c["add"]:
        out_w[...] = rng.uniform(0.5, 2.0, size=out_w.shape)
    q = synthetic.random_quaternions(nrot, seed=c["seed"] + 100)
    if c["rot"] == "quat":
        rot = q.astype(rdt)
        rot /= np.linalg.norm(rot, axis=1, keepdims=True)
    else:
        rot = synthetic.quaternion_to_matrix(q).astype(rdt)
    scale = None
    if c["scale"]:
        scale = synthetic.scale_matrices(nrot, (1.0, 1.0), seed=c["seed"] + 200, jitter=0.06).astype(rdt)
    rot2 = scale2 = None
    if func == "insert_extract":
        q2 = synthetic.random_quaternions(c["nout"], seed=c["seed"] + 300)
        rot2 = synthetic.quaternion_to_matrix(q2).astype(rdt)
        if c["rot"] == "quat":
            rot2 = q2.astype(rdt)
            rot2 /= np.linalg.norm(rot2, axis=1, keepdims=True)
        if c["scale"]:
            scale2 = synthetic.scale_matrices(c["nout"], (1.0, 1.0), seed=c["seed"] + 400, jitter=0.06).astype(rdt)
    return Call(func=func, remap=c["remap"], inp=inp, in_shape=in_shape, out=out, out_shape=out_shape,
                rot=rot, inp_w=inp_w, out_w=out_w, scale=scale, rot2=rot2, scale2=scale2,
                interp=INTERPS[c["interp"]], cutoff=c["cutoff"], target=tuple(c["target"]),
                ews=tuple(c["ews"]), sinc=tuple(c["sinc"]), w_sinc=tuple(c["w_sinc"]),
                add_to_output=c["add"], correct_weights=c["correct"])


def clone(call: Call) -> Call:
    c2 = copy.copy(call)
    c2.out = call.out.copy()
    c2.out_w = None if call.out_w is None else call.out_w.copy()
    c2.keep = []
    return c2


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    if den == 0:
        return float(num)
    return float(num / den)


def pin_cases() -> list[dict]:
    """Cases pinning the C restatement against the reference's CPU path (small, broad)."""
    cases = []
    remaps = ["h2h", "h2hc", "hc2h", "hc2hc"]
    # Extract: every remap x interp, weights, quaternions, scale, EWS, w-window, target shape.
    for remap, interp in itertools.product(remaps, INTERPS):
        cases.append(default_case("extract", remap=remap, interp=interp, n=24, nslices=3, seed=len(cases)))
    cases += [
        default_case("extract", out_w=True, seed=101),
        default_case("extract", in_w=True, out_w=True, interp="cubic", seed=102),
        default_case("extract", rot="quat", seed=103),
        default_case("extract", scale=True, seed=104),
        default_case("extract", ews=(50.0, 50.0), seed=105),
        default_case("extract", ews=(-40.0, 60.0), scale=True, seed=106),
        default_case("extract", w_sinc=(-1.0, 0.1), seed=107),
        default_case("extract", w_sinc=(0.05, 0.12), out_w=True, in_w=True, seed=108),
        default_case("extract", target=(1, 40, 40, 40), seed=109),
        default_case("extract", cutoff=0.3, interp="lanczos6", seed=110),
        default_case("extract", in_dt="f32", out_dt="f32", seed=111),
        default_case("extract", in_dt="c32", out_dt="f32", seed=112),
        default_case("extract", in_dt="f32", out_dt="f32", in_w=True, out_w=True, seed=113),
        default_case("extract", n=25, slice_n=25, seed=114),
        default_case("extract", n=32, slice_n=20, seed=115),
    ]
    # Rasterize: every remap, options (cutoff <= 0.5 and even sizes: see the u-bound deviation).
    for remap in remaps:
        cases.append(default_case("rasterize", remap=remap, n=24, nslices=4, seed=200 + len(cases)))
    cases += [
        default_case("rasterize", out_w=True, seed=201),
        default_case("rasterize", in_w=True, out_w=True, seed=202),
        default_case("rasterize", rot="quat", out_w=True, seed=203),
        default_case("rasterize", scale=True, seed=204),
        default_case("rasterize", ews=(60.0, 60.0), seed=205),
        default_case("rasterize", cutoff=0.45, slice_n=20, seed=206),
        default_case("rasterize", target=(1, 36, 36, 36), cutoff=0.4, seed=207),
        default_case("rasterize", in_dt="f32", out_dt="f32", seed=208),
        default_case("rasterize", in_dt="c32", out_dt="f32", seed=209),
        default_case("rasterize", in_dt="f32", out_dt="f32", in_w=True, out_w=True, seed=210),
    ]
    # Insert (gather, windowed-sinc).
    for remap, interp in itertools.product(remaps, ["nearest", "linear", "cubic", "lanczos4"]):
        cases.append(default_case("insert", remap=remap, interp=interp, n=16, nslices=5, seed=300 + len(cases)))
    cases += [
        default_case("insert", n=20, nslices=6, out_w=True, sinc=(-1.0, 0.08), seed=301),
        default_case("insert", n=20, nslices=6, in_w=True, out_w=True, sinc=(0.05, 0.1), seed=302),
        default_case("insert", n=20, nslices=6, rot="quat", seed=303),
        default_case("insert", n=20, nslices=6, scale=True, ews=(45.0, 45.0), seed=304),
        default_case("insert", n=20, nslices=6, target=(1, 24, 24, 24), seed=305),
        default_case("insert", n=16, nslices=5, in_dt="f32", out_dt="f32", in_w=True, out_w=True, seed=306),
        default_case("insert", n=16, nslices=5, in_dt="c32", out_dt="f32", seed=307),
        default_case("insert", n=18, slice_n=22, nslices=5, seed=308),
    ]
    # Insert and extract (virtual volume).
    for remap in remaps:
        cases.append(default_case("insert_extract", remap=remap, n=20, nslices=6, nout=3, sinc=(0.02, 0.06),
                                  seed=400 + len(cases)))
    cases += [
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), out_w=True, seed=401),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), in_w=True, out_w=True,
                     interp="lanczos6", seed=402),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), correct=True, seed=403),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), add=True, out_w=True,
                     seed=404),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), w_sinc=(-1.0, 0.15),
                     seed=405),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), rot="quat", scale=True,
                     ews=(30.0, 30.0), cutoff=0.8, seed=406),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), in_dt="f32", out_dt="f32",
                     seed=407),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), in_dt="c32", out_dt="f32",
                     seed=408),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), w_sinc=(0.05, 0.1),
                     add=True, out_w=True, in_w=True, seed=409),
    ]
    # FP64 (the reference instantiated in double) on a few representative calls.
    cases += [
        default_case("extract", in_dt="c64", out_dt="c64", out_w=True, seed=501),
        default_case("rasterize", in_dt="c64", out_dt="c64", out_w=True, seed=502),
        default_case("insert", n=16, nslices=5, in_dt="c64", out_dt="c64", out_w=True, seed=503),
        default_case("insert_extract", n=20, nslices=6, nout=3, sinc=(0.02, 0.06), in_dt="c64", out_dt="c64",
                     seed=504),
    ]
    return cases


def case_id(case: dict) -> str:
    d = default_case(case["func"])
    parts = [case["func"]] + [f"{k}={v}" for k, v in case.items() if k != "func" and d.get(k) != v and k != "seed"]
    return ",".join(str(p) for p in parts) + f",s{case['seed']}"
