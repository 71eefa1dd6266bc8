"""Runs an oracle.Call description on the GPU through noa_b200's C ABI (tests only)."""
from __future__ import annotations

import numpy as np
import torch

from noa_b200 import fourier_project as fp
from oracle.oracle import Call

_INTERP_NAMES = {v: k for k, v in fp.INTERPS.items()}


def _dev(a):
    if a is None:
        return None
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _xform(a):
    if a is None:
        return None
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run(call: Call, stream=None, scatter=False):
    """Copies the call's inputs to the device, runs the CUDA path, returns (out, out_w) as numpy.
    ``scatter``: insertions run the slice-major scatter form instead of the gather form."""
    inp = call.inp_value if call.inp_value is not None else _dev(call.inp)
    inp_w = _dev(call.inp_w)
    out = _dev(call.out)
    out_w = _dev(call.out_w)
    rot, scale = _xform(call.rot), _xform(call.scale)
    interp = _INTERP_NAMES[call.interp]
    ws = fp.WindowedSinc(*call.sinc)
    wws = fp.WindowedSinc(*call.w_sinc)
    target = call.target if any(call.target) else None
    if call.func == "rasterize":
        fp.rasterize_central_slices_3d(call.remap, inp, inp_w, call.in_shape, out, out_w, call.out_shape,
                                       scale, rot, fftfreq_cutoff=call.cutoff, target_shape=target,
                                       ews_radius=call.ews, stream=stream)
    elif call.func == "insert":
        f = fp.insert_central_slices_3d_scatter if scatter else fp.insert_central_slices_3d
        f(call.remap, inp, inp_w, call.in_shape, out, out_w, call.out_shape, scale, rot, interp=interp,
          windowed_sinc=ws, fftfreq_cutoff=call.cutoff, target_shape=target, ews_radius=call.ews, stream=stream)
    elif call.func == "extract":
        fp.extract_central_slices_3d(call.remap, inp, inp_w, call.in_shape, out, out_w, call.out_shape,
                                     scale, rot, interp=interp, w_windowed_sinc=wws, fftfreq_cutoff=call.cutoff,
                                     target_shape=target, ews_radius=call.ews, stream=stream)
    else:
        fp.insert_and_extract_central_slices_3d(
            call.remap, inp, inp_w, call.in_shape, out, out_w, call.out_shape,
            scale, rot, _xform(call.scale2), _xform(call.rot2), interp=interp, input_windowed_sinc=ws,
            w_windowed_sinc=wws, add_to_output=call.add_to_output, correct_weights=call.correct_weights,
            fftfreq_cutoff=call.cutoff, ews_radius=call.ews, stream=stream)
    torch.cuda.synchronize()
    return out.cpu().numpy(), (None if out_w is None else out_w.cpu().numpy())
