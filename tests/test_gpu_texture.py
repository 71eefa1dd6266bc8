"""GPU: a noa Texture<c32> passes through the reference-side binding (include/noa_b200/noa_binding.hpp).

noa's own CUDA backend (compiled from the reference sources into oracle/_ref/libnoa_ref_cuda.so) builds
the texture the way noa's users do (xform/Texture.hpp:63-170: a CUDA array and a texture object); the
binding stages the CUDA array into linear memory on the call's stream and takes the interpolation
method from the texture (FourierProject.hpp:1203-1217), then calls nb_extract_central_slices_3d. The
result must equal, bit for bit, the same call on the plain device array the texture was made from, and
the oracle within the extraction bar (1e-5).
"""
import numpy as np
import pytest

from cases import rel_l2
from noa_b200 import synthetic
from oracle.oracle import Call, FpOracle, ref_cuda_available, ref_texture_extract

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_cuda_available(), reason="noa CUDA backend not built (make -C oracle ref-cuda)")]


@pytest.mark.parametrize("interp", [1, 0, 2], ids=["linear", "nearest", "cubic"])
def test_texture_input_through_the_binding(interp):
    import noa_b200.fourier_project as fp
    fp.lib()  # the binding calls this library; load it from its in-tree path first
    n, count = 32, 12
    vol = synthetic.make_volume(n, seed=81)
    rot = synthetic.random_rotations(count, seed=82)
    from_texture, from_array = ref_texture_extract(vol, rot, interp)
    np.testing.assert_array_equal(from_texture, from_array)
    call = Call(func="extract", remap="hc2h", inp=vol, in_shape=(1, n, n, n),
                out=np.zeros((count, 1, n, n // 2 + 1), np.complex64), out_shape=(count, 1, n, n), rot=rot,
                interp=interp)
    FpOracle().run(call, 4)
    assert np.abs(from_array).sum() > 0
    assert rel_l2(from_texture, call.out) <= 1e-5
