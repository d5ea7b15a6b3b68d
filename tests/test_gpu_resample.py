"""Pyramid resampling on the GPU (b200bsp_resample) against the reference's
volume_resample_float_li output: bit-identical (the device forms the
reference's per-axis float arithmetic and its LI_VALUE sum order)."""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import golden_names
from test_resample import load_resample

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names("resample"))
def test_pyramid_level_matches_reference(name):
    v, mode, rate, rec = load_resample(name)
    out = P.pyramid_level(v, mode, rate)
    np.testing.assert_array_equal(out.img, rec["out"])


def test_grid_beyond_the_input_and_device_buffers():
    torch = pytest.importorskip("torch")
    v, _, _, _ = load_resample(golden_names("resample")[0])
    # an output box larger than the input: outside voxels are 0
    dim, origin, spacing = (30, 27, 15), (-20.0, 0.5, 2.0), (1.7, 1.5, 4.0)
    ref = np.zeros(dim[0] * dim[1] * dim[2], np.float32)
    import ctypes as C
    O.port().orc_resample_li(
        (C.c_int64 * 3)(*v.dim), (C.c_float * 3)(*v.origin),
        (C.c_float * 3)(*v.spacing), C.c_void_p(v.img.ctypes.data),
        (C.c_int64 * 3)(*dim), (C.c_float * 3)(*origin),
        (C.c_float * 3)(*spacing), C.c_void_p(ref.ctypes.data))
    out = P.resample(v, dim, origin, spacing)
    np.testing.assert_array_equal(out.img.ravel(), ref)
    assert (ref == 0).any() and (ref != 0).any()
    d_in = torch.from_numpy(v.img).cuda()
    d_out = torch.zeros(ref.size, device="cuda")
    P._check(P.lib().b200bsp_resample(
        C.byref(P._vol_desc(v)), d_in.data_ptr(),
        C.byref(P.VolumeDesc((C.c_int64 * 3)(*dim), (C.c_float * 3)(*origin),
                             (C.c_float * 3)(*spacing),
                             (C.c_float * 9)(*v.dcos))),
        d_out.data_ptr(), 0))
    np.testing.assert_array_equal(d_out.cpu().numpy(), ref)
