"""Pyramid-level geometry (b200bsp_resample_geometry) against the
reference's: host code of the library, no device needed.  Exact equality:
the grid is computed in the reference's arithmetic."""
import os

import numpy as np
import pytest

import plastimatch_b200 as P
from conftest import GOLDEN, golden_names
from plastimatch_b200.geometry import Volume


def load_resample(name):
    r = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    v = Volume(r["img"], origin=tuple(float(x) for x in r["origin"]),
               spacing=tuple(float(x) for x in r["spacing"]))
    return v, str(r["mode"]), tuple(float(x) for x in r["rate"]), r


@pytest.mark.parametrize("name", golden_names("resample"))
def test_geometry_matches_reference(name):
    v, mode, rate, rec = load_resample(name)
    dim, origin, spacing, copy = P.resample_geometry(v, mode, rate)
    assert not copy
    assert dim == tuple(int(x) for x in rec["out_dim"])
    np.testing.assert_array_equal(np.float32(origin), rec["out_origin"])
    np.testing.assert_array_equal(np.float32(spacing), rec["out_spacing"])


def test_unit_voxel_rate_is_a_copy_and_bad_arguments_fail():
    v, _, _, _ = load_resample(golden_names("resample")[0])
    for mode in ("voxel", "voxel_legacy"):
        dim, origin, spacing, copy = P.resample_geometry(v, mode, (1, 1, 1))
        assert copy and dim == v.dim
    # a unit rate in mm or percent still resamples
    assert not P.resample_geometry(v, "percent", (1, 1, 1))[3]
    with pytest.raises(P.B200Error):
        P.resample_geometry(v, "voxel", (0, 1, 1))
