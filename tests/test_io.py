"""B-spline coefficient files and MetaImage files against the reference's
own writers and readers (host code, no device needed).

The bar is exact: files written by this library are byte-identical to the
reference's, and what either side reads back is bit-identical.
"""
import numpy as np
import pytest

import oracle as O
import plastimatch_b200 as P
from conftest import golden_names, load_golden
from plastimatch_b200 import synth
from plastimatch_b200.geometry import Volume

needs_ref = pytest.mark.skipif(not O.ref_available(),
                               reason="reference build absent")

CASES = ["mse_small", "mse_dcos", "mse_roi"]


@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_xform_file_matches_reference(tmp_path, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    ours, theirs = tmp_path / "ours.txt", tmp_path / "ref.txt"
    P.xform_save(ours, fixed, grid, coeff)
    O.ref_xform_save(theirs, grid, fixed, coeff)
    assert ours.read_bytes() == theirs.read_bytes()
    # the reference reads our file back exactly
    g, gr, c = O.ref_xform_load(ours)
    np.testing.assert_array_equal(c, coeff)
    assert tuple(gr.roi_offset) == grid.roi_offset
    assert tuple(gr.vox_per_rgn) == grid.vox_per_rgn
    # and we read the reference's file exactly
    geom, grid2, c2 = P.xform_load(theirs)
    np.testing.assert_array_equal(c2, coeff)
    assert grid2.roi_dim == grid.roi_dim and grid2.cdims == grid.cdims
    assert geom["dim"] == fixed.dim
    np.testing.assert_array_equal(np.float32(geom["dcos"]), np.float32(g.dcos))
    np.testing.assert_array_equal(np.float32(geom["origin"]),
                                  np.float32(g.origin))


def test_xform_load_rejects_bad_files(tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("not a transform\n")
    with pytest.raises(P.B200Error) as e:
        P.xform_load(bad)
    assert e.value.code == -7
    fixed, moving, grid, coeff, rec = load_golden("mse_small")
    good = tmp_path / "good.txt"
    P.xform_save(good, fixed, grid, coeff)
    lines = good.read_text().splitlines()
    (tmp_path / "short.txt").write_text("\n".join(lines[:-5]) + "\n")
    with pytest.raises(P.B200Error):
        P.xform_load(tmp_path / "short.txt")
    with pytest.raises(P.B200Error):
        P.xform_load(tmp_path / "missing.txt")


@needs_ref
@pytest.mark.parametrize("name", ["mse_small", "mse_dcos"])
def test_mha_float_and_field_match_reference(tmp_path, name):
    fixed, moving, grid, coeff, rec = load_golden(name)
    vf = O.port_interpolate_vf(grid, fixed, coeff)
    for data in (None, vf):
        ours, theirs = tmp_path / "ours.mha", tmp_path / "ref.mha"
        P.mha_write(ours, fixed, vf=data)
        O.ref_write_mha(theirs, fixed, vf=data)
        assert ours.read_bytes() == theirs.read_bytes()
        g, ch, d = O.ref_read_mha(ours)
        want = fixed.img if data is None else data
        assert ch == (1 if data is None else 3)
        np.testing.assert_array_equal(d, want.ravel())
        back = P.mha_read(theirs)
        if data is None:
            np.testing.assert_array_equal(back.img, fixed.img)
            assert back.dim == fixed.dim
            np.testing.assert_array_equal(np.float32(back.dcos),
                                          np.float32(g.dcos))
        else:
            np.testing.assert_array_equal(back[0], data)


def _raw_mha(path, dim, etype, data: bytes, msb=False, channels=None):
    hdr = ("ObjectType = Image\nNDims = 3\nBinaryData = True\n"
           f"BinaryDataByteOrderMSB = {'True' if msb else 'False'}\n"
           "TransformMatrix = 1 0 0 0 1 0 0 0 1\nOffset = -2.5 3 4.25\n"
           "ElementSpacing = 0.8 1.25 2\n"
           f"DimSize = {dim[0]} {dim[1]} {dim[2]}\n"
           + (f"ElementNumberOfChannels = {channels}\n" if channels else "")
           + f"ElementType = {etype}\nElementDataFile = LOCAL\n")
    path.write_bytes(hdr.encode() + data)


@needs_ref
@pytest.mark.parametrize("etype,dtype", [("MET_SHORT", "<i2"),
                                         ("MET_UCHAR", "u1"),
                                         ("MET_FLOAT", "<f4")])
@pytest.mark.parametrize("msb", [False, True])
def test_mha_read_types_and_byte_order(tmp_path, etype, dtype, msb):
    rng = np.random.default_rng(5)
    dim = (7, 5, 3)
    vals = rng.integers(0, 200, size=dim[::-1]).astype(np.float32)
    if etype == "MET_SHORT":
        vals -= 100
    arr = vals.astype(dtype)
    if msb:
        arr = arr.astype(np.dtype(dtype).newbyteorder(">"))
    p = tmp_path / "x.mha"
    _raw_mha(p, dim, etype, arr.tobytes(), msb=msb)
    v = P.mha_read(p)
    np.testing.assert_array_equal(v.img, vals)
    g, ch, d = O.ref_read_mha(p)
    np.testing.assert_array_equal(d.reshape(vals.shape), vals)
    assert v.origin == (-2.5, 3.0, 4.25)
    np.testing.assert_array_equal(np.float32(v.spacing),
                                  np.float32((0.8, 1.25, 2.0)))


def test_mha_roundtrip_through_the_library(tmp_path):
    v = synth.gaussian_blobs((11, 9, 6), spacing=(0.7, 1.3, 2.1), seed=4)
    v = Volume(v.img, origin=(1.5, -2.0, 3.25), spacing=v.spacing,
               dcos=(0.0, 1.0, 0.0, -1.0, 0.0, 0.0, 0.0, 0.0, 1.0))
    P.mha_write(tmp_path / "v.mha", v)
    w = P.mha_read(tmp_path / "v.mha")
    np.testing.assert_array_equal(w.img, v.img)
    assert w.dcos == v.dcos and w.dim == v.dim
