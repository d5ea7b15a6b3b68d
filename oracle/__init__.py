"""The oracle: CPU checkers for the B-spline cost function.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference arm may import this package; the
product (plastimatch_b200) never does.

Two checkers live here:

* ``port``  -- oracle/liborc.so, the plain-C restatement of the reference
  (oracle/bspline_oracle.c): float routines in the reference's operation
  order plus double-precision versions used as the error yardstick.
* ``ref``   -- oracle/_ref/libplmref.so, the reference's own C++ flavours
  compiled from its sources by oracle/build_ref.sh (present when the
  reference tree was available at build time).

Inputs are plastimatch_b200.geometry.Volume / BsplineGrid objects.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liborc.so")
REF_SO = os.path.join(HERE, "_ref", "libplmref.so")

f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i64p = C.POINTER(C.c_int64)


def _p(a, t=f32p):
    return a.ctypes.data_as(t) if a is not None else None


class OrcVol(C.Structure):
    _fields_ = [("dim", C.c_int64 * 3), ("origin", C.c_float * 3),
                ("spacing", C.c_float * 3), ("dcos", C.c_float * 9),
                ("inv_dcos", C.c_float * 9), ("step", C.c_float * 9),
                ("proj", C.c_float * 9)]


class OrcGrid(C.Structure):
    _fields_ = [("img_origin", C.c_float * 3), ("img_spacing", C.c_float * 3),
                ("img_dim", C.c_int64 * 3), ("roi_offset", C.c_int64 * 3),
                ("roi_dim", C.c_int64 * 3), ("vox_per_rgn", C.c_int64 * 3),
                ("grid_spac", C.c_float * 3), ("rdims", C.c_int64 * 3),
                ("cdims", C.c_int64 * 3), ("num_knots", C.c_int64),
                ("num_coeff", C.c_int64)]


class OrcHist(C.Structure):
    _fields_ = [("bins", C.c_int64), ("offset", C.c_float),
                ("delta", C.c_float), ("keys", C.c_int64),
                ("key_lut", C.POINTER(C.c_int32))]


class OrcParzen(C.Structure):
    _fields_ = [("bins", C.c_int64), ("f_min", C.c_float),
                ("f_delta", C.c_float), ("m_min", C.c_float),
                ("m_delta", C.c_float)]


class RefGeom(C.Structure):
    _fields_ = [("dim", C.c_int64 * 3), ("origin", C.c_float * 3),
                ("spacing", C.c_float * 3), ("dcos", C.c_float * 9)]


class RefGrid(C.Structure):
    _fields_ = [("roi_offset", C.c_int64 * 3), ("roi_dim", C.c_int64 * 3),
                ("vox_per_rgn", C.c_int64 * 3)]


class RefResult(C.Structure):
    _fields_ = [("score", C.c_float), ("total_score", C.c_float),
                ("rmetric", C.c_float), ("num_vox", C.c_int64),
                ("num_coeff", C.c_int64), ("fixed_bins", C.c_int64),
                ("moving_bins", C.c_int64), ("f_offset", C.c_float),
                ("f_delta", C.c_float), ("m_offset", C.c_float),
                ("m_delta", C.c_float)]


@dataclass
class Result:
    score: float
    grad: np.ndarray
    num_vox: int = 0
    f_hist: np.ndarray | None = None
    m_hist: np.ndarray | None = None
    j_hist: np.ndarray | None = None


_port = None
_ref = None


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            raise RuntimeError("oracle/liborc.so not built (make -C oracle)")
        _port = C.CDLL(PORT_SO)
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("oracle/_ref/libplmref.so not built "
                               "(oracle/build_ref.sh)")
        _ref = C.CDLL(REF_SO)
    return _ref


# ---------------------------------------------------------------- port ---

class OrcRoi(C.Structure):
    _fields_ = [("vol", OrcVol), ("mask", C.POINTER(C.c_uint8))]


class _RoiScope:
    """orc_set_roi for the duration of one oracle call (ROIs are
    plastimatch_b200.geometry.Roi or None)."""

    def __init__(self, fixed_roi, moving_roi):
        self.keep = []
        self.f = self._mk(fixed_roi)
        self.m = self._mk(moving_roi)

    def _mk(self, roi):
        if roi is None:
            return None
        r = OrcRoi()
        r.vol = orc_vol(roi)
        r.mask = roi.mask.ctypes.data_as(C.POINTER(C.c_uint8))
        self.keep.append(roi.mask)
        return r

    def __enter__(self):
        port().orc_set_roi(C.byref(self.f) if self.f else None,
                           C.byref(self.m) if self.m else None)
        return self

    def __exit__(self, *a):
        port().orc_set_roi(None, None)


def orc_vol(v) -> OrcVol:
    o = OrcVol()
    d = (C.c_int64 * 3)(*v.dim)
    org = (C.c_float * 3)(*v.origin)
    sp = (C.c_float * 3)(*v.spacing)
    dc = (C.c_float * 9)(*v.dcos)
    if port().orc_vol_init(C.byref(o), d, org, sp, dc) != 0:
        raise ValueError("singular direction cosines")
    return o


def orc_grid(grid, fixed) -> OrcGrid:
    g = OrcGrid()
    rc = port().orc_grid_init(C.byref(g), C.byref(orc_vol(fixed)),
                              (C.c_int64 * 3)(*grid.roi_offset),
                              (C.c_int64 * 3)(*grid.roi_dim),
                              (C.c_int64 * 3)(*grid.vox_per_rgn))
    if rc:
        raise ValueError("bad grid")
    return g


def port_volume_grad(v) -> np.ndarray:
    out = np.zeros(v.npix * 3, np.float32)
    port().orc_volume_grad(C.byref(orc_vol(v)), _p(v.img), _p(out))
    return out


def port_basis_lut(vpr: int) -> np.ndarray:
    out = np.zeros(4 * vpr, np.float32)
    port().orc_basis_lut(_p(out), C.c_int64(vpr))
    return out


def port_mse(grid, fixed, moving, coeff, moving_grad=None, grad_mode=0,
             precision="f32", fixed_roi=None, moving_roi=None) -> Result:
    """MSE flavour g (nearest-voxel gradient, grad_mode 0) or o (trilinear
    derivative, 1) in float, or both in double; with image ROIs, flavour
    i's ROI tests."""
    if fixed_roi is not None or moving_roi is not None:
        with _RoiScope(fixed_roi, moving_roi):
            return port_mse(grid, fixed, moving, coeff, moving_grad,
                            grad_mode, precision)
    if moving_grad is None and grad_mode == 0:
        moving_grad = port_volume_grad(moving)
    g = orc_grid(grid, fixed)
    nv = C.c_int64(0)
    coeff = np.ascontiguousarray(coeff, np.float32)
    if precision == "f32":
        s = C.c_float(0)
        gr = np.zeros(grid.num_coeff, np.float32)
        rc = port().orc_mse_f32(C.byref(g), C.byref(orc_vol(fixed)),
                                _p(fixed.img), C.byref(orc_vol(moving)),
                                _p(moving.img), _p(moving_grad), _p(coeff),
                                C.c_int(grad_mode), C.byref(s), _p(gr),
                                C.byref(nv))
    else:
        s = C.c_double(0)
        gr = np.zeros(grid.num_coeff, np.float64)
        rc = port().orc_mse_f64(C.byref(g), C.byref(orc_vol(fixed)),
                                _p(fixed.img), C.byref(orc_vol(moving)),
                                _p(moving.img), _p(moving_grad), _p(coeff),
                                C.c_int(grad_mode), C.byref(s), _p(gr, f64p),
                                C.byref(nv))
    if rc:
        raise RuntimeError(f"oracle mse failed rc={rc}")
    return Result(s.value, gr, nv.value)


def port_hist_eqsp(img: np.ndarray, bins: int) -> OrcHist:
    h = OrcHist(bins, 0.0, 0.0)
    a = np.ascontiguousarray(img, np.float32).ravel()
    port().orc_hist_eqsp(C.byref(h), _p(a), C.c_int64(a.size))
    return h


def port_hist_vopt(img: np.ndarray, bins: int) -> OrcHist:
    """V-optimal histogram parameters; the key table lives on the returned
    object (h._lut) for as long as it does."""
    h = OrcHist(bins, 0.0, 0.0)
    lut = np.zeros(1000, np.int32)
    a = np.ascontiguousarray(img, np.float32).ravel()
    port().orc_hist_vopt(C.byref(h), lut.ctypes.data_as(C.POINTER(C.c_int32)),
                         _p(a), C.c_int64(a.size))
    h._lut = lut
    return h


def port_hist(img, bins, hist="eqsp"):
    return port_hist_vopt(img, bins) if hist == "vopt" else \
        port_hist_eqsp(img, bins)


def port_mi(grid, fixed, moving, coeff, bins=32, precision="f32",
            fixed_roi=None, moving_roi=None, hist="eqsp") -> Result:
    """Mattes MI flavour g (PVI-8) in float or double; with image ROIs,
    flavour h's ROI tests in both passes; hist "eqsp" (equal-spacing bins)
    or "vopt" (V-optimal bins)."""
    if fixed_roi is not None or moving_roi is not None:
        with _RoiScope(fixed_roi, moving_roi):
            return port_mi(grid, fixed, moving, coeff, bins, precision,
                           hist=hist)
    g = orc_grid(grid, fixed)
    fh, mh = port_hist(fixed.img, bins, hist), port_hist(moving.img, bins, hist)
    nv = C.c_int64(0)
    f_hist = np.zeros(bins)
    m_hist = np.zeros(bins)
    j_hist = np.zeros(bins * bins)
    coeff = np.ascontiguousarray(coeff, np.float32)
    if precision == "f32":
        s = C.c_float(0)
        gr = np.zeros(grid.num_coeff, np.float32)
        fn, gp = port().orc_mi_f32, _p(gr)
    else:
        s = C.c_double(0)
        gr = np.zeros(grid.num_coeff, np.float64)
        fn, gp = port().orc_mi_f64, _p(gr, f64p)
    rc = fn(C.byref(g), C.byref(orc_vol(fixed)), _p(fixed.img),
            C.byref(orc_vol(moving)), _p(moving.img), _p(coeff),
            C.byref(fh), C.byref(mh), C.byref(s), gp, C.byref(nv),
            _p(f_hist, f64p), _p(m_hist, f64p), _p(j_hist, f64p))
    if rc:
        raise RuntimeError(f"oracle mi failed rc={rc}")
    return Result(s.value, gr, nv.value, f_hist, m_hist,
                  j_hist.reshape(bins, bins))


def port_mi_pass1(grid, fixed, moving, coeff, bins=32):
    """PVI-8 pass 1 over the grid's ROI in double: (f, m, j, num_vox)."""
    g = orc_grid(grid, fixed)
    fh, mh = port_hist_eqsp(fixed.img, bins), port_hist_eqsp(moving.img, bins)
    nv = C.c_int64(0)
    f, m, j = np.zeros(bins), np.zeros(bins), np.zeros(bins * bins)
    rc = port().orc_mi_f64_pass1(
        C.byref(g), C.byref(orc_vol(fixed)), _p(fixed.img),
        C.byref(orc_vol(moving)), _p(moving.img),
        _p(np.ascontiguousarray(coeff, np.float32)), C.byref(fh), C.byref(mh),
        C.byref(nv), _p(f, f64p), _p(m, f64p), _p(j, f64p))
    if rc:
        raise RuntimeError(f"oracle mi pass 1 failed rc={rc}")
    return f, m, j, nv.value


def port_mi_pass2(grid, fixed, moving, coeff, f, m, j, num_vox, bins=32):
    """PVI-8 pass 2 over the grid's ROI with given histograms: (score,
    gradient of this ROI, double)."""
    g = orc_grid(grid, fixed)
    fh, mh = port_hist_eqsp(fixed.img, bins), port_hist_eqsp(moving.img, bins)
    s = C.c_double(0)
    gr = np.zeros(grid.num_coeff, np.float64)
    f, m, j = (np.ascontiguousarray(a, np.float64) for a in (f, m, j))
    rc = port().orc_mi_f64_pass2(
        C.byref(g), C.byref(orc_vol(fixed)), _p(fixed.img),
        C.byref(orc_vol(moving)), _p(moving.img),
        _p(np.ascontiguousarray(coeff, np.float32)), C.byref(fh), C.byref(mh),
        C.c_int64(num_vox), _p(f, f64p), _p(m, f64p), _p(j, f64p),
        C.byref(s), _p(gr, f64p))
    if rc:
        raise RuntimeError(f"oracle mi pass 2 failed rc={rc}")
    return s.value, gr


def port_parzen_params(fixed, moving, bins=32) -> OrcParzen:
    p = OrcParzen()
    f = np.ascontiguousarray(fixed.img, np.float32)
    m = np.ascontiguousarray(moving.img, np.float32)
    port().orc_parzen_init(C.byref(p), C.c_int64(bins), _p(f),
                           C.c_int64(f.size), _p(m), C.c_int64(m.size))
    return p


def port_mi_parzen(grid, fixed, moving, coeff, bins=32) -> Result:
    """Mattes MI with cubic B-spline Parzen windows, double precision (the
    published method; the reference has no such flavour)."""
    g = orc_grid(grid, fixed)
    p = port_parzen_params(fixed, moving, bins)
    nv = C.c_int64(0)
    s = C.c_double(0)
    gr = np.zeros(grid.num_coeff, np.float64)
    jh = np.zeros(bins * bins)
    coeff = np.ascontiguousarray(coeff, np.float32)
    rc = port().orc_mi_parzen_f64(
        C.byref(g), C.byref(orc_vol(fixed)), _p(fixed.img),
        C.byref(orc_vol(moving)), _p(moving.img), _p(coeff), C.byref(p),
        C.byref(s), _p(gr, f64p), C.byref(nv), _p(jh, f64p))
    if rc:
        raise RuntimeError(f"oracle parzen mi failed rc={rc}")
    j = jh.reshape(bins, bins)
    return Result(s.value, gr, nv.value, j.sum(axis=1), j.sum(axis=0), j)


def penalties(curvature=0.0, diffusion=0.0, lame_1=0.0, lame_2=0.0,
              total_displacement=0.0, third_order=0.0,
              linear_elastic_multiplier=1.0, curvature_mixed_weight=1.0):
    return np.array([curvature, diffusion, lame_1, lame_2, total_displacement,
                     third_order, linear_elastic_multiplier,
                     curvature_mixed_weight], np.float32)


def port_reg(grid, fixed, coeff, pen, precision="f32") -> Result:
    g = orc_grid(grid, fixed)
    coeff = np.ascontiguousarray(coeff, np.float32)
    if precision == "f32":
        s = C.c_float(0)
        gr = np.zeros(grid.num_coeff, np.float32)
        rc = port().orc_reg_f32(C.byref(g), _p(coeff), _p(pen), C.byref(s),
                                _p(gr))
    else:
        s = C.c_double(0)
        gr = np.zeros(grid.num_coeff, np.float64)
        rc = port().orc_reg_f64(C.byref(g), _p(coeff), _p(pen), C.byref(s),
                                _p(gr, f64p))
    if rc:
        raise RuntimeError("oracle reg failed")
    return Result(s.value, gr)


def port_landmarks_init(grid, fixed, fixed_pts):
    """Bspline_landmarks::initialize restated: (p, q) int64 arrays (n, 3),
    the tile and in-tile offset of each fixed landmark; raises ValueError
    when one lies outside the fixed image."""
    f = np.ascontiguousarray(np.asarray(fixed_pts, np.float32).reshape(-1, 3))
    n = len(f)
    p = np.zeros((n, 3), np.int64)
    q = np.zeros((n, 3), np.int64)
    port().orc_landmarks_init.restype = C.c_int64
    bad = port().orc_landmarks_init(C.byref(orc_grid(grid, fixed)),
                                    C.byref(orc_vol(fixed)), _p(f),
                                    C.c_int64(n), _p(p, i64p), _p(q, i64p))
    if bad:
        raise ValueError(f"fixed landmark {bad - 1} outside the fixed image")
    return p, q


def port_landmarks(grid, fixed, coeff, fixed_pts, moving_pts,
                   stiffness=1.0, grad=None) -> Result:
    """bspline_landmarks_score_a restated in the reference's float
    arithmetic: Result(lmetric, gradient), the landmark gradient added in
    place to a copy of `grad` (zeros when None), as the reference adds it to
    total_grad."""
    f = np.ascontiguousarray(np.asarray(fixed_pts, np.float32).reshape(-1, 3))
    m = np.ascontiguousarray(np.asarray(moving_pts, np.float32).reshape(-1, 3))
    n = min(len(f), len(m))
    f, m = np.ascontiguousarray(f[:n]), np.ascontiguousarray(m[:n])
    p, q = port_landmarks_init(grid, fixed, f)
    coeff = np.ascontiguousarray(coeff, np.float32)
    gr = (np.zeros(grid.num_coeff, np.float32) if grad is None
          else np.array(grad, np.float32))
    s = C.c_float(0)
    port().orc_landmarks_f32(C.byref(orc_grid(grid, fixed)), _p(coeff),
                             C.c_int64(n), _p(f), _p(m), _p(p, i64p),
                             _p(q, i64p), C.c_float(stiffness), C.byref(s),
                             _p(gr))
    return Result(s.value, gr)


def port_interpolate_vf(grid, fixed, coeff) -> np.ndarray:
    """bspline_interpolate_vf restated: field over the ROI, zero elsewhere;
    shape (nz, ny, nx, 3)."""
    vf = np.zeros(fixed.npix * 3, np.float32)
    coeff = np.ascontiguousarray(coeff, np.float32)
    rc = port().orc_interpolate_vf(C.byref(orc_grid(grid, fixed)),
                                   C.byref(orc_vol(fixed)), _p(coeff), _p(vf))
    if rc:
        raise RuntimeError("oracle interpolate_vf failed")
    nx, ny, nz = fixed.dim
    return vf.reshape(nz, ny, nx, 3)


def port_warp(grid, fixed, moving, coeff, default=0.0, with_vf=False):
    """bspline_warp (linear) restated: warped moving image on the fixed grid
    (and the field when with_vf)."""
    out = np.zeros(fixed.npix, np.float32)
    vf = np.zeros(fixed.npix * 3, np.float32) if with_vf else None
    coeff = np.ascontiguousarray(coeff, np.float32)
    rc = port().orc_warp(C.byref(orc_grid(grid, fixed)),
                         C.byref(orc_vol(fixed)), C.byref(orc_vol(moving)),
                         _p(moving.img), _p(coeff), C.c_float(default),
                         _p(out), _p(vf))
    if rc:
        raise RuntimeError(f"oracle warp failed rc={rc}")
    nx, ny, nz = fixed.dim
    out = out.reshape(nz, ny, nx)
    return (out, vf.reshape(nz, ny, nx, 3)) if with_vf else out


RESAMPLE_MODES = {"voxel": 0, "voxel_legacy": 1, "mm": 2, "percent": 3}


def port_resample_geometry(vol, mode, rate):
    """(dim, origin, spacing, is_copy) of registration_resample_volume."""
    od = (C.c_int64 * 3)()
    oo = (C.c_float * 3)()
    osp = (C.c_float * 3)()
    copy = port().orc_resample_geometry(
        (C.c_int64 * 3)(*vol.dim), (C.c_float * 3)(*vol.origin),
        (C.c_float * 3)(*vol.spacing), C.c_int(RESAMPLE_MODES[mode]),
        (C.c_float * 3)(*rate), od, oo, osp)
    return tuple(od), tuple(oo), tuple(osp), bool(copy)


def port_resample(vol, mode, rate):
    """registration_resample_volume on a float image: a Volume."""
    from plastimatch_b200.geometry import Volume
    od, oo, osp, copy = port_resample_geometry(vol, mode, rate)
    if copy:
        return Volume(vol.img.copy(), origin=vol.origin, spacing=vol.spacing,
                      dcos=vol.dcos)
    out = np.zeros(od[0] * od[1] * od[2], np.float32)
    img = np.ascontiguousarray(vol.img, np.float32)
    port().orc_resample_li((C.c_int64 * 3)(*vol.dim),
                           (C.c_float * 3)(*vol.origin),
                           (C.c_float * 3)(*vol.spacing), _p(img),
                           (C.c_int64 * 3)(*od), (C.c_float * 3)(*oo),
                           (C.c_float * 3)(*osp), _p(out))
    return Volume(out.reshape(od[2], od[1], od[0]), origin=oo, spacing=osp,
                  dcos=vol.dcos)


# ----------------------------------------------------------- reference ---

def _ref_geom(v) -> RefGeom:
    return RefGeom((C.c_int64 * 3)(*v.dim), (C.c_float * 3)(*v.origin),
                   (C.c_float * 3)(*v.spacing), (C.c_float * 9)(*v.dcos))


def _ref_grid(grid) -> RefGrid:
    return RefGrid((C.c_int64 * 3)(*grid.roi_offset),
                   (C.c_int64 * 3)(*grid.roi_dim),
                   (C.c_int64 * 3)(*grid.vox_per_rgn))


def ref_metric(grid, fixed, moving, coeff, flavor="g", metric="mse",
               bins=32, threads=0, moving_grad=None, fixed_roi=None,
               moving_roi=None, hist="eqsp") -> Result:
    """One reference flavour evaluation (bspline_score_mse / _mi); with
    image ROIs (geometry.Roi) the reference's ROI flavours (i / h); MI
    histogram type "eqsp" or "vopt" (Bspline_parms::mi_hist_type)."""
    ref().ref_set_mi_hist_type(C.c_int(1 if hist == "vopt" else 0))
    gr = np.zeros(grid.num_coeff, np.float32)
    res = RefResult()
    fh = np.zeros(bins)
    mh = np.zeros(bins)
    jh = np.zeros(bins * bins)
    coeff = np.ascontiguousarray(coeff, np.float32)
    head = (C.byref(_ref_geom(fixed)), _p(fixed.img),
            C.byref(_ref_geom(moving)), _p(moving.img), _p(moving_grad),
            C.byref(_ref_grid(grid)), _p(coeff), C.c_char(flavor.encode()),
            C.c_int(1 if metric == "mi" else 0), C.c_int(bins),
            C.c_int(threads))
    tail = (_p(gr), C.byref(res), _p(fh, f64p), _p(mh, f64p), _p(jh, f64p))
    if fixed_roi is None and moving_roi is None:
        rc = ref().ref_metric(*head, *tail)
    else:
        u8 = C.POINTER(C.c_uint8)
        rois = []
        for r in (fixed_roi, moving_roi):
            if r is None:
                rois += [None, None]
            else:
                rois += [C.byref(_ref_geom(r)), r.mask.ctypes.data_as(u8)]
        rc = ref().ref_metric_roi(*head, *rois, *tail)
    if rc:
        raise RuntimeError("reference metric failed")
    r = Result(res.score, gr, res.num_vox)
    if metric == "mi":
        r.f_hist, r.m_hist, r.j_hist = fh, mh, jh.reshape(bins, bins)
    return r


def ref_regularize(grid, fixed, coeff, curvature, impl="c",
                   threads=0) -> Result:
    gr = np.zeros(grid.num_coeff, np.float32)
    res = RefResult()
    coeff = np.ascontiguousarray(coeff, np.float32)
    rc = ref().ref_regularize(C.byref(_ref_geom(fixed)),
                              C.byref(_ref_grid(grid)), _p(coeff),
                              C.c_char(impl.encode()), C.c_float(curvature),
                              C.c_int(threads), _p(gr), C.byref(res))
    if rc:
        raise RuntimeError("reference regularize failed")
    return Result(res.rmetric, gr)


def ref_score(grid, fixed, moving, coeff, flavor="g", metric="mse", bins=32,
              reg_impl="", curvature=0.0, threads=0) -> Result:
    """The whole bspline_score(): metric + optional analytic regulariser."""
    gr = np.zeros(grid.num_coeff, np.float32)
    res = RefResult()
    coeff = np.ascontiguousarray(coeff, np.float32)
    rc = ref().ref_score(
        C.byref(_ref_geom(fixed)), _p(fixed.img), C.byref(_ref_geom(moving)),
        _p(moving.img), None, C.byref(_ref_grid(grid)), _p(coeff),
        C.c_char(flavor.encode()), C.c_int(1 if metric == "mi" else 0),
        C.c_int(bins), C.c_char(reg_impl.encode() if reg_impl else b"\0"),
        C.c_float(curvature), C.c_int(threads), _p(gr), C.byref(res))
    if rc:
        raise RuntimeError("reference score failed")
    return Result(res.total_score, gr, res.num_vox)


def ref_landmarks(grid, fixed, coeff, fixed_pts, moving_pts,
                  stiffness=1.0) -> Result:
    """The reference's own landmark term: Result(lmetric, gradient)."""
    f = np.ascontiguousarray(np.asarray(fixed_pts, np.float32).reshape(-1, 3))
    m = np.ascontiguousarray(np.asarray(moving_pts, np.float32).reshape(-1, 3))
    gr = np.zeros(grid.num_coeff, np.float32)
    res = RefResult()
    coeff = np.ascontiguousarray(coeff, np.float32)
    rc = ref().ref_landmarks(C.byref(_ref_geom(fixed)),
                             C.byref(_ref_grid(grid)), _p(coeff), _p(f),
                             _p(m), C.c_int64(min(len(f), len(m))),
                             C.c_float(stiffness), _p(gr), C.byref(res))
    if rc:
        raise RuntimeError("reference landmarks failed")
    return Result(res.score, gr)


def ref_score_landmarks(grid, fixed, moving, coeff, fixed_pts, moving_pts,
                        stiffness=1.0, flavor="g", metric="mse", bins=32,
                        reg_impl="", curvature=0.0, threads=0) -> Result:
    """bspline_score() with one metric, the optional analytic regulariser
    and landmark pairs: Result(total_score, total_grad, num_vox)."""
    f = np.ascontiguousarray(np.asarray(fixed_pts, np.float32).reshape(-1, 3))
    m = np.ascontiguousarray(np.asarray(moving_pts, np.float32).reshape(-1, 3))
    gr = np.zeros(grid.num_coeff, np.float32)
    res = RefResult()
    coeff = np.ascontiguousarray(coeff, np.float32)
    rc = ref().ref_score_landmarks(
        C.byref(_ref_geom(fixed)), _p(fixed.img), C.byref(_ref_geom(moving)),
        _p(moving.img), C.byref(_ref_grid(grid)), _p(coeff),
        C.c_char(flavor.encode()), C.c_int(1 if metric == "mi" else 0),
        C.c_int(bins), C.c_char(reg_impl.encode() if reg_impl else b"\0"),
        C.c_float(curvature), _p(f), _p(m), C.c_int64(min(len(f), len(m))),
        C.c_float(stiffness), C.c_int(threads), _p(gr), C.byref(res))
    if rc:
        raise RuntimeError("reference score failed")
    return Result(res.total_score, gr, res.num_vox)


def ref_volume_grad(v) -> np.ndarray:
    out = np.zeros(v.npix * 3, np.float32)
    ref().ref_volume_grad(C.byref(_ref_geom(v)), _p(v.img), _p(out))
    return out


def ref_luts(grid, fixed):
    vpr = grid.vox_per_rgn
    bx = np.zeros(4 * vpr[0], np.float32)
    by = np.zeros(4 * vpr[1], np.float32)
    bz = np.zeros(4 * vpr[2], np.float32)
    q = np.zeros(64 * vpr[0] * vpr[1] * vpr[2], np.float32)
    ref().ref_luts(C.byref(_ref_geom(fixed)), C.byref(_ref_grid(grid)),
                   _p(bx), _p(by), _p(bz), _p(q))
    return bx, by, bz, q


def ref_interpolate_vf(grid, fixed, coeff) -> np.ndarray:
    vf = np.zeros(fixed.npix * 3, np.float32)
    coeff = np.ascontiguousarray(coeff, np.float32)
    ref().ref_interpolate_vf(C.byref(_ref_geom(fixed)),
                             C.byref(_ref_grid(grid)), _p(coeff), _p(vf))
    nx, ny, nz = fixed.dim
    return vf.reshape(nz, ny, nx, 3)


def ref_warp(grid, fixed, moving, coeff, default=0.0, linear=True):
    """The reference's bspline_warp: (warped image, field)."""
    out = np.zeros(fixed.npix, np.float32)
    vf = np.zeros(fixed.npix * 3, np.float32)
    coeff = np.ascontiguousarray(coeff, np.float32)
    ref().ref_warp(C.byref(_ref_geom(fixed)), C.byref(_ref_geom(moving)),
                   _p(moving.img), C.byref(_ref_grid(grid)), _p(coeff),
                   C.c_int(1 if linear else 0), C.c_float(default), _p(out),
                   _p(vf))
    nx, ny, nz = fixed.dim
    return out.reshape(nz, ny, nx), vf.reshape(nz, ny, nx, 3)


def ref_resample(vol, mode, rate):
    """The reference's resampling (registration_resample_volume): a Volume."""
    from plastimatch_b200.geometry import Volume
    ref().ref_resample.restype = C.c_int64
    od = (C.c_int64 * 3)()
    oo = (C.c_float * 3)()
    osp = (C.c_float * 3)()
    img = np.ascontiguousarray(vol.img, np.float32)
    g = _ref_geom(vol)
    rate3 = (C.c_float * 3)(*rate)
    n = ref().ref_resample(C.byref(g), _p(img), C.c_int(RESAMPLE_MODES[mode]),
                           rate3, od, oo, osp, None, C.c_int64(0))
    out = np.zeros(n, np.float32)
    ref().ref_resample(C.byref(g), _p(img), C.c_int(RESAMPLE_MODES[mode]),
                       rate3, od, oo, osp, _p(out), C.c_int64(n))
    return Volume(out.reshape(od[2], od[1], od[0]), origin=tuple(oo),
                  spacing=tuple(osp), dcos=vol.dcos)


def ref_xform_save(path, grid, fixed, coeff):
    coeff = np.ascontiguousarray(coeff, np.float32)
    ref().ref_xform_save(os.fsencode(str(path)), C.byref(_ref_geom(fixed)),
                         C.byref(_ref_grid(grid)), _p(coeff))


def ref_xform_load(path):
    """(RefGeom, RefGrid, coeff) as bspline_xform_load reads them."""
    r = ref()
    r.ref_xform_load.restype = C.c_int64
    g, gr = RefGeom(), RefGrid()
    n = r.ref_xform_load(os.fsencode(str(path)), C.byref(g), C.byref(gr), None,
                         C.c_int64(0))
    if n < 0:
        raise RuntimeError("reference rejected the file")
    coeff = np.zeros(n, np.float32)
    r.ref_xform_load(os.fsencode(str(path)), C.byref(g), C.byref(gr), _p(coeff),
                     C.c_int64(n))
    return g, gr, coeff


def ref_write_mha(path, vol, vf=None):
    data = vol.img if vf is None else np.ascontiguousarray(vf, np.float32)
    ref().ref_write_mha(os.fsencode(str(path)), C.byref(_ref_geom(vol)),
                        C.c_int(1 if vf is None else 3), _p(data))


def ref_read_mha(path):
    """(RefGeom, channels, float data) as read_mha reads them."""
    r = ref()
    r.ref_read_mha.restype = C.c_int64
    g, ch = RefGeom(), C.c_int()
    n = r.ref_read_mha(os.fsencode(str(path)), C.byref(g), C.byref(ch), None,
                       C.c_int64(0))
    data = np.zeros(n * ch.value, np.float32)
    r.ref_read_mha(os.fsencode(str(path)), C.byref(g), C.byref(ch), _p(data),
                   C.c_int64(data.size))
    return g, ch.value, data


def ref_optimize(grid, fixed, moving, coeff, max_its=10, max_feval=10,
                 flavor="g", metric="mse", bins=32, reg_impl="", curvature=0.0,
                 threads=0):
    """Plastimatch's bspline_optimize with implementation liblbfgs:
    (final coefficients, last total score, iterations, evaluations)."""
    r = ref()
    c = np.array(coeff, np.float32)
    res = RefResult()
    it = r.ref_optimize(
        C.byref(_ref_geom(fixed)), _p(fixed.img), C.byref(_ref_geom(moving)),
        _p(moving.img), None, C.byref(_ref_grid(grid)), _p(c),
        C.c_char(flavor.encode()), C.c_int(1 if metric == "mi" else 0),
        C.c_int(bins), C.c_char(reg_impl.encode() if reg_impl else b"\0"),
        C.c_float(curvature), C.c_int(max_its), C.c_int(max_feval),
        C.c_int(threads), C.byref(res))
    return c, float(res.total_score), int(it), int(res.num_vox)


LBFGS_EVAL = C.CFUNCTYPE(C.c_double, C.c_void_p, C.POINTER(C.c_double),
                         C.POINTER(C.c_double), C.c_int, C.c_double)
LBFGS_PROGRESS = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double),
                             C.POINTER(C.c_double), C.c_double, C.c_double,
                             C.c_double, C.c_double, C.c_int, C.c_int, C.c_int)


def ref_lbfgs(fn, x0, max_its=1000):
    """liblbfgs (vendored in the reference) with default parameters on a
    Python function fn(x) -> (f, g), stopped by Plastimatch's progress rule
    (k > max_its; the linked liblbfgs consults it after every evaluation):
    (x, f, status, completed iterations, evaluations)."""
    n = len(x0)
    x = np.array(x0, np.float64)
    state = {"k": 0, "fe": 0}

    def ev(inst, xp, gp, nn, step):
        xa = np.ctypeslib.as_array(xp, shape=(nn,))
        f, g = fn(xa.copy())
        np.ctypeslib.as_array(gp, shape=(nn,))[:] = g
        state["fe"] += 1
        return float(f)

    def pr(inst, xp, gp, fx, xn, gn, st, nn, k, ls):
        if ls > 0:
            state["k"] = k          # completed line searches
        return 1 if k > max_its else 0

    cb_e, cb_p = LBFGS_EVAL(ev), LBFGS_PROGRESS(pr)
    fx = C.c_double()
    rc = ref().lbfgs(C.c_int(n), x.ctypes.data_as(C.POINTER(C.c_double)),
                     C.byref(fx), cb_e, cb_p, None, None)
    return x, fx.value, rc, state["k"], state["fe"]


# ------------------------------------------------------------- adapter ---

ADAPTER_SO = os.path.join(HERE, "_ref", "libb200adapter.so")


def adapter_available() -> bool:
    return os.path.exists(ADAPTER_SO)


def adapter_compare(grid, fixed, moving, coeff, flavor="g", metric="mse",
                    bins=32, hist="eqsp", threads=8, fixed_roi=None,
                    moving_roi=None):
    """Score the reference's own objects through the reference-side
    drop-in (oracle/ref/b200_adapter.cxx: bspline_b200_state_create +
    bspline_score_b200, linked with the reference build and the product
    library) and through the reference's CPU flavour: (b200 Result,
    reference Result).  Needs a GPU for the first."""
    lib = C.CDLL(ADAPTER_SO)
    n = grid.num_coeff
    g_b, g_r = np.zeros(n, np.float32), np.zeros(n, np.float32)
    s_b, s_r = C.c_float(), C.c_float()
    n_b, n_r = C.c_int64(), C.c_int64()
    u8 = C.POINTER(C.c_uint8)
    rois = []
    for r in (fixed_roi, moving_roi):
        rois += ([None, None] if r is None
                 else [C.byref(_ref_geom(r)), r.mask.ctypes.data_as(u8)])
    rc = lib.adapter_compare(
        C.byref(_ref_geom(fixed)), _p(fixed.img), C.byref(_ref_geom(moving)),
        _p(moving.img), C.byref(_ref_grid(grid)),
        _p(np.ascontiguousarray(coeff, np.float32)), C.c_char(flavor.encode()),
        C.c_int(1 if metric == "mi" else 0), C.c_int(bins),
        C.c_int(1 if hist == "vopt" else 0), C.c_int(threads), *rois,
        C.byref(s_b), C.byref(n_b), _p(g_b), C.byref(s_r), C.byref(n_r),
        _p(g_r))
    if rc:
        raise RuntimeError(f"adapter failed with status {rc}")
    return Result(s_b.value, g_b, n_b.value), Result(s_r.value, g_r, n_r.value)
