"""plastimatch_b200: B200-native B-spline registration cost function.

Python binding over the C ABI of libplastimatch_b200.so
(include/plastimatch_b200.h).  The compute path is the CUDA library only:
if the shared library is missing or fails to load, importing the binding's
entry points raises -- there is no CPU fallback.

    from plastimatch_b200 import Context
    from plastimatch_b200.geometry import Volume, BsplineGrid
    ctx = Context(fixed, moving, grid)          # b200bsp_create
    ctx.set_images()                            # b200bsp_set_images
    score, grad, nvox = ctx.score_mse(coeff)    # b200bsp_score_mse

Arrays may be numpy (host) or torch CUDA tensors (device); results come
back as numpy arrays unless `out` tensors are given.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .geometry import BsplineGrid, Volume  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libplastimatch_b200.so")

B200BSP_OK = 0
FORMS = {"tc": 0, "fp32": 1}
MSE_GRAD = {"nearest": 0, "trilinear": 1}
ERRORS = {-1: "E_BADARG", -2: "E_OOM", -3: "E_CUDA", -4: "E_TIMEOUT",
          -5: "E_STATE", -6: "E_UNSUPPORTED", -7: "E_IO"}


class B200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class VolumeDesc(C.Structure):
    _fields_ = [("dim", C.c_int64 * 3), ("origin", C.c_float * 3),
                ("spacing", C.c_float * 3), ("dcos", C.c_float * 9)]


class GridDesc(C.Structure):
    _fields_ = [("roi_offset", C.c_int64 * 3), ("roi_dim", C.c_int64 * 3),
                ("vox_per_rgn", C.c_int64 * 3)]


class Opts(C.Structure):
    _fields_ = [("form", C.c_int), ("mse_grad", C.c_int), ("mi_bins", C.c_int),
                ("device", C.c_int), ("mi_window", C.c_int),
                ("wait_limit", C.c_int), ("mi_hist", C.c_int),
                ("tc_kernel", C.c_int)]


MI_WINDOW = {"pvi8": 0, "parzen": 1}
MI_HIST = {"eqsp": 0, "vopt": 1}
TC_KERNEL = {"auto": 0, "xlane": 1, "tile": 2}


class RegParms(C.Structure):
    _fields_ = [("curvature_penalty", C.c_float),
                ("diffusion_penalty", C.c_float),
                ("lame_coefficient_1", C.c_float),
                ("lame_coefficient_2", C.c_float),
                ("total_displacement_penalty", C.c_float),
                ("third_order_penalty", C.c_float),
                ("linear_elastic_multiplier", C.c_float),
                ("curvature_mixed_weight", C.c_float)]


def reg_parms(curvature=0.0, diffusion=0.0, lame_1=0.0, lame_2=0.0,
              total_displacement=0.0, third_order=0.0,
              linear_elastic_multiplier=1.0,
              curvature_mixed_weight=1.0) -> RegParms:
    return RegParms(curvature, diffusion, lame_1, lame_2, total_displacement,
                    third_order, linear_elastic_multiplier,
                    curvature_mixed_weight)


class LbfgsParms(C.Structure):
    _fields_ = [("m", C.c_int), ("epsilon", C.c_double), ("max_its", C.c_int),
                ("max_feval", C.c_int), ("max_linesearch", C.c_int),
                ("min_step", C.c_double), ("max_step", C.c_double),
                ("ftol", C.c_double), ("gtol", C.c_double),
                ("xtol", C.c_double)]


class LbfgsResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int),
                ("fevals", C.c_int), ("score", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


EVAL_FN = C.CFUNCTYPE(C.c_double, C.c_void_p, C.POINTER(C.c_double),
                      C.POINTER(C.c_double), C.c_int64)


def lbfgs_parms(**kw) -> LbfgsParms:
    """Defaults of b200bsp_lbfgs_default_parms with keyword overrides."""
    p = LbfgsParms()
    lib().b200bsp_lbfgs_default_parms(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def lbfgs_minimize(fn, x0, device: int = 0, **parms):
    """Minimise fn(x) -> (f, g) (numpy, double) with the device L-BFGS:
    (x, result dict)."""
    x = np.array(x0, np.float64)

    def cb(user, xp, gp, n):
        f, g = fn(np.ctypeslib.as_array(xp, shape=(n,)).copy())
        np.ctypeslib.as_array(gp, shape=(n,))[:] = g
        return float(f)

    cfn = EVAL_FN(cb)
    res = LbfgsResult()
    p = lbfgs_parms(**parms)
    _check(lib().b200bsp_lbfgs_minimize(x.size, _ptr(x, np.float64), cfn, None,
                                        C.byref(p), C.byref(res), device))
    return x, res.as_dict()


_lib = None

# Every entry point of include/plastimatch_b200.h with its ctypes signature.
_VP = C.c_void_p
_SIGS = {
    "b200bsp_default_opts": (None, [_VP]),
    "b200bsp_version": (C.c_char_p, []),
    "b200bsp_create": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "b200bsp_destroy": (C.c_int, [_VP]),
    "b200bsp_grid_info": (C.c_int, [_VP, _VP, _VP, _VP]),
    "b200bsp_set_images": (C.c_int, [_VP, _VP, _VP, _VP]),
    "b200bsp_set_stream": (C.c_int, [_VP, _VP]),
    "b200bsp_score_mse": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "b200bsp_score_mse_f64": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "b200bsp_score_mi": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "b200bsp_regularize": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "b200bsp_regularize_f64": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "b200bsp_set_landmarks": (C.c_int, [_VP, _VP, C.c_int64, _VP, C.c_int64,
                                        C.c_float]),
    "b200bsp_landmarks_score": (C.c_int, [_VP, _VP, _VP, _VP]),
    "b200bsp_set_roi": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "b200bsp_set_wait_limit": (C.c_int, [_VP, C.c_int, C.c_int]),
    "b200bsp_debug_fail_alloc": (None, [C.c_int]),
    "b200bsp_debug_host_lbfgs": (None, [C.c_int]),
    "b200bsp_score": (C.c_int, [_VP, _VP, C.c_int, C.c_float, _VP, _VP, _VP,
                                _VP, _VP]),
    "b200bsp_interpolate_vf": (C.c_int, [_VP, _VP, _VP]),
    "b200bsp_warp": (C.c_int, [_VP, _VP, C.c_float, _VP]),
    "b200bsp_volume_grad": (C.c_int, [_VP, _VP, _VP, C.c_int]),
    "b200bsp_enable_timing": (C.c_int, [_VP, C.c_int]),
    "b200bsp_last_timing": (C.c_int, [_VP, _VP, _VP]),
    "b200bsp_last_main_ms": (C.c_int, [_VP, _VP]),
    "b200bsp_last_error": (C.c_char_p, [_VP]),
    "b200bsp_resample_geometry": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP]),
    "b200bsp_resample": (C.c_int, [_VP, _VP, _VP, _VP, C.c_int]),
    "b200bsp_xform_save": (C.c_int, [C.c_char_p, _VP, _VP, _VP]),
    "b200bsp_xform_load": (C.c_int, [C.c_char_p, _VP, _VP, _VP, C.c_int64,
                                     _VP]),
    "b200bsp_mha_write": (C.c_int, [C.c_char_p, _VP, C.c_int, _VP]),
    "b200bsp_mha_read": (C.c_int, [C.c_char_p, _VP, _VP, _VP, C.c_int64]),
    "b200bsp_lbfgs_default_parms": (None, [_VP]),
    "b200bsp_optimize_lbfgs": (C.c_int, [_VP, C.c_int, C.c_float, _VP, _VP,
                                         _VP, _VP]),
    "b200bsp_lbfgs_minimize": (C.c_int, [C.c_int64, _VP, _VP, _VP, _VP, _VP,
                                         C.c_int]),
    "b200bsp_score_mse_static": (C.c_int, [_VP, _VP, _VP, C.c_int, _VP, _VP,
                                           _VP, _VP, _VP, _VP, _VP, _VP]),
    "b200bsp_autotune": (C.c_int, [_VP, _VP, C.c_int, _VP]),
    "b200bsp_mse_kernel": (C.c_int, [_VP, _VP, _VP, _VP]),
    "b200bsp_mi_hist": (C.c_int, [_VP, _VP, _VP]),
    "b200bsp_mi_grad": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "b200bsp_batch_create": (C.c_int, [_VP, C.c_int, _VP]),
    "b200bsp_batch_destroy": (None, [_VP]),
    "b200bsp_batch_last_error": (C.c_char_p, [_VP]),
    "b200bsp_batch_score_mse": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "b200bsp_batch_optimize_lbfgs": (C.c_int, [_VP, C.c_float, _VP, _VP,
                                               _VP]),
}


def lib():
    """Load libplastimatch_b200.so (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with "
                "`python -m plastimatch_b200.build` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _vol_desc(v: Volume) -> VolumeDesc:
    return VolumeDesc((C.c_int64 * 3)(*v.dim), (C.c_float * 3)(*v.origin),
                      (C.c_float * 3)(*v.spacing), (C.c_float * 9)(*v.dcos))


def _ptr(a, dtype=np.float32):
    """Raw pointer of a numpy array or torch tensor (None passes through)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if not (a.flags["C_CONTIGUOUS"] and a.dtype == dtype):
        raise ValueError(f"need a C-contiguous {np.dtype(dtype)} array")
    return a.ctypes.data


def _check(rc, ctx_handle=None):
    if rc != B200BSP_OK:
        msg = lib().b200bsp_last_error(ctx_handle)
        raise B200Error(rc, msg.decode() if msg else "")


def volume_grad(vol: Volume, device: int = 0) -> np.ndarray:
    """Moving-image gradient on the device (volume_calc_grad)."""
    out = np.zeros(vol.npix * 3, np.float32)
    d = _vol_desc(vol)
    _check(lib().b200bsp_volume_grad(C.byref(d), _ptr(vol.img), _ptr(out),
                                     device))
    return out


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


def xform_save(path, fixed: Volume, grid: BsplineGrid, coeff) -> None:
    """Write a B-spline coefficient file (Bspline_xform::save format)."""
    gd = GridDesc((C.c_int64 * 3)(*grid.roi_offset),
                  (C.c_int64 * 3)(*grid.roi_dim),
                  (C.c_int64 * 3)(*grid.vox_per_rgn))
    _check(lib().b200bsp_xform_save(_path(path), C.byref(_vol_desc(fixed)),
                                    C.byref(gd), _ptr(coeff)))


def xform_load(path):
    """Read a B-spline coefficient file: (geometry dict, BsplineGrid over an
    image of that geometry, coefficients)."""
    v, g, n = VolumeDesc(), GridDesc(), C.c_int64()
    _check(lib().b200bsp_xform_load(_path(path), C.byref(v), C.byref(g), None,
                                    0, C.byref(n)))
    coeff = np.zeros(n.value, np.float32)
    _check(lib().b200bsp_xform_load(_path(path), C.byref(v), C.byref(g),
                                    _ptr(coeff), n.value, C.byref(n)))
    geom = dict(dim=tuple(v.dim), origin=tuple(v.origin),
                spacing=tuple(v.spacing), dcos=tuple(v.dcos))
    grid = BsplineGrid(geom["origin"], geom["spacing"], geom["dim"],
                       tuple(g.roi_offset), tuple(g.roi_dim),
                       tuple(g.vox_per_rgn), geom["dcos"])
    return geom, grid, coeff


def mha_write(path, vol: Volume, vf=None) -> None:
    """Write vol.img (or, when given, the vector field vf of vol's geometry,
    shape (nz, ny, nx, 3)) as MetaImage (write_mha format)."""
    data = vol.img if vf is None else np.ascontiguousarray(vf, np.float32)
    _check(lib().b200bsp_mha_write(_path(path), C.byref(_vol_desc(vol)),
                                   1 if vf is None else 3, _ptr(data)))


def mha_read(path):
    """Read a MetaImage: a Volume for one channel, else (vector field
    (nz, ny, nx, 3), Volume of the geometry with a zero image)."""
    v, ch = VolumeDesc(), C.c_int()
    _check(lib().b200bsp_mha_read(_path(path), C.byref(v), C.byref(ch), None, 0))
    nx, ny, nz = v.dim
    data = np.zeros(nx * ny * nz * ch.value, np.float32)
    _check(lib().b200bsp_mha_read(_path(path), C.byref(v), C.byref(ch),
                                  _ptr(data), data.size))
    kw = dict(origin=tuple(v.origin), spacing=tuple(v.spacing),
              dcos=tuple(v.dcos))
    if ch.value == 1:
        return Volume(data.reshape(nz, ny, nx), **kw)
    return data.reshape(nz, ny, nx, 3), Volume(np.zeros((nz, ny, nx)), **kw)


RESAMPLE = {"voxel": 0, "voxel_legacy": 1, "mm": 2, "percent": 3}


def resample_geometry(vol: Volume, mode: str, rate):
    """(dim, origin, spacing, is_copy) of one pyramid level
    (b200bsp_resample_geometry)."""
    d = _vol_desc(vol)
    o = VolumeDesc()
    cp = C.c_int()
    _check(lib().b200bsp_resample_geometry(C.byref(d), RESAMPLE[mode],
                                           (C.c_float * 3)(*rate), C.byref(o),
                                           C.byref(cp)))
    return tuple(o.dim), tuple(o.origin), tuple(o.spacing), bool(cp.value)


def resample(vol: Volume, dim, origin, spacing, out=None,
             device: int = 0) -> Volume:
    """Trilinear resampling onto the grid (dim, origin, spacing)
    (b200bsp_resample).  vol.img and `out` may be numpy arrays or device
    tensors; returns a Volume holding the numpy result when out is None."""
    d = _vol_desc(vol)
    o = VolumeDesc((C.c_int64 * 3)(*dim), (C.c_float * 3)(*origin),
                   (C.c_float * 3)(*spacing), (C.c_float * 9)(*vol.dcos))
    res = np.zeros(dim[0] * dim[1] * dim[2], np.float32) if out is None else out
    _check(lib().b200bsp_resample(C.byref(d), _ptr(vol.img), C.byref(o),
                                  _ptr(res), device))
    if out is not None:
        return out
    return Volume(res.reshape(dim[2], dim[1], dim[0]), origin=origin,
                  spacing=spacing, dcos=vol.dcos)


def pyramid_level(vol: Volume, mode: str, rate, device: int = 0) -> Volume:
    """registration_resample_volume: the image of one pyramid level."""
    dim, origin, spacing, copy = resample_geometry(vol, mode, rate)
    if copy:
        return Volume(vol.img.copy(), origin=vol.origin, spacing=vol.spacing,
                      dcos=vol.dcos)
    return resample(vol, dim, origin, spacing, device=device)


def score_mse_static(fixed: Volume, moving: Volume, grid: BsplineGrid,
                     fixed_img, moving_img, coeff, grad, score=None,
                     nvox=None, moving_grad=None, mse_grad: str = "nearest",
                     stream: int | None = None) -> None:
    """b200bsp_score_mse_static: MSE score + gradient without a context and
    without allocating; every buffer is a device tensor the caller owns
    (grad: num_coeff float32, score: 1 float32, nvox: 1 int64).  Ordered on
    `stream` (a cudaStream_t handle; None = the legacy default stream)."""
    fd, md = _vol_desc(fixed), _vol_desc(moving)
    gd = GridDesc((C.c_int64 * 3)(*grid.roi_offset),
                  (C.c_int64 * 3)(*grid.roi_dim),
                  (C.c_int64 * 3)(*grid.vox_per_rgn))
    _check(lib().b200bsp_score_mse_static(
        C.byref(fd), C.byref(md), C.byref(gd), MSE_GRAD[mse_grad],
        _ptr(fixed_img), _ptr(moving_img), _ptr(moving_grad), _ptr(coeff),
        _ptr(score), _ptr(grad), _ptr(nvox), stream))


class Context:
    """One registration stage's device state (b200bsp_ctx)."""

    def __init__(self, fixed: Volume, moving: Volume, grid: BsplineGrid,
                 form: str = "tc", mse_grad: str = "nearest",
                 mi_bins: int = 32, device: int = 0, mi_window: str = "pvi8",
                 mi_hist: str = "eqsp", wait_limit: int = 0,
                 tc_kernel: str = "auto"):
        L = lib()
        self.fixed, self.moving, self.grid = fixed, moving, grid
        self.form = form
        self.mi_bins = mi_bins
        o = Opts()
        L.b200bsp_default_opts(C.byref(o))
        o.form = FORMS[form]
        o.mse_grad = MSE_GRAD[mse_grad]
        o.mi_bins = mi_bins
        o.mi_window = MI_WINDOW[mi_window]
        o.mi_hist = MI_HIST[mi_hist]
        o.wait_limit = wait_limit
        o.tc_kernel = TC_KERNEL[tc_kernel]
        o.device = device
        self._fd, self._md = _vol_desc(fixed), _vol_desc(moving)
        self._gd = GridDesc((C.c_int64 * 3)(*grid.roi_offset),
                            (C.c_int64 * 3)(*grid.roi_dim),
                            (C.c_int64 * 3)(*grid.vox_per_rgn))
        h = C.c_void_p()
        rc = L.b200bsp_create(C.byref(self._fd), C.byref(self._md),
                              C.byref(self._gd), C.byref(o), C.byref(h))
        _check(rc)
        self._h = h
        rd = (C.c_int64 * 3)()
        cd = (C.c_int64 * 3)()
        nc = C.c_int64()
        _check(L.b200bsp_grid_info(h, rd, cd, C.byref(nc)), h)
        self.rdims, self.cdims = tuple(rd), tuple(cd)
        self.num_coeff = nc.value
        assert self.rdims == grid.rdims and self.num_coeff == grid.num_coeff

    def close(self):
        if getattr(self, "_h", None):
            lib().b200bsp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_images(self, fixed_img=None, moving_img=None, moving_grad=None):
        f = self.fixed.img if fixed_img is None else fixed_img
        m = self.moving.img if moving_img is None else moving_img
        _check(lib().b200bsp_set_images(self._h, _ptr(f), _ptr(m),
                                        _ptr(moving_grad)), self._h)
        return self

    def set_stream(self, stream_handle: int | None):
        _check(lib().b200bsp_set_stream(self._h, stream_handle), self._h)

    def enable_timing(self, on=True):
        _check(lib().b200bsp_enable_timing(self._h, int(on)), self._h)

    def last_timing(self):
        ms = C.c_float()
        n = C.c_int()
        main = C.c_float()
        _check(lib().b200bsp_last_timing(self._h, C.byref(ms), C.byref(n)),
               self._h)
        _check(lib().b200bsp_last_main_ms(self._h, C.byref(main)), self._h)
        return ms.value, main.value, n.value

    def score_mse(self, coeff, grad_out=None, score_out=None, nvox_out=None):
        """(score, grad, num_vox).  With torch CUDA tensors for coeff and
        all outputs the call is stream-ordered and returns the tensors."""
        if grad_out is not None:
            _check(lib().b200bsp_score_mse(self._h, _ptr(coeff),
                                           _ptr(score_out), _ptr(grad_out),
                                           _ptr(nvox_out)), self._h)
            return score_out, grad_out, nvox_out
        g = np.zeros(self.num_coeff, np.float32)
        s = C.c_float()
        n = C.c_int64()
        _check(lib().b200bsp_score_mse(self._h, _ptr(coeff), C.addressof(s),
                                       _ptr(g), C.addressof(n)), self._h)
        return s.value, g, n.value

    def autotune(self, coeff, evals=3) -> int:
        """b200bsp_autotune: pick the tensor-core kernel's batch split by
        timing; returns its tiles per batch."""
        t = C.c_int()
        _check(lib().b200bsp_autotune(self._h, _ptr(coeff), evals,
                                      C.byref(t)), self._h)
        return t.value

    def mse_kernel(self):
        """b200bsp_mse_kernel: ("xlane" | "tile" | "fp32", tiles per
        batch, batches) of the next MSE evaluation."""
        k, t, b = C.c_int(), C.c_int(), C.c_int()
        _check(lib().b200bsp_mse_kernel(self._h, C.byref(k), C.byref(t),
                                        C.byref(b)), self._h)
        name = {0: "fp32", 1: "xlane", 2: "tile"}[k.value]
        return name, t.value, b.value

    def score_mse_f64(self, coeff):
        g = np.zeros(self.num_coeff, np.float64)
        s = C.c_double()
        n = C.c_int64()
        _check(lib().b200bsp_score_mse_f64(self._h, _ptr(coeff),
                                           C.addressof(s), _ptr(g, np.float64),
                                           C.addressof(n)), self._h)
        return s.value, g, n.value

    def score_mi(self, coeff, with_hist=False):
        b = None
        g = np.zeros(self.num_coeff, np.float32)
        s = C.c_float()
        n = C.c_int64()
        fh = mh = jh = None
        if with_hist:
            b = self.mi_bins
            fh, mh, jh = np.zeros(b), np.zeros(b), np.zeros(b * b)
        _check(lib().b200bsp_score_mi(self._h, _ptr(coeff), C.addressof(s),
                                      _ptr(g), C.addressof(n),
                                      _ptr(fh, np.float64), _ptr(mh, np.float64),
                                      _ptr(jh, np.float64)), self._h)
        if with_hist:
            return s.value, g, n.value, (fh, mh, jh.reshape(b, b))
        return s.value, g, n.value

    def mi_hist(self, coeff) -> np.ndarray:
        """MI pass 1 over the ROI: exact integer histograms (f, m, joint,
        count) as int64 (b200bsp_mi_hist)."""
        b = self.mi_bins
        h = np.zeros(2 * b + b * b + 1, np.int64)
        _check(lib().b200bsp_mi_hist(self._h, _ptr(coeff), _ptr(h, np.int64)),
               self._h)
        return h

    def mi_grad(self, coeff, hist):
        """MI pass 2 with given (summed) histograms: (score, this ROI's
        gradient in double, num_vox) (b200bsp_mi_grad)."""
        h = np.ascontiguousarray(hist, np.int64)
        g = np.zeros(self.num_coeff, np.float64)
        s = C.c_float()
        n = C.c_int64()
        _check(lib().b200bsp_mi_grad(self._h, _ptr(coeff), _ptr(h, np.int64),
                                     C.addressof(s), _ptr(g, np.float64),
                                     C.addressof(n)), self._h)
        return s.value, g, n.value

    def regularize(self, coeff, parms: RegParms, grad=None):
        """(rmetric, grad): grad accumulates the regulariser gradient."""
        g = np.zeros(self.num_coeff, np.float32) if grad is None else grad
        s = C.c_float()
        _check(lib().b200bsp_regularize(self._h, _ptr(coeff), C.byref(parms),
                                        C.addressof(s), _ptr(g)), self._h)
        return s.value, g

    def regularize_f64(self, coeff, parms: RegParms, grad=None):
        """(rmetric as a double, grad): for finite-difference checks."""
        g = np.zeros(self.num_coeff, np.float32) if grad is None else grad
        s = C.c_double()
        _check(lib().b200bsp_regularize_f64(self._h, _ptr(coeff),
                                            C.byref(parms), C.addressof(s),
                                            _ptr(g)), self._h)
        return s.value, g

    def set_landmarks(self, fixed_pts, moving_pts, stiffness=1.0):
        """Landmark pairs (points in mm, one xyz row each) that score()
        adds as stiffness * mean squared distance (b200bsp_set_landmarks);
        empty lists remove them."""
        f = np.ascontiguousarray(np.asarray(fixed_pts, np.float32).reshape(-1, 3))
        m = np.ascontiguousarray(np.asarray(moving_pts, np.float32).reshape(-1, 3))
        _check(lib().b200bsp_set_landmarks(self._h, _ptr(f), len(f), _ptr(m),
                                           len(m), stiffness), self._h)
        return self

    def set_roi(self, fixed_roi=None, moving_roi=None):
        """Image ROIs (geometry.Roi or None) that every later evaluation
        respects: fixed voxels outside the fixed ROI and moving positions
        outside the moving ROI do not count (b200bsp_set_roi); no
        arguments remove them."""
        args = []
        self._roi_keep = []
        for r in (fixed_roi, moving_roi):
            if r is None:
                args += [None, None]
            else:
                d = _vol_desc(r)
                self._roi_keep += [d, r.mask]
                args += [C.byref(d), r.mask.ctypes.data]
        _check(lib().b200bsp_set_roi(self._h, *args), self._h)
        return self

    def landmarks_score(self, coeff, grad=None):
        """(lmetric, grad): grad accumulates the landmark gradient
        (b200bsp_landmarks_score)."""
        g = np.zeros(self.num_coeff, np.float32) if grad is None else grad
        s = C.c_float()
        _check(lib().b200bsp_landmarks_score(self._h, _ptr(coeff),
                                             C.addressof(s), _ptr(g)), self._h)
        return s.value, g

    def score(self, coeff, metric="mse", lam=1.0, reg: RegParms | None = None):
        """bspline_score(): (total_score, total_grad, smetric, num_vox)."""
        g = np.zeros(self.num_coeff, np.float32)
        ts, sm = C.c_float(), C.c_float()
        n = C.c_int64()
        _check(lib().b200bsp_score(self._h, _ptr(coeff),
                                   0 if metric == "mse" else 1, lam,
                                   C.byref(reg) if reg is not None else None,
                                   C.addressof(ts), _ptr(g), C.addressof(sm),
                                   C.addressof(n)), self._h)
        return ts.value, g, sm.value, n.value

    def optimize_lbfgs(self, coeff, metric="mse", lam=1.0,
                       reg: RegParms | None = None, **parms):
        """b200bsp_optimize_lbfgs from x0 = coeff: (coefficients, result
        dict).  parms override the defaults (max_its, max_feval, m, ...)."""
        c = np.array(coeff, np.float32) if not hasattr(coeff, "data_ptr") \
            else coeff
        res = LbfgsResult()
        p = lbfgs_parms(**parms)
        _check(lib().b200bsp_optimize_lbfgs(
            self._h, 0 if metric == "mse" else 1, lam,
            C.byref(reg) if reg is not None else None, C.byref(p), _ptr(c),
            C.byref(res)), self._h)
        return c, res.as_dict()

    def interpolate_vf(self, coeff):
        nx, ny, nz = self.fixed.dim
        vf = np.zeros(nx * ny * nz * 3, np.float32)
        _check(lib().b200bsp_interpolate_vf(self._h, _ptr(coeff), _ptr(vf)),
               self._h)
        return vf.reshape(nz, ny, nx, 3)

    def warp(self, coeff, default_value=0.0):
        nx, ny, nz = self.fixed.dim
        out = np.zeros(nx * ny * nz, np.float32)
        _check(lib().b200bsp_warp(self._h, _ptr(coeff), default_value,
                                  _ptr(out)), self._h)
        return out.reshape(nz, ny, nx)



class Batch:
    """Registrations on one device evaluated together (b200bsp_batch): one
    CUDA graph launch per round of evaluations over all contexts."""

    def __init__(self, contexts):
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(
            *[c._h.value for c in self.contexts])
        h = C.c_void_p()
        _check(lib().b200bsp_batch_create(arr, len(self.contexts),
                                          C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().b200bsp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _fail(self, rc):
        if rc:
            msg = lib().b200bsp_batch_last_error(self._h)
            raise B200Error(rc, msg.decode() if msg else "")

    def score_mse(self, coeffs, grads, scores, num_vox=None):
        """All buffers torch CUDA tensors: coeffs[i], grads[i] (float32,
        num_coeff of context i), scores (n float32), num_vox (n int64)."""
        n = len(self.contexts)
        cp = (C.c_void_p * n)(*[_ptr(c) for c in coeffs])
        gp = (C.c_void_p * n)(*[_ptr(g) for g in grads])
        self._fail(lib().b200bsp_batch_score_mse(
            self._h, cp, gp, _ptr(scores), _ptr(num_vox, np.int64)))

    def optimize_lbfgs(self, coeffs, lam=1.0, **parms):
        """One L-BFGS registration per context from coeffs[i] (numpy float32
        arrays, updated in place): a list of result dicts."""
        n = len(self.contexts)
        arrs = [np.ascontiguousarray(c, np.float32) for c in coeffs]
        cp = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
        res = (LbfgsResult * n)()
        p = lbfgs_parms(**parms)
        self._fail(lib().b200bsp_batch_optimize_lbfgs(self._h, lam,
                                                      C.byref(p), cp, res))
        for a, c in zip(arrs, coeffs):
            if a is not c:
                c[...] = a
        return [r.as_dict() for r in res]
