"""Generate tests/golden/*.npz from the reference's own CPU flavours.

Run where the reference tree is available and oracle/_ref/libplmref.so has
been built (oracle/build_ref.sh):

    python tests/golden/make_golden.py [--force]

(existing fixtures are kept unless --force)

Each fixture holds the inputs (images, geometry, grid, coefficients) and
the outputs of the compiled reference on them, so parity is pinned even
where the reference itself is absent (the GPU host).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from plastimatch_b200 import synth  # noqa: E402
from plastimatch_b200.geometry import BsplineGrid, Roi, Volume  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

ROT = (0.894427190999916, 0.447213595499958, 0.0,
       -0.447213595499958, 0.894427190999916, 0.0, 0.0, 0.0, 1.0)


def make_pair(dim, spacing, seed, dcos=None, remap=None, moving_shift=(0.5, -0.3, 0.2)):
    fixed = synth.gaussian_blobs(dim, spacing=spacing, seed=seed)
    if dcos is not None:
        fixed = Volume(fixed.img, origin=(-3.0, 2.0, 1.0), spacing=spacing, dcos=dcos)
    g0 = BsplineGrid.for_volume(fixed, (8, 7, 6))
    c0 = synth.random_coeff(g0, 2.0, seed=seed + 1)
    mov = synth.warp_trilinear(fixed, fixed, g0, c0)
    if remap is not None:
        mov = synth.intensity_remap(mov, remap, 5.0, seed + 2)
    org = tuple(o + s for o, s in zip(fixed.origin, moving_shift))
    moving = Volume(mov.img, origin=org, spacing=spacing, dcos=fixed.dcos)
    return fixed, moving


CASES = {
    # name: (dim, spacing, vpr, roi_offset, roi_dim, seed, dcos, remap, coeff sigma)
    "mse_small": ((24, 20, 18), (1.0, 1.1, 1.3), (5, 4, 6), (0, 0, 0), None, 11, None, None, 1.5),
    "mse_roi": ((26, 22, 17), (0.9, 1.0, 1.2), (4, 5, 4), (2, 3, 1), (19, 15, 13), 21, None, None, 1.2),
    "mse_dcos": ((22, 20, 16), (1.0, 1.0, 1.5), (5, 5, 4), (0, 0, 0), None, 31, ROT, None, 1.0),
    "mse_vpr8": ((33, 31, 30), (1.0, 1.0, 1.0), (8, 8, 8), (0, 0, 0), None, 41, None, None, 2.0),
    "mi_small": ((24, 22, 18), (1.0, 1.1, 1.3), (5, 6, 4), (0, 0, 0), None, 51, None, 0.7, 1.5),
    "mi_dcos": ((22, 20, 16), (1.0, 1.0, 1.5), (5, 5, 4), (0, 0, 0), None, 61, ROT, 1.6, 1.0),
}


# Dense vector field / warp fixtures: the inputs of an MSE case and the
# reference's bspline_interpolate_vf and bspline_warp (linear, default -7)
# on them.  Warp needs the ROI to be the whole image.
WARP_CASES = {"warp_small": "mse_small", "warp_dcos": "mse_dcos",
              "vf_roi": "mse_roi"}
WARP_DEFAULT = -7.0


# Pyramid resampling fixtures: one float image (odd sizes, anisotropic
# spacing, off-origin) through registration_resample_volume per type.
RESAMPLE_CASES = {
    "resample_voxel": ("voxel", (2.0, 3.0, 1.0)),
    "resample_voxel4": ("voxel", (4.0, 4.0, 2.0)),
    "resample_legacy": ("voxel_legacy", (2.0, 2.0, 3.0)),
    "resample_mm": ("mm", (2.3, 1.7, 3.1)),
    "resample_percent": ("percent", (0.5, 0.37, 0.8)),
}


# Landmark fixtures: the inputs of an MSE case, landmark pairs (spread,
# clustered so that landmarks share knots, and inside the first half voxel,
# which truncates to index 0) and the reference's landmark term alone and
# its whole bspline_score (MSE flavour g + curvature 0.005 + landmarks).
LANDMARK_CASES = {"landmarks_small": ("mse_small", 0.8, 17),
                  "landmarks_dcos": ("mse_dcos", 2.5, 23)}


# Image-ROI fixtures (Bspline_state::fixed_roi / moving_roi): the inputs of
# a case, a fixed ROI from an intensity window on the fixed image (as a
# registration stage builds it from its MI window) and a moving ROI on its
# own coarser, shifted grid (a box minus a slab), and the reference's ROI
# flavours on them: MSE i (via 'g') and k (via 'c'), MI h (via 'g').
# Names: roimask_<base>.
ROI_CASES = {"roimask_mse_small": "mse_small", "roimask_mse_roi": "mse_roi",
             "roimask_mse_dcos": "mse_dcos", "roimask_mi_small": "mi_small",
             "roimask_mi_dcos": "mi_dcos"}

# MI with a grid that starts at voxel 0 and covers the image with fewer
# ROI voxels than the image (the reference's histogram pass still scans
# the whole image): name -> (base, roi_dim).
MI_PARTIAL_CASES = {"mi_partial": ("mi_small", (22, 19, 17))}


# V-optimal histogram fixtures: the inputs of an MI case and the reference's
# MI flavour g with Bspline_parms::mi_hist_type = HIST_VOPT.
VOPT_CASES = {"vopt_mi_small": "mi_small", "vopt_mi_dcos": "mi_dcos"}


def roi_pair(fixed, moving, seed):
    lo = float(np.percentile(fixed.img, 35))
    froi = Roi.from_window(fixed, lo, 1e30)
    rng = np.random.default_rng(seed)
    sp = tuple(1.7 * s for s in moving.spacing)
    dim = tuple(int(np.ceil(d * s0 / s)) + 2 for d, s0, s in
                zip(moving.dim, moving.spacing, sp))
    m = np.zeros(dim[::-1], np.uint8)
    m[1:-2, 2:-1, 1:-3] = 1
    m[:, :, dim[0] // 2: dim[0] // 2 + 2] = 0
    org = tuple(o - 0.6 * s + float(rng.uniform(-0.3, 0.3))
                for o, s in zip(moving.origin, sp))
    mroi = Roi(m, origin=org, spacing=sp, dcos=moving.dcos)
    return froi, mroi


def roi_record(froi, mroi):
    return dict(froi_mask=froi.mask, froi_origin=np.array(froi.origin, np.float32),
                froi_spacing=np.array(froi.spacing, np.float32),
                froi_dcos=np.array(froi.dcos, np.float32),
                mroi_mask=mroi.mask, mroi_origin=np.array(mroi.origin, np.float32),
                mroi_spacing=np.array(mroi.spacing, np.float32),
                mroi_dcos=np.array(mroi.dcos, np.float32))


def landmark_points(fixed, n, seed):
    rng = np.random.default_rng(seed)
    dim = np.array(fixed.dim, np.float64)
    ijk = rng.uniform(0.0, 1.0, (n, 3)) * (dim - 1.0)
    ijk[: n // 4] = dim / 2 + rng.uniform(-1.5, 1.5, (n // 4, 3))
    ijk[n // 4] = (-0.4, -0.3, -0.2)
    dc = np.array(fixed.dcos, np.float64).reshape(3, 3)
    step = dc * np.array(fixed.spacing, np.float64)[None, :]
    f = (np.array(fixed.origin, np.float64) + ijk @ step.T).astype(np.float32)
    m = (f + rng.normal(0.0, 1.5, f.shape)).astype(np.float32)
    return f, m


def resample_input():
    v = synth.gaussian_blobs((37, 30, 23), spacing=(0.9, 1.1, 2.5), seed=71)
    return Volume(v.img, origin=(-11.3, 4.2, 7.7), spacing=v.spacing)


def main(force=False):
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libplmref.so missing; run oracle/build_ref.sh")
    for name, (dim, sp, vpr, roff, rdim, seed, dcos, remap, csig) in CASES.items():
        if not force and os.path.exists(os.path.join(OUT, f"{name}.npz")):
            continue
        fixed, moving = make_pair(dim, sp, seed, dcos, remap)
        grid = BsplineGrid.for_volume(fixed, vpr, roi_offset=roff,
                                      roi_dim=rdim)
        coeff = synth.random_coeff(grid, csig, seed=seed + 3)
        rec = dict(
            fixed=fixed.img, moving=moving.img,
            f_origin=np.array(fixed.origin, np.float32),
            f_spacing=np.array(fixed.spacing, np.float32),
            m_origin=np.array(moving.origin, np.float32),
            m_spacing=np.array(moving.spacing, np.float32),
            dcos=np.array(fixed.dcos, np.float32),
            roi_offset=np.array(grid.roi_offset), roi_dim=np.array(grid.roi_dim),
            vpr=np.array(grid.vox_per_rgn), coeff=coeff)
        rec["moving_grad"] = O.ref_volume_grad(moving)
        if name.startswith("mse"):
            # flavours c and o scan the whole fixed image (p = fijk/vpr), so
            # they are only defined when the ROI is the whole image
            flavors = "gh" if rdim is not None else "gco"
            for fl in flavors:
                r = O.ref_metric(grid, fixed, moving, coeff, flavor=fl)
                rec[f"{fl}_score"] = np.float32(r.score)
                rec[f"{fl}_grad"] = r.grad
                rec[f"{fl}_num_vox"] = np.int64(r.num_vox)
            rr = O.ref_regularize(grid, fixed, coeff, 0.005, impl="c")
            rec["reg_score"] = np.float32(rr.score)
            rec["reg_grad"] = rr.grad
            rt = O.ref_score(grid, fixed, moving, coeff, flavor="g",
                             reg_impl="c", curvature=0.005)
            rec["total_score"] = np.float32(rt.score)
            rec["total_grad"] = rt.grad
        else:
            if rdim is not None:
                raise SystemExit("MI flavour g needs the whole image as ROI")
            r = O.ref_metric(grid, fixed, moving, coeff, flavor="g",
                             metric="mi", bins=32)
            rec["mi_score"] = np.float32(r.score)
            rec["mi_grad"] = r.grad
            rec["mi_num_vox"] = np.int64(r.num_vox)
            rec["f_hist"], rec["m_hist"], rec["j_hist"] = r.f_hist, r.m_hist, r.j_hist
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **rec)
        print("wrote", name)
    for name, base in WARP_CASES.items():
        if not force and os.path.exists(os.path.join(OUT, f"{name}.npz")):
            continue
        dim, sp, vpr, roff, rdim, seed, dcos, remap, csig = CASES[base]
        fixed, moving = make_pair(dim, sp, seed, dcos, remap)
        grid = BsplineGrid.for_volume(fixed, vpr, roi_offset=roff,
                                      roi_dim=rdim)
        coeff = synth.random_coeff(grid, csig, seed=seed + 3)
        rec = dict(
            fixed=fixed.img, moving=moving.img,
            f_origin=np.array(fixed.origin, np.float32),
            f_spacing=np.array(fixed.spacing, np.float32),
            m_origin=np.array(moving.origin, np.float32),
            m_spacing=np.array(moving.spacing, np.float32),
            dcos=np.array(fixed.dcos, np.float32),
            roi_offset=np.array(grid.roi_offset), roi_dim=np.array(grid.roi_dim),
            vpr=np.array(grid.vox_per_rgn), coeff=coeff,
            vf=O.ref_interpolate_vf(grid, fixed, coeff),
            default=np.float32(WARP_DEFAULT))
        if rdim is None:
            rec["warped"], rec["warp_vf"] = O.ref_warp(grid, fixed, moving,
                                                       coeff, WARP_DEFAULT)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **rec)
        print("wrote", name)

    for name, (base, stiffness, n) in LANDMARK_CASES.items():
        if not force and os.path.exists(os.path.join(OUT, f"{name}.npz")):
            continue
        dim, sp, vpr, roff, rdim, seed, dcos, remap, csig = CASES[base]
        fixed, moving = make_pair(dim, sp, seed, dcos, remap)
        grid = BsplineGrid.for_volume(fixed, vpr, roi_offset=roff,
                                      roi_dim=rdim)
        coeff = synth.random_coeff(grid, csig, seed=seed + 3)
        fpts, mpts = landmark_points(fixed, n, seed + 4)
        rl = O.ref_landmarks(grid, fixed, coeff, fpts, mpts, stiffness)
        rt = O.ref_score(grid, fixed, moving, coeff, flavor="g",
                         reg_impl="c", curvature=0.005)
        rs = O.ref_score_landmarks(grid, fixed, moving, coeff, fpts, mpts,
                                   stiffness, flavor="g", reg_impl="c",
                                   curvature=0.005)
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            fixed=fixed.img, moving=moving.img,
            f_origin=np.array(fixed.origin, np.float32),
            f_spacing=np.array(fixed.spacing, np.float32),
            m_origin=np.array(moving.origin, np.float32),
            m_spacing=np.array(moving.spacing, np.float32),
            dcos=np.array(fixed.dcos, np.float32),
            roi_offset=np.array(grid.roi_offset), roi_dim=np.array(grid.roi_dim),
            vpr=np.array(grid.vox_per_rgn), coeff=coeff,
            fixed_pts=fpts, moving_pts=mpts, stiffness=np.float32(stiffness),
            lm_score=np.float32(rl.score), lm_grad=rl.grad,
            total_score=np.float32(rt.score), total_grad=rt.grad,
            total_lm_score=np.float32(rs.score), total_lm_grad=rs.grad)
        print("wrote", name)

    for name, base in ROI_CASES.items():
        if not force and os.path.exists(os.path.join(OUT, f"{name}.npz")):
            continue
        dim, sp, vpr, roff, rdim, seed, dcos, remap, csig = CASES[base]
        fixed, moving = make_pair(dim, sp, seed, dcos, remap)
        grid = BsplineGrid.for_volume(fixed, vpr, roi_offset=roff,
                                      roi_dim=rdim)
        coeff = synth.random_coeff(grid, csig, seed=seed + 3)
        froi, mroi = roi_pair(fixed, moving, seed + 5)
        rec = dict(
            fixed=fixed.img, moving=moving.img,
            f_origin=np.array(fixed.origin, np.float32),
            f_spacing=np.array(fixed.spacing, np.float32),
            m_origin=np.array(moving.origin, np.float32),
            m_spacing=np.array(moving.spacing, np.float32),
            dcos=np.array(fixed.dcos, np.float32),
            roi_offset=np.array(grid.roi_offset), roi_dim=np.array(grid.roi_dim),
            vpr=np.array(grid.vox_per_rgn), coeff=coeff, **roi_record(froi, mroi))
        rec["moving_grad"] = O.ref_volume_grad(moving)
        for tag, fr, mr in (("f", froi, None), ("m", None, mroi),
                            ("fm", froi, mroi)):
            if base.startswith("mse"):
                # flavour k (chosen for 'c') scans the whole fixed image,
                # defined only when the grid's ROI is the image
                for fl in ("gc" if rdim is None else "g"):
                    r = O.ref_metric(grid, fixed, moving, coeff, flavor=fl,
                                     fixed_roi=fr, moving_roi=mr)
                    rec[f"{tag}_{fl}_score"] = np.float32(r.score)
                    rec[f"{tag}_{fl}_grad"] = r.grad
                    rec[f"{tag}_{fl}_num_vox"] = np.int64(r.num_vox)
            else:
                r = O.ref_metric(grid, fixed, moving, coeff, flavor="g",
                                 metric="mi", bins=32, fixed_roi=fr,
                                 moving_roi=mr)
                rec[f"{tag}_mi_score"] = np.float32(r.score)
                rec[f"{tag}_mi_grad"] = r.grad
                rec[f"{tag}_mi_num_vox"] = np.int64(r.num_vox)
                rec[f"{tag}_j_hist"] = r.j_hist
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **rec)
        print("wrote", name)

    for name, base in VOPT_CASES.items():
        if not force and os.path.exists(os.path.join(OUT, f"{name}.npz")):
            continue
        dim, sp, vpr, roff, rdim, seed, dcos, remap, csig = CASES[base]
        fixed, moving = make_pair(dim, sp, seed, dcos, remap)
        grid = BsplineGrid.for_volume(fixed, vpr, roi_offset=roff,
                                      roi_dim=rdim)
        coeff = synth.random_coeff(grid, csig, seed=seed + 3)
        r = O.ref_metric(grid, fixed, moving, coeff, flavor="g", metric="mi",
                         bins=32, hist="vopt")
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            fixed=fixed.img, moving=moving.img,
            f_origin=np.array(fixed.origin, np.float32),
            f_spacing=np.array(fixed.spacing, np.float32),
            m_origin=np.array(moving.origin, np.float32),
            m_spacing=np.array(moving.spacing, np.float32),
            dcos=np.array(fixed.dcos, np.float32),
            roi_offset=np.array(grid.roi_offset), roi_dim=np.array(grid.roi_dim),
            vpr=np.array(grid.vox_per_rgn), coeff=coeff,
            mi_score=np.float32(r.score), mi_grad=r.grad,
            mi_num_vox=np.int64(r.num_vox), f_hist=r.f_hist, m_hist=r.m_hist,
            j_hist=r.j_hist)
        print("wrote", name)

    for name, (base, rdim) in MI_PARTIAL_CASES.items():
        if not force and os.path.exists(os.path.join(OUT, f"{name}.npz")):
            continue
        dim, sp, vpr, roff, _, seed, dcos, remap, csig = CASES[base]
        fixed, moving = make_pair(dim, sp, seed, dcos, remap)
        grid = BsplineGrid.for_volume(fixed, vpr, roi_dim=rdim)
        coeff = synth.random_coeff(grid, csig, seed=seed + 3)
        r = O.ref_metric(grid, fixed, moving, coeff, flavor="g", metric="mi",
                         bins=32)
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            fixed=fixed.img, moving=moving.img,
            f_origin=np.array(fixed.origin, np.float32),
            f_spacing=np.array(fixed.spacing, np.float32),
            m_origin=np.array(moving.origin, np.float32),
            m_spacing=np.array(moving.spacing, np.float32),
            dcos=np.array(fixed.dcos, np.float32),
            roi_offset=np.array(grid.roi_offset), roi_dim=np.array(grid.roi_dim),
            vpr=np.array(grid.vox_per_rgn), coeff=coeff,
            mi_score=np.float32(r.score), mi_grad=r.grad,
            mi_num_vox=np.int64(r.num_vox), f_hist=r.f_hist, m_hist=r.m_hist,
            j_hist=r.j_hist)
        print("wrote", name)

    for name, (mode, rate) in RESAMPLE_CASES.items():
        if not force and os.path.exists(os.path.join(OUT, f"{name}.npz")):
            continue
        v = resample_input()
        r = O.ref_resample(v, mode, rate)
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"), img=v.img,
            origin=np.array(v.origin, np.float32),
            spacing=np.array(v.spacing, np.float32),
            mode=np.array(mode), rate=np.array(rate, np.float32),
            out=r.img, out_dim=np.array(r.dim),
            out_origin=np.array(r.origin, np.float32),
            out_spacing=np.array(r.spacing, np.float32))
        print("wrote", name)


if __name__ == "__main__":
    main(force="--force" in sys.argv)
