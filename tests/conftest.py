import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_names(prefix=""):
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and f.startswith(prefix))


def load_golden(name):
    """A golden case as (fixed, moving, grid, coeff, record)."""
    from plastimatch_b200.geometry import BsplineGrid, Volume
    rec = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    dcos = tuple(float(v) for v in rec["dcos"])
    fixed = Volume(rec["fixed"], origin=rec["f_origin"],
                   spacing=rec["f_spacing"], dcos=dcos)
    moving = Volume(rec["moving"], origin=rec["m_origin"],
                    spacing=rec["m_spacing"], dcos=dcos)
    grid = BsplineGrid.for_volume(fixed, tuple(int(v) for v in rec["vpr"]),
                                  roi_offset=tuple(int(v) for v in rec["roi_offset"]),
                                  roi_dim=tuple(int(v) for v in rec["roi_dim"]))
    return fixed, moving, grid, rec["coeff"], rec


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def load_rois(rec):
    """The (fixed, moving) image ROIs stored in a roimask_* golden case."""
    from plastimatch_b200.geometry import Roi

    def mk(p):
        return Roi(rec[f"{p}_mask"], origin=tuple(float(v) for v in rec[f"{p}_origin"]),
                   spacing=tuple(float(v) for v in rec[f"{p}_spacing"]),
                   dcos=tuple(float(v) for v in rec[f"{p}_dcos"]))
    return mk("froi"), mk("mroi")


ROI_TAGS = ("f", "m", "fm")


def pick_rois(tag, froi, mroi):
    return (froi if "f" in tag else None), (mroi if "m" in tag else None)
