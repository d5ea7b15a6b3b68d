"""The landmark term of the cost function, oracle side (CPU).

The restatement (oracle/bspline_oracle.c, orc_landmarks_*) must equal the
reference's bspline_landmarks_score_a bit for bit -- the fixtures under
tests/golden/ were written by the compiled reference -- and the whole
bspline_score with landmarks must equal the score without them plus the
landmark term added in place, in float, in the reference's order.
"""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden
from plastimatch_b200 import synth
from plastimatch_b200.geometry import BsplineGrid

CASES = ["landmarks_small", "landmarks_dcos"]


@pytest.mark.parametrize("name", CASES)
def test_port_matches_golden(name):
    fixed, _, grid, coeff, rec = load_golden(name)
    r = O.port_landmarks(grid, fixed, coeff, rec["fixed_pts"],
                         rec["moving_pts"], float(rec["stiffness"]))
    assert np.float32(r.score) == rec["lm_score"]
    np.testing.assert_array_equal(r.grad, rec["lm_grad"])
    assert np.count_nonzero(r.grad) > 0


@pytest.mark.parametrize("name", CASES)
def test_total_with_landmarks_is_total_plus_term(name):
    """bspline_score adds stiffness * lmetric to the total after the
    regulariser, and the landmark gradient into total_grad in place."""
    fixed, _, grid, coeff, rec = load_golden(name)
    k = rec["stiffness"]
    r = O.port_landmarks(grid, fixed, coeff, rec["fixed_pts"],
                         rec["moving_pts"], float(k), grad=rec["total_grad"])
    np.testing.assert_array_equal(r.grad, rec["total_lm_grad"])
    total = np.float32(rec["total_score"]) + np.float32(k) * np.float32(r.score)
    assert np.float32(total) == rec["total_lm_score"]


@pytest.mark.skipif(not O.ref_available(), reason="reference not built")
@pytest.mark.parametrize("name", CASES)
def test_reference_reproduces_golden(name):
    fixed, _, grid, coeff, rec = load_golden(name)
    r = O.ref_landmarks(grid, fixed, coeff, rec["fixed_pts"],
                        rec["moving_pts"], float(rec["stiffness"]))
    assert np.float32(r.score) == rec["lm_score"]
    np.testing.assert_array_equal(r.grad, rec["lm_grad"])


@pytest.mark.skipif(not O.ref_available(), reason="reference not built")
def test_shorter_list_sets_the_count():
    """Bspline_landmarks::set_landmarks uses min(#fixed, #moving) pairs."""
    fixed, _, grid, coeff, rec = load_golden("landmarks_small")
    f, m = rec["fixed_pts"], rec["moving_pts"][:9]
    a = O.port_landmarks(grid, fixed, coeff, f, m, 1.3)
    b = O.ref_landmarks(grid, fixed, coeff, f, m, 1.3)
    assert a.score == b.score
    np.testing.assert_array_equal(a.grad, b.grad)


def test_grid_coordinates():
    """Tile and offset from the truncated voxel index; a point within the
    first half voxel below the origin truncates to index 0."""
    fixed = synth.gaussian_blobs((20, 18, 16), spacing=(1.0, 2.0, 0.5), seed=3)
    grid = BsplineGrid.for_volume(fixed, (4, 5, 3))
    o = np.array(fixed.origin, np.float32)
    pts = np.array([o + (0.0, 0.0, 0.0), o + (-0.4, -0.9, -0.2),
                    o + (13.7, 2.0 * 11.2, 0.5 * 14.99)], np.float32)
    p, q = O.port_landmarks_init(grid, fixed, pts)
    np.testing.assert_array_equal(p, [[0, 0, 0], [0, 0, 0], [3, 2, 4]])
    np.testing.assert_array_equal(q, [[0, 0, 0], [0, 0, 0], [1, 1, 2]])
    with pytest.raises(ValueError):
        O.port_landmarks_init(grid, fixed, o[None, :] + (-1.5, 0.0, 0.0))
    with pytest.raises(ValueError):
        O.port_landmarks_init(grid, fixed, o[None, :] + (0.0, 0.0, 8.2))
