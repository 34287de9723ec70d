"""Host-side checks of the batched uneven-geometry inputs: the fault
generator's triangle counts, orientation and depth (every triangle below the
free surface, as the image plan requires)."""
import numpy as np
import pytest

from elfmmlib3d_b200.batch import fault_problem


@pytest.mark.parametrize("ntri", [1000, 6603, 49506])
def test_fault_problem_sizes_and_depth(ntri):
    rng = np.random.default_rng(ntri)
    strike, dip, depth = rng.uniform(0, 360), rng.uniform(15, 90), rng.uniform(0.5, 5)
    tri, nrm, cen, slip = fault_problem(ntri, strike, dip, depth, seed=1)
    n = len(cen)
    assert tri.shape == (n, 3, 3) and nrm.shape == (n, 3) and slip.shape == (n, 3)
    assert abs(n - ntri) <= 0.05 * ntri + 4          # cells of two triangles, aspect 2:1
    assert tri[:, :, 2].max() <= -depth + 1e-12       # top edge at z = -depth, dipping down
    assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0)
    # the normal is perpendicular to the strike direction (azimuth `strike`)
    us = np.array([np.cos(np.deg2rad(strike)), np.sin(np.deg2rad(strike)), 0.0])
    assert np.abs(nrm @ us).max() < 1e-12
    # and makes the dip angle with the vertical
    assert np.allclose(np.abs(nrm[:, 2]), np.cos(np.deg2rad(dip)), atol=1e-12)
    # one slip vector N(0,1) per triangle, reproducible from the seed
    assert np.array_equal(slip, fault_problem(ntri, strike, dip, depth, seed=1)[3])
