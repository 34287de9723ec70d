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


def _boxes(k, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        lo = rng.uniform(-50, 50, size=3)
        ext = rng.uniform(0.1, 40, size=3)
        lo[2] = -rng.uniform(0.5, 5) - ext[2]
        out.append(np.concatenate([lo, lo + ext]))
    return np.array(out)


@pytest.mark.parametrize("k", [1, 2, 5, 16, 17, 256, 300])
def test_forest_layout_columns(k):
    """efmm_forest_layout (host code): every problem's shifted box lies inside
    its own column of level L with a margin, columns are distinct, and the
    root cube (centred on z = 0) holds every depth."""
    import elfmmlib3d_b200 as E
    bb = _boxes(k, k)
    root, shift = E.forest_layout(bb)
    L = int(root[4])
    g = 2 ** L
    assert g * g >= k and (L == 1 or (g // 2) ** 2 < k)
    assert root[2] == 0.0
    side = root[3]
    s = side / g
    cols = set()
    for b, sh in zip(bb, shift):
        lo = b[:2] + sh
        hi = b[3:5] + sh
        i = int(np.floor((lo[0] + side / 2) / s))
        j = int(np.floor((lo[1] + side / 2) / s))
        x0, y0 = -side / 2 + i * s, -side / 2 + j * s
        margin = s / 2048
        assert x0 + margin < lo[0] and hi[0] < x0 + s - margin
        assert y0 + margin < lo[1] and hi[1] < y0 + s - margin
        assert -b[2] < side / 2
        cols.add((i, j))
    assert len(cols) == k
    # the problems' boxes are centred in their columns: a shift moves only x, y
    assert shift.shape == (k, 2)


def test_forest_layout_rejects():
    import elfmmlib3d_b200 as E
    bb = _boxes(3, 1)
    bad = bb.copy()
    bad[1, 5] = 0.5                     # a centroid above the surface
    with pytest.raises(E.ElfmmError):
        E.forest_layout(bad)
    bad = bb.copy()
    bad[0, 0] = bad[0, 3] + 1           # min > max
    with pytest.raises(E.ElfmmError):
        E.forest_layout(bad)
    with pytest.raises(E.ElfmmError):
        E.forest_layout(np.zeros((0, 6)))
