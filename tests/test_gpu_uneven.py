"""Many independent half-space problems of uneven sizes and orientations
(the batched uneven-geometry configuration) through worker threads that
each own a free-space and an image plan: every problem's result against the
FP64 direct sums (free-space analytic + image refined quadrature), in the
mixed and the FP64 forms, and independent of how the problems are spread
over the workers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(k, seed):
    from elfmmlib3d_b200.batch import fault_problem
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        ntri = int(np.exp(rng.uniform(np.log(400), np.log(4000))))
        tri, nrm, cen, slip = fault_problem(ntri, rng.uniform(0, 360), rng.uniform(15, 90), rng.uniform(0.5, 5),
                                            seed=1000 * seed + i)
        out.append((tri, nrm, cen, None, slip))
    return out


@pytest.mark.parametrize("precision", [1, 0])
def test_uneven_batch_matches_direct_sums(gpu, precision):
    from elfmmlib3d_b200.batch import halfspace_many
    probs = _problems(6, 3)
    res, info = halfspace_many(probs, iprec=3, precision=precision, workers=3, check=200)
    assert len(res) == len(probs) and all(r is not None for r in res)
    worst = max(max(e) for e in info["errors"])
    print(f"precision {precision}: sizes {[len(p[2]) for p in probs]}, worst rel err {worst:.2e}, "
          f"{info['seconds']:.2f} s")
    assert worst < (1e-6 if precision == 1 else 1e-7)
    # one worker: the same results up to the order of the translations'
    # atomic sums (FP64: 1e-12; FP32 expansions: FP32 rounding)
    res1, _ = halfspace_many(probs, iprec=3, precision=precision, workers=1)
    tol = 2e-6 if precision == 1 else 1e-12
    for (u, e), (u1, e1) in zip(res, res1):
        assert np.linalg.norm(u - u1) <= tol * np.linalg.norm(u1)
        assert np.linalg.norm(e - e1) <= tol * np.linalg.norm(e1)
