"""The product's free-space analytic near field (tri_integrals.cuh, the code
the device near field runs, evaluated on the host through
efmm_pair_eval_host) against the oracle's numerical integration of the
same layer potentials (oracle.c slp_one / dlp_one) for single triangles:
targets far, close above the plane, in the plane outside the triangle,
collinear with an edge, and the on-surface self evaluation at the centroid.
No device is used."""
import ctypes

import numpy as np
import pytest

_dp = ctypes.POINTER(ctypes.c_double)


def _pair(L, rlam, rmu, tri, ssl, sdl, x, self):
    u, e6 = np.zeros(3), np.zeros(6)
    p = lambda a: np.ascontiguousarray(a, float).ctypes.data_as(_dp) if a is not None else None
    keep = [np.ascontiguousarray(a, float) for a in (tri, x)]
    ier = L.efmm_pair_eval_host(ctypes.c_double(rlam), ctypes.c_double(rmu), keep[0].ctypes.data_as(_dp), p(ssl),
                                p(sdl), keep[1].ctypes.data_as(_dp), ctypes.c_int(int(self)), u.ctypes.data_as(_dp),
                                e6.ctypes.data_as(_dp))
    assert ier == 0
    e = np.array([[e6[0], e6[3], e6[4]], [e6[3], e6[1], e6[5]], [e6[4], e6[5], e6[2]]])
    return u, e


def _targets(tri, rng):
    a, b, c = tri
    cen = (a + b + c) / 3
    nrm = np.cross(b - a, c - a)
    nrm /= np.linalg.norm(nrm)
    diam = max(np.linalg.norm(b - a), np.linalg.norm(c - b), np.linalg.norm(a - c))
    out = [(cen, True)]
    out.append((cen + 5.0 * diam * rng.normal(size=3), False))                 # far
    out.append((cen + 0.05 * diam * nrm + 0.2 * diam * (b - a), False))       # close above
    out.append((cen - 0.01 * diam * nrm, False))                              # just below the centroid
    out.append((a + 1.7 * (b - a), False))                                     # in-plane, collinear with an edge
    out.append((cen + 1.3 * (cen - c), False))                                 # in-plane, outside
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_pair_matches_oracle(lib, oracle, seed):
    L = ctypes.CDLL(lib.library_path())
    L.efmm_pair_eval_host.restype = ctypes.c_int
    rng = np.random.default_rng(seed)
    worst = {"slp": [0.0, 0.0], "dlp": [0.0, 0.0]}
    for _ in range(4):
        tri = rng.normal(size=(3, 3))
        rlam, rmu = rng.uniform(0.5, 2.0, 2)
        sig = rng.normal(size=3)
        for x, self in _targets(tri, rng):
            for kind in ("slp", "dlp"):
                up, ep = _pair(L, rlam, rmu, tri, sig if kind == "slp" else None, sig if kind == "dlp" else None,
                               x, self)
                f = oracle.slp_one if kind == "slp" else oracle.dlp_one
                uo, eo = f(rlam, rmu, tri, sig, x, self=self)
                worst[kind][0] = max(worst[kind][0], np.abs(up - uo).max() / np.abs(uo).max())
                worst[kind][1] = max(worst[kind][1], np.abs(ep - eo).max() / np.abs(eo).max())
    for kind, (wu, we) in worst.items():
        assert wu < 5e-12 and we < 5e-12, (kind, wu, we)


def test_pair_rejects_missing_densities(lib):
    L = ctypes.CDLL(lib.library_path())
    L.efmm_pair_eval_host.restype = ctypes.c_int
    tri = np.eye(3)
    u, e6 = np.zeros(3), np.zeros(6)
    ier = L.efmm_pair_eval_host(ctypes.c_double(1.0), ctypes.c_double(1.0), tri.ctypes.data_as(_dp), None, None,
                                tri.ctypes.data_as(_dp), ctypes.c_int(0), u.ctypes.data_as(_dp),
                                e6.ctypes.data_as(_dp))
    assert ier == 16
