"""Flat-triangle geometry I/O (efmm_tri_read / _write / _refine / _build, the
reference's atrireadchk, atriwrite, matlab/atrirefine.m and buildtri) on the
CPU: round trips, the refinement's vertex and face order, the triangle
arrays against plain numpy, and the reference's error codes."""
import os

import numpy as np
import pytest

import elfmmlib3d_b200 as E
from elfmmlib3d_b200 import geometry as G


def _octahedron():
    v = np.array([[1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=float)
    f = np.array([[1, 2, 5], [2, 3, 5], [3, 4, 5], [4, 1, 5], [2, 1, 6], [3, 2, 6], [4, 3, 6], [1, 4, 6]],
                 dtype=np.int32)
    return v, f


def test_write_read_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(3)
    v = rng.normal(size=(50, 3)) * 10.0 ** rng.integers(-8, 8, size=(50, 1))
    f = rng.integers(1, 51, size=(70, 3)).astype(np.int32)
    p = tmp_path / "x.tri"
    E.write_tri(p, v, f)
    v2, f2 = E.read_tri(p)
    assert np.array_equal(v2, v) and np.array_equal(f2, f)


def test_read_fortran_exponents_and_free_format(tmp_path):
    p = tmp_path / "y.tri"
    p.write_text(" 3 1\n 0.1D+01 0.0 -.5E+00\n 2.0 0.25d0\n 1e-3 0 0 1\n 1 2\n 3\n")
    v, f = E.read_tri(p)
    assert np.array_equal(v, [[1.0, 0.0, -0.5], [2.0, 0.25, 1e-3], [0.0, 0.0, 1.0]])
    assert np.array_equal(f, [[1, 2, 3]])


def test_read_error_codes(tmp_path):
    import ctypes
    L = E.load()
    nv, nf = ctypes.c_int(), ctypes.c_int()
    missing = os.fsencode(str(tmp_path / "none.tri"))
    assert L.efmm_tri_read(missing, None, 0, ctypes.byref(nv), None, 0, ctypes.byref(nf)) == 1
    p = tmp_path / "z.tri"
    E.write_tri(p, *_octahedron())
    v = np.zeros((6, 3))
    fa = np.zeros((8, 3), dtype=np.int32)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    assert L.efmm_tri_read(os.fsencode(str(p)), dp(v), 5, ctypes.byref(nv), ip(fa), 8, ctypes.byref(nf)) == 2
    assert (nv.value, nf.value) == (6, 8)
    assert L.efmm_tri_read(os.fsencode(str(p)), dp(v), 6, ctypes.byref(nv), ip(fa), 7, ctypes.byref(nf)) == 3
    assert L.efmm_tri_read(os.fsencode(str(p)), dp(v), 6, ctypes.byref(nv), ip(fa), 8, ctypes.byref(nf)) == 0
    bad = tmp_path / "bad.tri"
    bad.write_text("2 1\n0 0 0\n1 1 1\n1 2 3\n")  # index 3 > nverts
    with pytest.raises(ValueError):
        E.read_tri(bad)
    with pytest.raises(OSError):
        E.read_tri(tmp_path / "none.tri")


def _refine_numpy(v, f):
    """matlab/atrirefine.m restated with numpy (0-based work, 1-based out)."""
    nv, nf = len(v), len(f)
    a, b, c = f[:, 0] - 1, f[:, 1] - 1, f[:, 2] - 1
    v1 = np.vstack([v, (v[a] + v[b]) / 2, (v[b] + v[c]) / 2, (v[c] + v[a]) / 2])
    m12 = nv + np.arange(nf) + 1
    m23 = nv + nf + np.arange(nf) + 1
    m31 = nv + 2 * nf + np.arange(nf) + 1
    f1 = np.vstack([np.stack([f[:, 0], m12, m31], 1), np.stack([f[:, 1], m23, m12], 1),
                    np.stack([f[:, 2], m31, m23], 1), np.stack([m12, m23, m31], 1)])
    return v1, f1


def test_refine_matches_restatement_and_conserves_area():
    v, f = _octahedron()
    v1, f1 = E.refine_tri(v, f)
    vr, fr = _refine_numpy(v, f)
    assert np.array_equal(v1, vr) and np.array_equal(f1, fr)
    _, _, _, a0 = E.build_tri(v, f)
    _, _, n1, a1 = E.build_tri(v1, f1)
    assert a1.sum() == pytest.approx(a0.sum(), rel=1e-14)
    assert len(f1) == 4 * len(f)


def test_build_matches_numpy_and_package_geometry():
    v, f = _octahedron()
    v2, f2 = E.refine_tri(*E.refine_tri(v, f))
    tri, cen, nrm, area = E.build_tri(v2, f2)
    T = v2[f2 - 1]
    assert np.array_equal(tri, T)
    assert np.allclose(cen, T.mean(axis=1), rtol=0, atol=1e-15)
    cr = np.cross(T[:, 1] - T[:, 0], T[:, 2] - T[:, 0])
    assert np.allclose(area, 0.5 * np.linalg.norm(cr, axis=1), rtol=1e-14)
    assert np.allclose(nrm, cr / np.linalg.norm(cr, axis=1, keepdims=True), atol=1e-14)
    # outward normals of a closed, positively oriented surface: sum of
    # area-weighted normals vanishes, and they point away from the centre
    assert np.abs((area[:, None] * nrm).sum(axis=0)).max() < 1e-13
    assert np.all(np.einsum("ij,ij->i", nrm, cen) > 0)
    # the same triangle arrays as the package's own icosphere builder gives
    # for a mesh written and read back
    t4, n4, c4 = G.sphere_triangles(1)
    verts = t4.reshape(-1, 3)
    faces = np.arange(1, len(verts) + 1, dtype=np.int32).reshape(-1, 3)
    tri2, cen2, nrm2, _ = E.build_tri(verts, faces)
    assert np.array_equal(tri2, t4)
    assert np.allclose(nrm2, n4, atol=1e-14) and np.allclose(cen2, c4, atol=1e-15)


REF_MESH = "/root/reference/matlab/sphere320.a.tri"


@pytest.mark.skipif(not os.path.exists(REF_MESH), reason="reference mesh not present")
def test_reads_a_reference_mesh():
    """The reference ships .tri meshes of the sphere with its MATLAB
    examples; the reader takes one as is (320 faces on the unit sphere,
    closed and outward oriented)."""
    v, f = E.read_tri(REF_MESH)
    assert v.shape == (960, 3) and f.shape == (320, 3)
    tri, cen, nrm, area = E.build_tri(v, f)
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-12)
    assert np.abs((area[:, None] * nrm).sum(axis=0)).max() < 1e-12
    assert np.all(np.einsum("ij,ij->i", nrm, cen) > 0)
