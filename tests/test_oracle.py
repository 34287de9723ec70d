"""CPU tests of the oracle (test infrastructure): pins against the integral
definitions, exact identities and tree invariants."""
import numpy as np
import pytest

from conftest import golden, rel
from elfmmlib3d_b200 import geometry as G


def test_tables_match_definition_quadrature(oracle):
    g = golden("golden_tables.npz")
    for i, x in enumerate(g["targets"]):
        R, B = oracle.tables(g["tri"], x)
        r = np.array([R[tuple(a)] for a in g["r_idx"]])
        b = np.array([B[tuple(a)] for a in g["b_idx"]])
        assert np.abs(r - g["R"][i]).max() <= 1e-11 * np.abs(g["R"][i]).max()
        assert np.abs(b - g["B"][i]).max() <= 1e-11 * np.abs(g["B"][i]).max()


def test_self_value_is_two_sided_limit(oracle):
    """On-surface (iquad = 0) values = average of the limits z0 -> 0+ and 0-
    (principal value / finite part, src/triahquad.f:4037-4055)."""
    tri = np.array([[0.1, 0.2, 0.05], [1.2, 0.1, -0.1], [0.4, 1.1, 0.2]])
    rot, v = oracle.frame(tri)
    c = tri.mean(0)
    n = rot[:, 2]
    R0, B0 = oracle.tables(tri, c, self=True)
    hs = np.array([1e-3, 2e-3, 4e-3])
    A = np.vander(hs, 3, increasing=True)
    lim = []
    for sg in (1, -1):
        vals = [oracle.tables(tri, c + sg * h * n) for h in hs]
        Rl = np.linalg.solve(A, np.stack([x[0].ravel() for x in vals]))[0].reshape(R0.shape)
        Bl = np.linalg.solve(A, np.stack([x[1].ravel() for x in vals]))[0].reshape(B0.shape)
        lim.append((Rl, Bl))
    Ra = (lim[0][0] + lim[1][0]) / 2
    Ba = (lim[0][1] + lim[1][1]) / 2
    assert np.abs(Ra - R0).max() < 1e-6 * np.abs(R0).max()
    assert np.abs(Ba - B0).max() < 1e-6 * np.abs(B0).max()
    assert abs(lim[0][0][0, 0, 1] - 2 * np.pi) < 1e-6  # solid angle jumps by 4 pi


def test_double_layer_rigid_body_identity(oracle):
    """Constant displacement jump b on a closed polyhedron (outward normals):
    u = -4 pi b inside, 0 outside, -2 pi b on the surface, zero strain."""
    tri, nrm, cen = G.sphere_triangles(1)
    b = np.array([0.3, -0.7, 0.5])
    tg = np.array([[0.1, 0.2, -0.1], [0.0, 0.0, 0.3], [2.0, 1.0, 0.5], [-1.5, 0.3, 0.2]])
    pt, st, ptt, stt = oracle.direct(3.2, 2.3, tri, cen, None, np.tile(b, (len(cen), 1)), tg)
    assert np.allclose(ptt[:2], -4 * np.pi * b, atol=1e-12)
    assert np.allclose(ptt[2:], 0, atol=1e-12)
    assert np.allclose(pt, -2 * np.pi * b, atol=1e-12)
    assert np.abs(stt).max() < 1e-12 and np.abs(st).max() < 1e-12


def test_oracle_direct_reproduces_golden(oracle):
    g = golden("golden_sphere320.npz")
    pt, st, ptt, stt = oracle.direct(float(g["rlam"]), float(g["rmu"]), g["tri"], g["cen"], g["ssl"],
                                     g["sdl"], g["tgt"], rows=(0, 8), trows=(0, 4))
    assert rel(pt[:8], g["pt"][:8]) < 1e-13 and rel(st[:8], g["st"][:8]) < 1e-13
    assert rel(ptt[:4], g["ptt"][:4]) < 1e-13 and rel(stt[:4], g["stt"][:4]) < 1e-13


@pytest.mark.parametrize("mindlin", [False, True])
def test_tree_invariants(oracle, mindlin):
    if mindlin:
        tri, nrm, src, _ = G.planar_fault(30, 15)
        tgt = np.zeros((0, 3))
        nbox = 240
    else:
        tri, nrm, src = G.sphere_triangles(3)
        tgt = G.box_targets(300, 3)
        nbox = 40
    T = oracle.Tree(src, tgt, nbox, mindlin)
    B = T.boxes
    assert sorted(T.iz.tolist()) == list(range(1, len(src) + 1))
    for b in range(T.nboxes):
        kids = [k for k in B[b, 5:13] if k > 0]
        if kids:
            assert sum(B[k - 1, 14] for k in kids) == B[b, 14]
            assert sum(B[k - 1, 16] for k in kids) == B[b, 16]
        else:
            assert B[b, 14] <= nbox and B[b, 16] <= nbox
    for b in range(T.nboxes):
        for j in T.lists[1][b]:
            assert b + 1 in T.lists[1][j - 1].tolist()
        for j in T.lists[3][b]:
            assert b + 1 in T.lists[4][j - 1].tolist()
    if mindlin:
        assert T.center[2] == 0.0


def test_c1_fixture_geometry_regenerates():
    """The C1 fixture stores the densities and targets; its triangles are
    regenerated from the package's icosphere and checked by hash."""
    import hashlib
    from elfmmlib3d_b200 import geometry as G
    from conftest import golden
    g = golden("golden_c1_sphere5120.npz")
    tri, nrm, cen = G.sphere_triangles(4)
    assert hashlib.sha256(np.ascontiguousarray(tri).tobytes()).hexdigest() == str(g["tri_sha256"])
    assert g["u_c"].shape == (256, 3) and g["e_t"].shape == (256, 3, 3)
    assert np.all(np.linalg.norm(g["tgt"], axis=1) > 1.1)
