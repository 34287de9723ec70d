"""The oracle's half-space image kernels (oracle/mindlin.py), pinned by the
physics the reference's image part must satisfy: the total (free + image)
field of a point force and of a point displacement jump is traction-free on
z = 0, the total Green's function is reciprocal, and the oracle's kernel
quadrature reproduces the analytic free-space layers of oracle.c."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def mind():
    from oracle import mindlin as M
    return M


def _unit(v):
    return v / np.linalg.norm(v)


def test_total_field_traction_free_on_surface(mind):
    tr = mind.traction_on_surface()
    rng = np.random.default_rng(3)
    for _ in range(8):
        lam, mu = rng.uniform(0.3, 3.0, 2)
        x, y = rng.uniform(-3, 3, 2)
        s = np.array([*rng.uniform(-1, 1, 2), -rng.uniform(0.1, 3.0)])
        b, f = rng.normal(size=3), rng.normal(size=3)
        n = _unit(rng.normal(size=3))
        t = np.array(tr(lam, mu, x, y, *s, *b, *n, *f), dtype=float)
        # scale: the free-space traction of the same sources at that point
        ref = np.abs(t).max() + 1.0 / (1.0 + np.hypot(x - s[0], y - s[1]) ** 2 + s[2] ** 2)
        assert np.abs(t).max() < 1e-12 * ref


def test_total_green_function_reciprocal(mind):
    fsl_i, _ = mind.kernels("image")
    fsl_f, _ = mind.kernels("free")
    rng = np.random.default_rng(5)
    for _ in range(6):
        lam, mu = rng.uniform(0.3, 3.0, 2)
        P = np.array([*rng.uniform(-1, 1, 2), -rng.uniform(0.1, 2)])
        Q = np.array([*rng.uniform(-1, 1, 2), -rng.uniform(0.1, 2)])
        a = np.array(fsl_i(lam, mu, *P, *Q), float) + np.array(fsl_f(lam, mu, *P, *Q), float)
        b = np.array(fsl_i(lam, mu, *Q, *P), float) + np.array(fsl_f(lam, mu, *Q, *P), float)
        G = np.array([[a[9 * k + i] for i in range(3)] for k in range(3)])   # G[k][i](P; Q)
        H = np.array([[b[9 * k + i] for i in range(3)] for k in range(3)])   # G[k][i](Q; P)
        assert np.abs(G - H.T).max() < 1e-13 * np.abs(G).max()


def test_kernel_quadrature_reproduces_free_space_layers(mind, oracle):
    tri = np.array([[[0.1, 0.2, -1.0], [0.5, 0.1, -1.2], [0.2, 0.6, -0.9]]])
    n = _unit(np.cross(tri[0, 1] - tri[0, 0], tri[0, 2] - tri[0, 1]))
    X = np.array([[1.5, -0.7, -2.2], [-1.1, 0.4, -0.3]])
    sd = np.array([[0.3, -1.2, 0.8]])
    ss = np.array([[1.1, 0.2, -0.4]])
    ud, ed = mind.image_direct(1.3, 0.7, tri, n[None], None, sd, X, level=3, part="free")
    us, es = mind.image_direct(1.3, 0.7, tri, n[None], ss, None, X, level=3, part="free")
    for i in range(2):
        uo, eo = oracle.dlp_one(1.3, 0.7, tri[0], sd[0], X[i])
        assert np.abs(ud[i] - uo).max() < 1e-12 * np.abs(uo).max()
        assert np.abs(ed[i] - eo).max() < 1e-12 * np.abs(eo).max()
        uo, eo = oracle.slp_one(1.3, 0.7, tri[0], ss[0], X[i])
        assert np.abs(us[i] - uo).max() < 1e-12 * np.abs(uo).max()
        assert np.abs(es[i] - eo).max() < 1e-12 * np.abs(eo).max()
