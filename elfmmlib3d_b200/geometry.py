"""Seeded synthetic geometries and densities of the benchmark shapes.

The reference reads Cart3D ``.tri`` meshes (src/trilib.f:59, examples/*.tri);
its benchmark configurations are synthetic, so they are generated here:

  * ``icosphere(level)``: unit sphere, icosahedron refined ``level`` times
    (20*4**level flat triangles, outward orientation).
  * ``planar_fault(...)``: rectangular fault plane split into right triangles.
  * ``shell_targets`` / ``box_targets``: off-surface targets.

All functions return numpy float64 arrays in the reference layouts
(triangles (n,3,3), normals (n,3), centroids (n,3)).
"""
import numpy as np


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], float)
    v /= np.linalg.norm(v, axis=1)[:, None]
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                  [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], int)
    return v, f


def icosphere(level, radius=1.0):
    """Vertices (nv,3) and faces (nf,3) of the refined icosahedron (midpoints
    pushed to the sphere; vectorised, shared edges deduplicated)."""
    v, f = _icosahedron()
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0].astype(np.int64) * (len(v) + 1) + e[:, 1]
        uk, inv = np.unique(key, return_inverse=True)
        a = uk // (len(v) + 1)
        b = uk % (len(v) + 1)
        mid = (v[a] + v[b]) / 2.0
        mid /= np.linalg.norm(mid, axis=1)[:, None]
        nf = len(f)
        m = inv.reshape(3, nf).T + len(v)
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([f[:, 0], ab, ca], 1), np.stack([f[:, 1], bc, ab], 1),
                            np.stack([f[:, 2], ca, bc], 1), np.stack([ab, bc, ca], 1)])
        v = np.vstack([v, mid])
    return v * radius, f


def triangles_from_mesh(verts, faces):
    """(triangles (n,3,3), normals (n,3), centroids (n,3)) with the normal of
    the vertex order (trilib.f:243 triangle_norm) and centroids = vertex mean."""
    tri = verts[faces]
    e1 = tri[:, 1] - tri[:, 0]
    e2 = tri[:, 2] - tri[:, 1]
    nrm = np.cross(e1, e2)
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    cen = tri.mean(axis=1)
    return np.ascontiguousarray(tri), np.ascontiguousarray(nrm), np.ascontiguousarray(cen)


def sphere_triangles(level, radius=1.0):
    v, f = icosphere(level, radius)
    tri, nrm, cen = triangles_from_mesh(v, f)
    # orient outward
    flip = np.einsum("ij,ij->i", nrm, cen) < 0
    if flip.any():
        tri[flip] = tri[flip][:, [0, 2, 1]]
        tri, nrm, cen = triangles_from_mesh(tri.reshape(-1, 3), np.arange(3 * len(tri)).reshape(-1, 3))
    return tri, nrm, cen


def box_targets(m, seed, lo=-2.0, hi=2.0, rmin=1.1):
    """m targets uniform in [lo,hi]^3 with |x| > rmin (rejection sampling)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((0, 3))
    while len(out) < m:
        x = rng.uniform(lo, hi, size=(2 * m, 3))
        x = x[np.linalg.norm(x, axis=1) > rmin]
        out = np.vstack([out, x])
    return np.ascontiguousarray(out[:m])


def shell_targets(m, seed, r0=1.05, r1=3.0):
    """m targets uniform in the shell r0 < |x| < r1."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(m, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    u = rng.uniform(size=m)
    r = (r0 ** 3 + u * (r1 ** 3 - r0 ** 3)) ** (1.0 / 3.0)
    return np.ascontiguousarray(d * r[:, None])


def planar_fault(nl, nw, length=40.0, width=20.0, dip_deg=45.0, top_depth=1.0, strike_deg=0.0,
                 center_xy=(0.0, 0.0)):
    """Rectangular fault of nl x nw cells, two right triangles per cell
    (2*nl*nw triangles), top edge at z = -top_depth, dipping dip_deg downwards.
    Returns (triangles, normals, centroids, along-strike unit vector)."""
    s = np.deg2rad(strike_deg)
    d = np.deg2rad(dip_deg)
    ustrike = np.array([np.cos(s), np.sin(s), 0.0])
    horiz = np.array([-np.sin(s), np.cos(s), 0.0])
    udip = np.cos(d) * horiz + np.array([0, 0, -np.sin(d)])
    origin = np.array([center_xy[0], center_xy[1], -top_depth]) - 0.5 * length * ustrike
    a = np.linspace(0.0, length, nl + 1)
    b = np.linspace(0.0, width, nw + 1)
    P = origin[None, None, :] + a[:, None, None] * ustrike[None, None, :] + b[None, :, None] * udip[None, None, :]
    i, j = np.meshgrid(np.arange(nl), np.arange(nw), indexing="ij")
    i = i.ravel()
    j = j.ravel()
    p00, p10, p01, p11 = P[i, j], P[i + 1, j], P[i, j + 1], P[i + 1, j + 1]
    t1 = np.stack([p00, p10, p11], axis=1)
    t2 = np.stack([p00, p11, p01], axis=1)
    tri = np.empty((2 * len(i), 3, 3))
    tri[0::2] = t1
    tri[1::2] = t2
    tri, nrm, cen = triangles_from_mesh(tri.reshape(-1, 3), np.arange(3 * len(tri)).reshape(-1, 3))
    return tri, nrm, cen, ustrike


def tapered_slip(cen, ustrike, length, width, top_depth, dip_deg, noise, seed):
    """cos^2-window slip along strike plus `noise` * N(0,1) per component."""
    rng = np.random.default_rng(seed)
    d = np.deg2rad(dip_deg)
    # along-strike and down-dip coordinates in [0,1]
    xs = (cen @ ustrike + 0.5 * length) / length
    zs = (-cen[:, 2] - top_depth) / (width * np.sin(d)) if np.sin(d) > 0 else np.zeros(len(cen))
    win = (np.sin(np.pi * np.clip(xs, 0, 1)) * np.sin(np.pi * np.clip(zs, 0, 1))) ** 2
    return win[:, None] * ustrike[None, :] + noise * rng.normal(size=(len(cen), 3))
