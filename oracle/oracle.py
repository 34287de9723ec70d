"""ctypes front end for the CPU oracle (oracle.c, image.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU legs of ``bench.py``; never by the product package.  Array layouts follow the
reference's Fortran column-major conventions: ``triangle(3,3,n)`` is a C array
of shape (n,3,3) [tri][vertex][xyz], ``sigma(3,n)`` is (n,3), ``strain(3,3,n)``
is (n,3,3) stored so that ``strain[k].ravel()[3*j+i] = strain(i,j,k)``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _stale():
    if not os.path.exists(_SO):
        return True
    t = os.path.getmtime(_SO)
    return any(os.path.getmtime(os.path.join(_HERE, f)) > t for f in ("oracle.c", "image.c", "image_gen.h"))


def lib():
    global _lib
    if _lib is None:
        if _stale():
            build()
        _lib = ctypes.CDLL(_SO)
        _lib.oracle_tree_build.restype = ctypes.c_int
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def c64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def frame(tri):
    tri = c64(tri, (3, 3))
    rot = np.zeros(9)
    v = np.zeros(6)
    lib().oracle_frame(_d(tri), _d(rot), _d(v))
    return rot.reshape(3, 3), v.reshape(3, 2)


def tables(tri, target, self=False):
    """Derivative tables R (3,3,3) [|a|<=2] and B (5,5,5) [|a|<=4] for one triangle."""
    tri = c64(tri, (3, 3))
    tg = c64(target, (3,))
    r = np.zeros(27)
    b = np.zeros(125)
    lib().oracle_tables_flat(_d(tri), _d(tg), ctypes.c_int(int(self)), _d(r), _d(b))
    return r.reshape(3, 3, 3), b.reshape(5, 5, 5)


def slp_one(rlam, rmu, tri, sigma, target, self=False, ifstrain=True):
    u = np.zeros(3)
    e = np.zeros(9)
    lib().oracle_slp_one(ctypes.c_double(rlam), ctypes.c_double(rmu), _d(c64(tri, (3, 3))),
                         _d(c64(sigma, (3,))), ctypes.c_int(int(self)), _d(c64(target, (3,))),
                         ctypes.c_int(int(ifstrain)), _d(u), _d(e))
    return u, e.reshape(3, 3).T.copy()


def dlp_one(rlam, rmu, tri, sigma, target, self=False, ifstrain=True):
    u = np.zeros(3)
    e = np.zeros(9)
    lib().oracle_dlp_one(ctypes.c_double(rlam), ctypes.c_double(rmu), _d(c64(tri, (3, 3))),
                         _d(c64(sigma, (3,))), ctypes.c_int(int(self)), _d(c64(target, (3,))),
                         ctypes.c_int(int(ifstrain)), _d(u), _d(e))
    return u, e.reshape(3, 3).T.copy()


def direct(rlam, rmu, triangles, centroids, sigma_sl=None, sigma_dl=None, targets=None,
           rows=None, trows=None, ifstrain=True):
    """Direct O(N^2) sum (el3dtriadirecttarg, elfmm3dtria.f:1483).

    Returns (ptfrc (n,3), strain (n,3,3), ptfrctarg (m,3), straintarg (m,3,3)) with
    strain[k][i][j] = strain(i,j,k).  ``rows``/``trows`` = (start, stop) restrict which
    evaluation points are computed (others stay zero).
    """
    tri = c64(triangles).reshape(-1, 3, 3)
    n = tri.shape[0]
    src = c64(centroids).reshape(n, 3)
    tg = c64(targets if targets is not None else np.zeros((0, 3))).reshape(-1, 3)
    m = tg.shape[0]
    ssl = c64(sigma_sl if sigma_sl is not None else np.zeros((n, 3))).reshape(n, 3)
    sdl = c64(sigma_dl if sigma_dl is not None else np.zeros((n, 3))).reshape(n, 3)
    pt = np.zeros((n, 3))
    st = np.zeros((n, 9))
    ptt = np.zeros((max(m, 1), 3))
    stt = np.zeros((max(m, 1), 9))
    r0, r1 = rows if rows is not None else (0, n)
    t0, t1 = trows if trows is not None else (0, m)
    I = ctypes.c_int
    lib().oracle_direct(ctypes.c_double(rlam), ctypes.c_double(rmu), I(n), _d(tri), _d(src),
                        I(sigma_sl is not None), _d(ssl), I(sigma_dl is not None), _d(sdl),
                        I(1), _d(pt), I(int(ifstrain)), _d(st), I(m), _d(tg), I(1), _d(ptt),
                        I(int(ifstrain)), _d(stt), I(r0), I(r1), I(t0), I(t1))
    st = st.reshape(n, 3, 3).transpose(0, 2, 1).copy()
    stt = stt.reshape(-1, 3, 3).transpose(0, 2, 1)[:m].copy()
    return pt, st, ptt[:m].copy(), stt


def image_direct(rlam, rmu, triangles, normals, sigma_sl, sigma_dl, targets, level=-1):
    """Image part of the half-space potentials (image.c; the image of
    src/el3greenh.f:643-787 integrated over every triangle), at targets in
    z < 0: returns (u (m,3), strain (m,3,3)).  level >= 0: 4**level uniform
    sub-triangles per triangle (as mindlin.image_direct); level < 0:
    refinement by distance to the reflected target.  None disables a layer."""
    tri = c64(triangles).reshape(-1, 3, 3)
    n = tri.shape[0]
    nrm = c64(normals).reshape(n, 3)
    tg = c64(targets).reshape(-1, 3)
    m = tg.shape[0]
    ssl = c64(sigma_sl).reshape(n, 3) if sigma_sl is not None else None
    sdl = c64(sigma_dl).reshape(n, 3) if sigma_dl is not None else None
    u = np.zeros((m, 3))
    e = np.zeros((m, 3, 3))
    f = lib().oracle_image_direct
    f.restype = ctypes.c_int
    ier = f(ctypes.c_double(rlam), ctypes.c_double(rmu), ctypes.c_int(n), _d(tri), _d(nrm),
            _d(ssl) if ssl is not None else None, _d(sdl) if sdl is not None else None, ctypes.c_int(m),
            _d(tg), ctypes.c_int(int(level)), _d(u), _d(e))
    if ier:
        raise ValueError(f"oracle_image_direct ier={ier}")
    return u, e


def image_direct_adaptive(rlam, rmu, triangles, normals, sigma_sl, sigma_dl, targets, eps=1e-11, maxdepth=40):
    """Image part as image_direct, every pair and layer integrated by the
    adaptive scheme of the reference's tria3adam (src/tria3adamar.f:33-395)
    to relative tolerance eps with at most maxdepth halvings.  Returns
    (u (m,3), strain (m,3,3), pairs that reached the depth cap)."""
    tri = c64(triangles).reshape(-1, 3, 3)
    n = tri.shape[0]
    nrm = c64(normals).reshape(n, 3)
    tg = c64(targets).reshape(-1, 3)
    m = tg.shape[0]
    ssl = c64(sigma_sl).reshape(n, 3) if sigma_sl is not None else None
    sdl = c64(sigma_dl).reshape(n, 3) if sigma_dl is not None else None
    u = np.zeros((m, 3))
    e = np.zeros((m, 3, 3))
    capped = ctypes.c_int(0)
    f = lib().oracle_image_direct_adaptive
    f.restype = ctypes.c_int
    ier = f(ctypes.c_double(rlam), ctypes.c_double(rmu), ctypes.c_int(n), _d(tri), _d(nrm),
            _d(ssl) if ssl is not None else None, _d(sdl) if sdl is not None else None, ctypes.c_int(m),
            _d(tg), ctypes.c_double(eps), ctypes.c_int(int(maxdepth)), _d(u), _d(e), ctypes.byref(capped))
    if ier:
        raise ValueError(f"oracle_image_direct_adaptive ier={ier}")
    return u, e, capped.value


class Tree:
    """Bit-exact restatement of d3tstrcr (d3tstrcr.f:31).  All ids are 1-based."""

    def __init__(self, sources, targets, nbox, mindlin=False):
        src = c64(sources).reshape(-1, 3)
        tg = c64(targets if targets is not None else np.zeros((0, 3))).reshape(-1, 3)
        n, nt = src.shape[0], tg.shape[0]
        L = lib()
        ier = L.oracle_tree_build(ctypes.c_int(n), _d(src), ctypes.c_int(nt), _d(tg),
                                  ctypes.c_int(nbox), ctypes.c_int(int(mindlin)))
        if ier:
            raise RuntimeError(f"oracle tree ier={ier}")
        nb = ctypes.c_int()
        nl = ctypes.c_int()
        cen = np.zeros(3)
        size = ctypes.c_double()
        lc = np.zeros(5, dtype=np.int32)
        L.oracle_tree_info(ctypes.byref(nb), ctypes.byref(nl), _d(cen), ctypes.byref(size), _i(lc))
        self.nboxes, self.nlev = nb.value, nl.value
        self.center, self.size = cen, size.value
        boxes = np.zeros((self.nboxes, 20), dtype=np.int32)
        iz = np.zeros(max(n, 1), dtype=np.int32)
        izt = np.zeros(max(nt, 1), dtype=np.int32)
        laddr = np.zeros((self.nlev + 1, 2), dtype=np.int32)
        lstart = np.zeros((5, self.nboxes + 1), dtype=np.int32)
        litems = np.zeros(max(int(lc.sum()), 1), dtype=np.int32)
        L.oracle_tree_get(_i(boxes), _i(iz), _i(izt), _i(laddr), ctypes.c_int(n), ctypes.c_int(nt),
                          _i(lstart), _i(litems))
        self.boxes, self.iz, self.iztarg, self.laddr = boxes, iz[:n], izt[:nt], laddr
        self.lists = {}
        off = 0
        for t in range(1, 6):
            cnt = int(lc[t - 1])
            items = litems[off:off + cnt]
            off += cnt
            st = lstart[t - 1]
            self.lists[t] = [items[st[b]:st[b + 1]].copy() for b in range(self.nboxes)]
