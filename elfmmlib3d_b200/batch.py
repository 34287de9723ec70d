"""Many independent half-space problems of uneven sizes (the batched
uneven-geometry configuration): every problem is a half-space
self-evaluation at its centroids -- the direct arrival (free-space plan on
the centroids) plus the image part (image plan on the reflected centroids),
the sum the reference's drivers form (examples/elhfmm3dtria_self_iter_dr.f:
331-385) -- with one right-hand side each.

Worker threads each own a free-space and an image plan (each plan has its
own CUDA stream) and take the problems from one queue, largest first, so
that the device runs several problems at once and the small ones fill in
behind the large ones.  The plans' native calls release the interpreter
lock, so the workers' passes overlap on the device.
"""
import queue
import threading
import time

import numpy as np

from . import Plan, hs_image_direct, ElfmmError

__all__ = ["halfspace_many", "fault_problem"]


def fault_problem(ntri, strike_deg, dip_deg, depth, seed, length=40.0, width=20.0):
    """A planar fault of about ntri right triangles (aspect length : width,
    cells of 2 triangles), top edge at z = -depth, one slip vector N(0,1) per
    triangle.  Returns (triangles, normals, centroids, slip)."""
    from . import geometry as G
    nw = max(1, int(round(np.sqrt(ntri * width / (2.0 * length)))))
    nl = max(1, int(round(ntri / (2.0 * nw))))
    tri, nrm, cen, _ = G.planar_fault(nl, nw, length, width, dip_deg, depth, strike_deg)
    slip = np.random.default_rng(seed).normal(size=cen.shape)
    return tri, nrm, cen, slip


def halfspace_many(problems, iprec=2, rlam=1.0, rmu=1.0, precision=1, workers=4, device=0, check=0):
    """Half-space self-evaluation of every problem.

    problems: list of (triangles (n,3,3), normals (n,3), centroids (n,3),
    sigma_sl (n,3) or None, sigma_dl (n,3) or None), all below z = 0.
    precision 1: the mixed form (FP32 far field and stored-block products,
    FP64 near-singular parts); 0: FP64.  check > 0: also the relative l2
    error of each result against the FP64 direct sums (free-space analytic +
    image refined quadrature) on its first `check` centroids.

    Returns (results, info): results[i] = (u (n,3), strain (n,3,3)) as numpy
    arrays; info = dict(seconds=wall time of all problems, per_problem=[
    seconds], errors=[(u, strain)] when checked).
    """
    import torch
    dev = torch.device("cuda", device)
    order = sorted(range(len(problems)), key=lambda i: -len(problems[i][2]))
    q = queue.Queue()
    for i in order:
        q.put(i)
    results = [None] * len(problems)
    per = [0.0] * len(problems)
    errs = [None] * len(problems)
    failures = []

    def d(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)

    def work():
        torch.cuda.set_device(dev)
        F, I = Plan(device), Plan(device)
        try:
            while True:
                try:
                    i = q.get_nowait()
                except queue.Empty:
                    return
                t0 = time.perf_counter()
                tri, nrm, cen, ssl, sdl = problems[i]
                n = len(cen)
                dtri, dnrm, dcen = d(tri), d(nrm), d(cen)
                dssl = d(np.asarray(ssl)[None]) if ssl is not None else None
                dsdl = d(np.asarray(sdl)[None]) if sdl is not None else None
                F.set_geometry(dtri, dnrm, dcen, None, iprec=iprec)
                I.set_geometry(dtri, dnrm, dcen, d(cen * np.array([1.0, 1.0, -1.0])), iprec=iprec, mindlin=True)
                uf = torch.zeros((1, n, 3), dtype=torch.float64, device=dev)
                ef = torch.zeros((1, n, 3, 3), dtype=torch.float64, device=dev)
                ui, ei = torch.zeros_like(uf), torch.zeros_like(ef)
                F.evaluate_batch(rlam, rmu, 1, dssl, dsdl, uf, ef, precision=precision)
                I.evaluate_image(rlam, rmu, 1, dssl, dsdl, ui, ei, precision=precision)
                u = (uf + ui)[0].cpu().numpy()
                e = (ef + ei)[0].cpu().numpy()
                results[i] = (u, e)
                per[i] = time.perf_counter() - t0
                if check > 0:
                    ns = min(check, n)
                    ud = torch.zeros((ns, 3), dtype=torch.float64, device=dev)
                    ed = torch.zeros((ns, 3, 3), dtype=torch.float64, device=dev)
                    F.evaluate_direct_subset(rlam, rmu, ns, dssl[0] if dssl is not None else None,
                                             dsdl[0] if dsdl is not None else None, ud, ed)
                    ier, uid, eid = hs_image_direct(rlam, rmu, tri, nrm, ssl, sdl, cen[:ns])
                    if ier:
                        raise ElfmmError(ier, "hs_image_direct")
                    ur = ud.cpu().numpy() + uid
                    er = ed.cpu().numpy() + eid
                    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
                    errs[i] = (rel(u[:ns], ur), rel(e[:ns], er))
        except Exception as ex:  # reported after the other workers finish
            failures.append(ex)
        finally:
            F.close()
            I.close()

    t0 = time.perf_counter()
    threads = [threading.Thread(target=work) for _ in range(max(1, int(workers)))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    if failures:
        raise failures[0]
    info = {"seconds": wall, "per_problem": per}
    if check > 0:
        info["errors"] = errs
    return results, info
