"""Many independent half-space problems of uneven sizes (the batched
uneven-geometry configuration): every problem is a half-space
self-evaluation at its centroids -- the direct arrival (free-space FMM on the
centroids) plus the image part (image FMM on the reflected centroids), the
sum the reference's drivers form (examples/elhfmm3dtria_self_iter_dr.f:
331-385) -- with one right-hand side each.

engine "forest" (default): all problems in one pair of plans (efmm_forest_*,
csrc/forest.cu): the problems are moved side by side in x and y, one per
column of boxes of a common root, and both trees are built as a forest whose
lists never join two problems, so that every stage is one launch over the
boxes of all problems.

engine "plans": worker threads each own a free-space and an image plan
(each plan has its own CUDA stream) and take the problems from one queue,
largest first; the plans' native calls release the interpreter lock, so the
workers' passes overlap on the device.
"""
import queue
import threading
import time

import numpy as np

from . import Plan, Forest, hs_image_direct, ElfmmError

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


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _check(problem, u, e, ns, rlam, rmu, dev, plan=None):
    """Relative l2 errors (u, strain) of a problem's result on its first ns
    centroids against the FP64 direct sums (free-space analytic + image
    refined quadrature)."""
    import torch
    tri, nrm, cen, ssl, sdl = problem
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    own = plan is None
    F = Plan(dev.index) if own else plan
    try:
        if own:
            F.set_geometry(d(tri), d(nrm), d(cen), None, iprec=2)
        ud = torch.zeros((ns, 3), dtype=torch.float64, device=dev)
        ed = torch.zeros((ns, 3, 3), dtype=torch.float64, device=dev)
        F.evaluate_direct_subset(rlam, rmu, ns, d(ssl) if ssl is not None else None,
                                 d(sdl) if sdl is not None else None, ud, ed)
    finally:
        if own:
            F.close()
    ier, uid, eid = hs_image_direct(rlam, rmu, tri, nrm, ssl, sdl, cen[:ns])
    if ier:
        raise ElfmmError(ier, "hs_image_direct")
    return _rel(u[:ns], ud.cpu().numpy() + uid), _rel(e[:ns], ed.cpu().numpy() + eid)


def halfspace_many(problems, iprec=2, rlam=1.0, rmu=1.0, precision=1, workers=4, device=0, check=0,
                   engine="forest", check_every=1):
    """Half-space self-evaluation of every problem.

    problems: list of (triangles (n,3,3), normals (n,3), centroids (n,3),
    sigma_sl (n,3) or None, sigma_dl (n,3) or None), all below z = 0.
    precision 1: the mixed form (FP32 far field and stored-block products,
    FP64 near-singular parts); 0: FP64.  check > 0: also the relative l2
    error of every check_every-th problem's result against the FP64 direct
    sums (free-space analytic + image refined quadrature) on its first
    `check` centroids.  workers: threads of the "plans" engine.

    Returns (results, info): results[i] = (u (n,3), strain (n,3,3)) as numpy
    arrays; info = dict(seconds=wall time of the evaluation, errors=[(u,
    strain) or None] when checked; "plans" also per_problem=[seconds];
    "forest" also setup / evaluate seconds).
    """
    if engine == "forest":
        return _many_forest(problems, iprec, rlam, rmu, precision, device, check, check_every)
    if engine != "plans":
        raise ValueError(f"engine {engine!r}")
    return _many_plans(problems, iprec, rlam, rmu, precision, workers, device, check, check_every)


def _many_forest(problems, iprec, rlam, rmu, precision, device, check, check_every):
    import torch
    dev = torch.device("cuda", device)
    counts = np.array([len(p[2]) for p in problems], dtype=np.int32)
    off = np.concatenate([[0], np.cumsum(counts)])
    has_sl = any(p[3] is not None for p in problems)
    has_dl = any(p[4] is not None for p in problems)
    cat = lambda j, w: np.concatenate([np.asarray(p[j], dtype=np.float64).reshape(-1, w) for p in problems])
    lay = lambda j: np.concatenate([np.zeros((len(p[2]), 3)) if p[j] is None
                                    else np.asarray(p[j], dtype=np.float64).reshape(-1, 3) for p in problems])
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    tri, nrm, cen = d(cat(0, 9)), d(cat(1, 3)), d(cat(2, 3))
    ssl = d(lay(3)) if has_sl else None
    sdl = d(lay(4)) if has_dl else None
    n = int(off[-1])
    u = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    e = torch.zeros((n, 3, 3), dtype=torch.float64, device=dev)
    F = Forest(device)
    try:
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        F.set_geometry(counts, tri, nrm, cen, iprec=iprec)
        t1 = time.perf_counter()
        F.evaluate(rlam, rmu, ssl, sdl, u, e, precision=precision)
        t2 = time.perf_counter()
    finally:
        F.close()
    uh, eh = u.cpu().numpy(), e.cpu().numpy()
    results = [(uh[off[i]:off[i + 1]], eh[off[i]:off[i + 1]]) for i in range(len(problems))]
    info = {"seconds": t2 - t0, "setup": t1 - t0, "evaluate": t2 - t1}
    if check > 0:
        info["errors"] = [_check(problems[i], *results[i], min(check, int(counts[i])), rlam, rmu, dev)
                          if i % check_every == 0 else None for i in range(len(problems))]
    return results, info


def _many_plans(problems, iprec, rlam, rmu, precision, workers, device, check, check_every):
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
                if check > 0 and i % check_every == 0:
                    errs[i] = _check(problems[i], u, e, min(check, n), rlam, rmu, dev, plan=F)
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
