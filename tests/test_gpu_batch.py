"""Many right-hand sides in one pass (efmm_plan_evaluate_batch) against the
same number of single evaluations on the same plan, and against the direct
sum at the iprec tolerance."""
import numpy as np
import pytest

from conftest import rel
from elfmmlib3d_b200 import geometry as G

pytestmark = pytest.mark.gpu

# the batched pass reorders the same FP64 sums (pair blocks x densities,
# wider translation tiles)
SAME = 1e-12


def _t():
    import torch
    return torch


def _plan(gpu, level=3, ntarg=120, iprec=2, seed=0):
    torch = _t()
    tri, nrm, cen = G.sphere_triangles(level)
    tg = G.box_targets(ntarg, 21 + seed)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    P = gpu.Plan(0)
    P.set_geometry(d(tri), d(nrm), d(cen), d(tg), iprec=iprec)
    return P, tri, nrm, cen, tg, d


def _single(P, d, ssl, sdl, n, m, strain=True):
    torch = _t()
    R = ssl.shape[0] if ssl is not None else sdl.shape[0]
    out = [np.zeros((R, n, 3)), np.zeros((R, n, 3, 3)), np.zeros((R, m, 3)), np.zeros((R, m, 3, 3))]
    for r in range(R):
        u = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        e = torch.zeros((n, 3, 3), dtype=torch.float64, device="cuda") if strain else None
        ut = torch.zeros((m, 3), dtype=torch.float64, device="cuda")
        et = torch.zeros((m, 3, 3), dtype=torch.float64, device="cuda") if strain else None
        P.evaluate(1.3, 0.7, d(ssl[r]) if ssl is not None else None, d(sdl[r]) if sdl is not None else None,
                   u, e, ut, et)
        out[0][r], out[2][r] = u.cpu().numpy(), ut.cpu().numpy()
        if strain:
            out[1][r], out[3][r] = e.cpu().numpy(), et.cpu().numpy()
    return out


def _batch(P, d, R, ssl, sdl, n, m, strain=True):
    torch = _t()
    u = torch.zeros((R, n, 3), dtype=torch.float64, device="cuda")
    e = torch.zeros((R, n, 3, 3), dtype=torch.float64, device="cuda") if strain else None
    ut = torch.zeros((R, m, 3), dtype=torch.float64, device="cuda")
    et = torch.zeros((R, m, 3, 3), dtype=torch.float64, device="cuda") if strain else None
    P.evaluate_batch(1.3, 0.7, R, d(ssl) if ssl is not None else None, d(sdl) if sdl is not None else None,
                     u, e, ut, et)
    return [u.cpu().numpy(), e.cpu().numpy() if strain else None, ut.cpu().numpy(),
            et.cpu().numpy() if strain else None]


@pytest.mark.parametrize("R", [1, 5, 37, 70])
def test_batch_equals_single_evaluations(gpu, R):
    P, tri, nrm, cen, tg, d = _plan(gpu, seed=R)
    n, m = len(cen), len(tg)
    rng = np.random.default_rng(R)
    ssl, sdl = rng.normal(size=(R, n, 3)), rng.normal(size=(R, n, 3))
    a = _batch(P, d, R, ssl, sdl, n, m)
    b = _single(P, d, ssl, sdl, n, m)
    for x, y in zip(a, b):
        assert rel(x, y) < SAME
    P.close()


def test_batch_single_layer_without_strain(gpu):
    P, tri, nrm, cen, tg, d = _plan(gpu, level=2, ntarg=50, iprec=1, seed=3)
    n, m = len(cen), len(tg)
    R = 20
    ssl = np.random.default_rng(9).normal(size=(R, n, 3))
    a = _batch(P, d, R, ssl, None, n, m, strain=False)
    b = _single(P, d, ssl, None, n, m, strain=False)
    assert rel(a[0], b[0]) < SAME and rel(a[2], b[2]) < SAME
    P.close()


def test_batch_within_tolerance_of_direct(gpu):
    P, tri, nrm, cen, tg, d = _plan(gpu, level=3, ntarg=100, iprec=2, seed=5)
    n, m = len(cen), len(tg)
    R = 3
    rng = np.random.default_rng(11)
    ssl, sdl = rng.normal(size=(R, n, 3)), rng.normal(size=(R, n, 3))
    a = _batch(P, d, R, ssl, sdl, n, m)
    for r in range(R):
        dd = gpu.el3dtriadirecttarg(1.3, 0.7, tri, nrm, cen, ssl[r], sdl[r], tg)
        assert rel(a[0][r], dd[0]) < 1e-6 and rel(a[2][r], dd[2]) < 1e-6
        assert rel(a[1][r], dd[1]) < 1e-5 and rel(a[3][r], dd[3]) < 1e-5
    P.close()


def test_batch_mixed_precision_error(gpu):
    # mixed form: FP32 expansions and translations; its error against the
    # FP64 form stays within the iprec-2 tolerance (relative l2)
    P, tri, nrm, cen, tg, d = _plan(gpu, level=4, ntarg=300, iprec=2, seed=7)
    n, m = len(cen), len(tg)
    R = 8
    rng = np.random.default_rng(13)
    ssl, sdl = rng.normal(size=(R, n, 3)), rng.normal(size=(R, n, 3))
    a = _batch(P, d, R, ssl, sdl, n, m)
    torch = _t()
    u = torch.zeros((R, n, 3), dtype=torch.float64, device="cuda")
    e = torch.zeros((R, n, 3, 3), dtype=torch.float64, device="cuda")
    ut = torch.zeros((R, m, 3), dtype=torch.float64, device="cuda")
    et = torch.zeros((R, m, 3, 3), dtype=torch.float64, device="cuda")
    P.evaluate_batch(1.3, 0.7, R, d(ssl), d(sdl), u, e, ut, et, precision=1)
    b = [u.cpu().numpy(), e.cpu().numpy(), ut.cpu().numpy(), et.cpu().numpy()]
    assert rel(b[0], a[0]) < 0.5e-6 and rel(b[2], a[2]) < 0.5e-6
    assert rel(b[1], a[1]) < 0.5e-5 and rel(b[3], a[3]) < 0.5e-5
    # and the FP32 parts do change the result (the mixed path ran)
    assert rel(b[0], a[0]) > 1e-13
    P.close()


def test_batch_host_entry_matches_device_batch(gpu):
    # efmm_batch_host (host arrays, C ABI) == device-resident batch
    P, tri, nrm, cen, tg, d = _plan(gpu, level=3, ntarg=60, iprec=2, seed=17)
    n, m = len(cen), len(tg)
    R = 9
    rng = np.random.default_rng(23)
    ssl, sdl = rng.normal(size=(R, n, 3)), rng.normal(size=(R, n, 3))
    a = _batch(P, d, R, ssl, sdl, n, m)
    ier, pt, st, ptt, stt = gpu.batch_host(2, 1.3, 0.7, tri, nrm, cen, ssl, sdl, tg, precision=0)
    assert ier == 0
    for x, y in zip((pt, st, ptt, stt), a):
        assert rel(x, y) < SAME
    P.close()


def test_direct_subset_matches_full_direct(gpu):
    torch = _t()
    P, tri, nrm, cen, tg, d = _plan(gpu, level=3, ntarg=10, iprec=2, seed=19)
    n = len(cen)
    rng = np.random.default_rng(29)
    ssl, sdl = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    full = gpu.el3dtriadirecttarg(1.3, 0.7, tri, nrm, cen, ssl, sdl, tg)
    ns = 100
    u = torch.zeros((ns, 3), dtype=torch.float64, device="cuda")
    e = torch.zeros((ns, 3, 3), dtype=torch.float64, device="cuda")
    P.evaluate_direct_subset(1.3, 0.7, ns, d(ssl), d(sdl), u, e)
    assert rel(u.cpu().numpy(), full[0][:ns]) < 1e-14 and rel(e.cpu().numpy(), full[1][:ns]) < 1e-14
    P.close()


def _batch_mode(P, d, R, ssl, sdl, n, m, mode, precision=0, rlam=1.3, strain=True):
    torch = _t()
    u = torch.zeros((R, n, 3), dtype=torch.float64, device="cuda")
    e = torch.zeros((R, n, 3, 3), dtype=torch.float64, device="cuda") if strain else None
    ut = torch.zeros((R, m, 3), dtype=torch.float64, device="cuda")
    et = torch.zeros((R, m, 3, 3), dtype=torch.float64, device="cuda") if strain else None
    P.evaluate_batch(rlam, 0.7, R, d(ssl) if ssl is not None else None, d(sdl) if sdl is not None else None,
                     u, e, ut, et, precision=precision, mode=mode)
    return [u.cpu().numpy(), e.cpu().numpy() if strain else None, ut.cpu().numpy(),
            et.cpu().numpy() if strain else None]


@pytest.mark.parametrize("R", [3, 37, 70])
def test_batch_iter_store_and_replay(gpu, R):
    # mode 1 stores the near-field pair responses and contracts them with
    # all right-hand sides; mode 2 replays them for new densities.  Both
    # equal the analytic batched pass (R = 70 runs as two passes: store,
    # then replay)
    torch = _t()
    tri, nrm, cen = G.sphere_triangles(3)
    tg = G.box_targets(90, 41)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    P = gpu.Plan(0)
    P.set_geometry(d(tri), d(nrm), d(cen), d(tg), iprec=2, iter=True)
    n, m = len(cen), len(tg)
    rng = np.random.default_rng(100 + R)
    ssl, sdl = rng.normal(size=(R, n, 3)), rng.normal(size=(R, n, 3))
    a = _batch_mode(P, d, R, ssl, sdl, n, m, 0)
    b = _batch_mode(P, d, R, ssl, sdl, n, m, 1)
    for x, y in zip(a, b):
        assert rel(x, y) < SAME
    assert P.stored_bytes() > 0
    s2, d2 = rng.normal(size=(R, n, 3)), rng.normal(size=(R, n, 3))
    c = _batch_mode(P, d, R, s2, d2, n, m, 2)
    e = _batch_mode(P, d, R, s2, d2, n, m, 0)
    for x, y in zip(c, e):
        assert rel(x, y) < SAME
    # mixed precision on the stored near field (its FP32 copy replayed on
    # the tensor cores): all four outputs within the FP32 tolerance
    f = _batch_mode(P, d, R, s2, d2, n, m, 2, precision=1)
    errs = [rel(x, y) for x, y in zip(f, e)]
    print("mixed replay vs FP64:", " ".join(f"{v:.2e}" for v in errs))
    assert errs[0] < 0.5e-6 and errs[2] < 0.5e-6 and errs[1] < 0.5e-5 and errs[3] < 0.5e-5
    assert max(errs) > 1e-13  # the FP32 path ran
    # the same store serves the single-density ITER call
    u = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    ee = torch.zeros((n, 3, 3), dtype=torch.float64, device="cuda")
    ut = torch.zeros((m, 3), dtype=torch.float64, device="cuda")
    et = torch.zeros((m, 3, 3), dtype=torch.float64, device="cuda")
    P.evaluate(1.3, 0.7, d(s2[0]), d(d2[0]), u, ee, ut, et, mode=2)
    assert rel(u.cpu().numpy(), e[0][0]) < SAME and rel(et.cpu().numpy(), e[3][0]) < SAME
    # other Lame constants than the store's: handle mismatch
    with pytest.raises(gpu.ElfmmError) as ex:
        _batch_mode(P, d, R, s2, d2, n, m, 2, rlam=1.4)
    assert ex.value.ier == 512
    P.close()


def test_batch_iter_single_layer_displacement_only(gpu):
    torch = _t()
    tri, nrm, cen = G.sphere_triangles(2)
    tg = G.box_targets(30, 43)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    P = gpu.Plan(0)
    P.set_geometry(d(tri), d(nrm), d(cen), d(tg), iprec=1, iter=True)
    n, m = len(cen), len(tg)
    R = 17
    rng = np.random.default_rng(5)
    ssl = rng.normal(size=(R, n, 3))
    _batch_mode(P, d, R, ssl, None, n, m, 1, strain=False)
    s2 = rng.normal(size=(R, n, 3))
    a = _batch_mode(P, d, R, s2, None, n, m, 2, strain=False)
    b = _batch_mode(P, d, R, s2, None, n, m, 0, strain=False)
    assert rel(a[0], b[0]) < SAME and rel(a[2], b[2]) < SAME
    # single-layer store without strain rows (KB = 3) replayed in FP32
    c = _batch_mode(P, d, R, s2, None, n, m, 2, strain=False, precision=1)
    assert rel(c[0], b[0]) < 1e-5 and rel(c[2], b[2]) < 1e-5 and rel(c[0], b[0]) > 1e-13
    # a replay asking for strain the store does not hold is a mismatch
    with pytest.raises(gpu.ElfmmError):
        _batch_mode(P, d, R, s2, None, n, m, 2)
    P.close()


@pytest.mark.parametrize("R", [8, 64])
def test_batch_p2m_unit_multipoles_match_node_products(gpu, monkeypatch, R):
    # the batched P2M through per-triangle unit-density multipoles equals the
    # node-feature product form (ELFMM3D_P2M=nodes): the same FP64 sums
    # regrouped, and the mixed form within FP32 rounding
    P, tri, nrm, cen, tg, d = _plan(gpu, level=3, ntarg=80, iprec=3, seed=23)
    monkeypatch.setenv("ELFMM3D_P2M", "nodes")
    Pn = gpu.Plan(0)
    monkeypatch.delenv("ELFMM3D_P2M")
    Pn.set_geometry(d(tri), d(nrm), d(cen), d(tg), iprec=3)
    n, m = len(cen), len(tg)
    rng = np.random.default_rng(29)
    ssl, sdl = rng.normal(size=(R, n, 3)), rng.normal(size=(R, n, 3))
    a = _batch(P, d, R, ssl, sdl, n, m)
    b = _batch(Pn, d, R, ssl, sdl, n, m)
    for x, y in zip(a, b):
        assert rel(x, y) < SAME
    torch = _t()
    outs = []
    for Q in (P, Pn):
        o = [torch.zeros((R, n, 3), dtype=torch.float64, device="cuda"),
             torch.zeros((R, n, 3, 3), dtype=torch.float64, device="cuda"),
             torch.zeros((R, m, 3), dtype=torch.float64, device="cuda"),
             torch.zeros((R, m, 3, 3), dtype=torch.float64, device="cuda")]
        Q.evaluate_batch(1.3, 0.7, R, d(ssl), d(sdl), *o, precision=1)
        outs.append([t.cpu().numpy() for t in o])
    for x, y, z in zip(outs[0], outs[1], a):
        print(f"unit vs nodes (mixed): {rel(x, y):.2e}   unit mixed vs FP64: {rel(x, z):.2e}")
        assert rel(x, y) < 1e-6 and rel(x, z) < 1e-6
    P.close()
    Pn.close()


def test_mixed_form_orders_floor(gpu):
    # the mixed form truncates no finer than its FP32 rounding (default
    # floor 5e-8): at iprec 3 its order drops below the iprec order and its
    # error against the FP64 form stays at the FP32 level; floor 0 restores
    # the iprec orders
    P, tri, nrm, cen, tg, d = _plan(gpu, level=3, ntarg=100, iprec=3, seed=31)
    n, m = len(cen), len(tg)
    R = 8
    rng = np.random.default_rng(37)
    ssl, sdl = rng.normal(size=(R, n, 3)), rng.normal(size=(R, n, 3))
    ref = _batch(P, d, R, ssl, sdl, n, m)
    p_iprec = P.info()["p"]
    torch = _t()
    outs = {}
    for floor in (5e-8, 0.0):
        pm = P.set_mixed_floor(floor)
        assert (pm < p_iprec) if floor > 0 else (pm == p_iprec)
        o = [torch.zeros((R, n, 3), dtype=torch.float64, device="cuda"),
             torch.zeros((R, n, 3, 3), dtype=torch.float64, device="cuda"),
             torch.zeros((R, m, 3), dtype=torch.float64, device="cuda"),
             torch.zeros((R, m, 3, 3), dtype=torch.float64, device="cuda")]
        P.evaluate_batch(1.3, 0.7, R, d(ssl), d(sdl), *o, precision=1)
        outs[floor] = [t.cpu().numpy() for t in o]
        errs = [rel(x, y) for x, y in zip(outs[floor], ref)]
        print(f"floor {floor:g}: order {pm} (iprec {p_iprec}), mixed vs FP64:", " ".join(f"{v:.2e}" for v in errs))
        assert errs[0] < 1e-6 and errs[2] < 1e-6 and errs[1] < 1e-5 and errs[3] < 1e-5
    # the FP64 form keeps the iprec orders whatever the mixed floor
    assert rel(_batch(P, d, R, ssl, sdl, n, m)[0], ref[0]) < SAME
    P.close()

