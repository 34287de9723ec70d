"""B200-native elastostatic triangle-layer-potential FMM.

Python host layer over the C ABI of ``libelfmm3d_b200.so`` (declared in
``include/elfmm3d_b200.h``).  The functions mirror the reference's Fortran
routines (same names, argument meaning, array layouts and ``ier`` codes):

    elfmm3dtria(iprec, rlam, rmu, triangle, trinorm, source, ...)
        -> src/elfmm3dtria.f:71
    elfmm3dtriatarg(iprec, rlam, rmu, triangle, trinorm, source, ..., target=...)
        -> src/elfmm3dtria.f:162
    el3dtriadirecttarg(rlam, rmu, triangle, trinorm, source, ...)
        -> src/elfmm3dtria.f:1483
    elfmm3dtriatargiter(iprec, rlam, rmu, ..., icomp_type=, wsave=)
        -> src/elfmm3dtria_iter_1.f:160

Arrays are numpy, shaped in C order as the transpose of the Fortran shapes:
``triangle`` (n,3,3) [triangle][vertex][xyz], ``sigma`` (n,3), ``ptfrc`` (n,3),
``strain`` (n,3,3).  Outputs carry no 1/(4 pi) factor, like the reference.

There is no CPU fallback: if the CUDA library is missing or no GPU is
visible, every compute call raises.
"""
import ctypes
import os

import numpy as np

__all__ = ["elfmm3dtria", "elfmm3dtriatarg", "el3dtriadirecttarg", "elfmm3dtriatargiter", "batch_host",
           "elhfmm3dtriatargiter", "halfspace_self",
           "elfmm3dtriaiter", "iter_release", "iter_stored_bytes", "Plan", "load",
           "library_path", "device_count", "ElfmmError"]

_HERE = os.path.dirname(os.path.abspath(__file__))
# ELFMM3D_LIB may point at another build of the same library (e.g. a variant)
_LIB_PATH = os.environ.get("ELFMM3D_LIB", os.path.join(_HERE, "libelfmm3d_b200.so"))
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_llp = ctypes.POINTER(ctypes.c_longlong)
_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p

# symbols the library must export (checked by the CPU test suite)
EXPORTS = ["elfmm3dtria_", "elfmm3dtriatarg_", "el3dtriadirecttarg_", "efmm_device_count",
           "efmm_plan_create", "efmm_plan_destroy", "efmm_plan_set_geometry",
           "efmm_plan_evaluate", "efmm_plan_evaluate_direct", "efmm_plan_timings", "efmm_plan_product_stats", "efmm_plan_near_stats",
           "efmm_plan_info", "efmm_plan_tree_export", "efmm_kernel_launches", "efmm_plan_record",
           "efmm_plan_elapsed", "efmm_direct_noalloc", "elfmm3dtriatargiter_", "elfmm3dtriaiter_",
           "efmm_iter_release", "efmm_iter_stored_bytes", "efmm_plan_setup_timings",
           "efmm_plan_evaluate_batch", "efmm_plan_flops",
           "efmm_plan_evaluate_direct_subset", "efmm_batch_host", "efmm_factored_selfcheck",
           "efmm_plan_evaluate_iter", "efmm_plan_evaluate_batch_iter", "efmm_plan_evaluate_image", "efmm_plan_evaluate_batch_graph", "efmm_plan_evaluate_image_graph", "efmm_hs_image_direct", "efmm_u_m2l_selfcheck", "efmm_tc_gemm_selfcheck", "efmm_tc_gemm_selfcheck_tile", "efmm_plan_stored_bytes", "efmm_plan_set_mixed_floor", "efmm_plan_translation_flops", "elhfmm3dtriatargiter_",
           "elhfmm3dtria_total_", "efmm_mindlin_image_kernel",
           "efmm_pair_eval_host", "elhfmm3dtria_batch_host", "efmm_tri_read", "efmm_tri_write",
           "efmm_tri_refine", "efmm_tri_build", "efmm_rot_tc_selfcheck", "efmm_rot_tc_selfcheck_device",
           "efmm_rot_tc_bench",
           "efmm_hs_capped", "efmm_plan_solve", "efmm_gcr_dense_host",
           "efmm_tune_pick", "efmm_tune_report", "efmm_tune_reset", "efmm_tune_dump", "efmm_tc_variant",
           "efmm_split_variant", "efmm_tc_bulk_selfcheck",
           "elfmm3dparttarg_", "elfmm3dpart_", "el3dpartdirecttarg_", "efmm_part_pair_host",
           "elhfmm3dparttarg_", "elhfmm3dpart_", "elh3dpartdirecttarg_", "efmm_plan_set_forest",
           "efmm_forest_create", "efmm_forest_destroy", "efmm_forest_set_geometry", "efmm_forest_evaluate",
           "efmm_forest_plan", "efmm_forest_layout", "elhfmm3dtria_many_host", "efmm_plan_set_leaf",
           "efmm_forest_set_leaf", "efmm_forest_set_mixed_floor", "efmm_many_host_set_mixed_floor"]


class ElfmmError(RuntimeError):
    def __init__(self, ier, where=""):
        super().__init__(f"elfmm3d_b200 error ier={ier} {where}")
        self.ier = ier


def library_path():
    return _LIB_PATH


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ElfmmError(-1, f"CUDA library not built: {_LIB_PATH} (run python -m elfmmlib3d_b200.build)")
    L = ctypes.CDLL(_LIB_PATH)
    L.efmm_device_count.restype = ctypes.c_int
    L.efmm_plan_create.restype = _vp
    L.efmm_plan_create.argtypes = [ctypes.c_int]
    L.efmm_plan_destroy.argtypes = [_vp]
    L.efmm_plan_set_geometry.restype = ctypes.c_int
    L.efmm_plan_set_geometry.argtypes = [_vp, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int]
    for f in (L.efmm_plan_evaluate, L.efmm_plan_evaluate_direct):
        f.restype = ctypes.c_int
        f.argtypes = [_vp, ctypes.c_double, ctypes.c_double, _vp, _vp, _vp, _vp, _vp, _vp]
    L.efmm_plan_evaluate_batch.restype = ctypes.c_int
    L.efmm_plan_evaluate_batch.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp, _vp,
                                           _vp, _vp, _vp, ctypes.c_int]
    L.efmm_plan_flops.argtypes = [_vp, _dp]
    L.efmm_plan_stored_bytes.restype = ctypes.c_longlong
    L.efmm_plan_stored_bytes.argtypes = [_vp]
    L.efmm_plan_set_mixed_floor.restype = ctypes.c_int
    L.efmm_plan_set_mixed_floor.argtypes = [_vp, ctypes.c_double, _vp]
    L.efmm_plan_translation_flops.restype = ctypes.c_int
    L.efmm_plan_translation_flops.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _dp]
    L.efmm_plan_evaluate_batch_graph.restype = ctypes.c_int
    L.efmm_plan_evaluate_batch_graph.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp,
                                                 _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int]
    L.efmm_plan_evaluate_image_graph.restype = ctypes.c_int
    L.efmm_plan_evaluate_image_graph.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp,
                                                 _vp, _vp, ctypes.c_int]
    L.efmm_plan_evaluate_image.restype = ctypes.c_int
    L.efmm_plan_evaluate_image.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp, _vp,
                                           _vp, ctypes.c_int, ctypes.c_int]
    L.efmm_plan_evaluate_batch_iter.restype = ctypes.c_int
    L.efmm_plan_evaluate_batch_iter.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp,
                                                _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int]
    L.efmm_plan_evaluate_iter.restype = ctypes.c_int
    L.efmm_plan_evaluate_iter.argtypes = [_vp, ctypes.c_double, ctypes.c_double, _vp, _vp, _vp, _vp, _vp, _vp,
                                          ctypes.c_int]
    L.efmm_plan_evaluate_direct_subset.restype = ctypes.c_int
    L.efmm_plan_evaluate_direct_subset.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp,
                                                   _vp, _vp, _vp]
    L.efmm_plan_timings.argtypes = [_vp, _fp]
    L.efmm_plan_info.argtypes = [_vp, _llp]
    L.efmm_plan_setup_timings.argtypes = [_vp, _fp]
    L.efmm_kernel_launches.restype = ctypes.c_longlong
    L.efmm_plan_record.restype = ctypes.c_int
    L.efmm_plan_record.argtypes = [_vp, ctypes.c_int]
    L.efmm_plan_elapsed.restype = ctypes.c_float
    L.efmm_plan_elapsed.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.efmm_direct_noalloc.restype = ctypes.c_int
    L.efmm_direct_noalloc.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp, _vp, _vp,
                                      ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp]
    L.efmm_batch_host.restype = ctypes.c_int
    L.efmm_batch_host.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp,
                                  ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int]
    L.elhfmm3dtria_batch_host.restype = ctypes.c_int
    L.elhfmm3dtria_batch_host.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp, _dp,
                                          _dp, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, _dp,
                                          ctypes.c_int]
    L.efmm_plan_set_forest.restype = ctypes.c_int
    L.efmm_plan_set_forest.argtypes = [_vp, _dp]
    L.efmm_forest_create.restype = _vp
    L.efmm_forest_create.argtypes = [ctypes.c_int]
    L.efmm_forest_destroy.argtypes = [_vp]
    L.efmm_forest_set_geometry.restype = ctypes.c_int
    L.efmm_forest_set_geometry.argtypes = [_vp, ctypes.c_int, _ip, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int]
    L.efmm_forest_evaluate.restype = ctypes.c_int
    L.efmm_forest_evaluate.argtypes = [_vp, ctypes.c_double, ctypes.c_double, _vp, _vp, _vp, _vp, ctypes.c_int,
                                       ctypes.c_int]
    L.efmm_plan_set_leaf.restype = ctypes.c_int
    L.efmm_plan_set_leaf.argtypes = [_vp, ctypes.c_int]
    L.efmm_forest_set_leaf.restype = ctypes.c_int
    L.efmm_forest_set_leaf.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.efmm_forest_set_mixed_floor.restype = ctypes.c_int
    L.efmm_forest_set_mixed_floor.argtypes = [_vp, ctypes.c_double]
    L.efmm_many_host_set_mixed_floor.restype = ctypes.c_int
    L.efmm_many_host_set_mixed_floor.argtypes = [ctypes.c_double]
    L.efmm_forest_plan.restype = _vp
    L.efmm_forest_plan.argtypes = [_vp, ctypes.c_int]
    L.efmm_forest_layout.restype = ctypes.c_int
    L.efmm_forest_layout.argtypes = [ctypes.c_int, _dp, _dp, _dp]
    L.elhfmm3dtria_many_host.restype = ctypes.c_int
    L.elhfmm3dtria_many_host.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _ip, _dp,
                                         _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int]
    L.efmm_tri_read.restype = ctypes.c_int
    L.efmm_tri_read.argtypes = [ctypes.c_char_p, _dp, ctypes.c_int, _ip, _ip, ctypes.c_int, _ip]
    L.efmm_tri_write.restype = ctypes.c_int
    L.efmm_tri_write.argtypes = [ctypes.c_char_p, _dp, ctypes.c_int, _ip, ctypes.c_int]
    L.efmm_tri_refine.restype = ctypes.c_int
    L.efmm_tri_refine.argtypes = [_dp, ctypes.c_int, _ip, ctypes.c_int, _dp, _ip]
    L.efmm_tri_build.restype = ctypes.c_int
    L.efmm_tri_build.argtypes = [_dp, ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, _dp, _dp]
    L.efmm_iter_release.restype = ctypes.c_int
    L.efmm_iter_release.argtypes = [_dp, ctypes.c_int]
    L.efmm_iter_stored_bytes.restype = ctypes.c_longlong
    L.efmm_iter_stored_bytes.argtypes = [_dp, ctypes.c_int]
    L.efmm_plan_tree_export.restype = ctypes.c_int
    L.efmm_plan_tree_export.argtypes = [_vp, _ip, _ip, _ip, _ip, _dp, _ip, _ip, _llp]
    _lib = L
    return L


def device_count():
    return load().efmm_device_count()


def kernel_launches():
    """Kernels of this library launched so far in the process."""
    return int(load().efmm_kernel_launches())


def _need_gpu():
    if device_count() < 1:
        raise ElfmmError(1024, "no CUDA device visible")


def _c(a, shape):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))


def _ref_args(triangle, trinorm, source, sigma_sl, sigma_dl):
    tri = _c(triangle, (-1, 3, 3))
    n = tri.shape[0]
    nrm = _c(trinorm, (n, 3))
    src = _c(source, (n, 3))
    ssl = _c(sigma_sl, (n, 3)) if sigma_sl is not None else np.zeros((n, 3))
    sdl = _c(sigma_dl, (n, 3)) if sigma_dl is not None else np.zeros((n, 3))
    return tri, nrm, src, ssl, sdl, n


def _byref_i(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _byref_d(v):
    return ctypes.byref(ctypes.c_double(float(v)))


def elfmm3dtriatarg(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None,
                    target=None, ifptfrc=1, ifstrain=1, ifptfrctarg=1, ifstraintarg=1):
    """Displacement/strain of piecewise-constant single (traction ``sigma_sl``)
    and double (displacement jump ``sigma_dl``) layers on flat triangles, at the
    n source points and at optional targets (src/elfmm3dtria.f:162).

    Returns (ier, ptfrc (n,3), strain (n,3,3), ptfrctarg (m,3), straintarg (m,3,3)).
    """
    L = load()
    _need_gpu()
    tri, nrm, src, ssl, sdl, n = _ref_args(triangle, trinorm, source, sigma_sl, sigma_dl)
    tg = _c(target if target is not None else np.zeros((0, 3)), (-1, 3))
    m = tg.shape[0]
    pt = np.zeros((n, 3))
    st = np.zeros((n, 3, 3))
    ptt = np.zeros((max(m, 1), 3))
    stt = np.zeros((max(m, 1), 3, 3))
    ier = ctypes.c_int(0)
    L.elfmm3dtriatarg_(ctypes.byref(ier), _byref_i(iprec), _byref_d(rlam), _byref_d(rmu),
                       tri.ctypes.data_as(_dp), nrm.ctypes.data_as(_dp), _byref_i(n),
                       src.ctypes.data_as(_dp), _byref_i(sigma_sl is not None), ssl.ctypes.data_as(_dp),
                       _byref_i(sigma_dl is not None), sdl.ctypes.data_as(_dp), _byref_i(ifptfrc),
                       pt.ctypes.data_as(_dp), _byref_i(ifstrain), st.ctypes.data_as(_dp), _byref_i(m),
                       tg.ctypes.data_as(_dp), _byref_i(ifptfrctarg), ptt.ctypes.data_as(_dp),
                       _byref_i(ifstraintarg), stt.ctypes.data_as(_dp))
    return ier.value, pt, st, ptt[:m], stt[:m]


def elfmm3dtria(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None,
                ifptfrc=1, ifstrain=1):
    """On-surface evaluation only (src/elfmm3dtria.f:71). Returns (ier, ptfrc, strain)."""
    ier, pt, st, _, _ = elfmm3dtriatarg(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl,
                                        sigma_dl, None, ifptfrc, ifstrain, 0, 0)
    return ier, pt, st


def el3dtriadirecttarg(rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None,
                       target=None, ifptfrc=1, ifstrain=1, ifptfrctarg=1, ifstraintarg=1):
    """O(N^2) direct evaluation on the GPU (src/elfmm3dtria.f:1483).
    Returns (ptfrc, strain, ptfrctarg, straintarg)."""
    L = load()
    _need_gpu()
    tri, nrm, src, ssl, sdl, n = _ref_args(triangle, trinorm, source, sigma_sl, sigma_dl)
    tg = _c(target if target is not None else np.zeros((0, 3)), (-1, 3))
    m = tg.shape[0]
    pt = np.zeros((n, 3))
    st = np.zeros((n, 3, 3))
    ptt = np.zeros((max(m, 1), 3))
    stt = np.zeros((max(m, 1), 3, 3))
    L.el3dtriadirecttarg_(_byref_d(rlam), _byref_d(rmu), tri.ctypes.data_as(_dp), nrm.ctypes.data_as(_dp),
                          _byref_i(n), src.ctypes.data_as(_dp), _byref_i(sigma_sl is not None),
                          ssl.ctypes.data_as(_dp), _byref_i(sigma_dl is not None), sdl.ctypes.data_as(_dp),
                          _byref_i(ifptfrc), pt.ctypes.data_as(_dp), _byref_i(ifstrain),
                          st.ctypes.data_as(_dp), _byref_i(m), tg.ctypes.data_as(_dp),
                          _byref_i(ifptfrctarg), ptt.ctypes.data_as(_dp), _byref_i(ifstraintarg),
                          stt.ctypes.data_as(_dp))
    return pt, st, ptt[:m], stt[:m]


def _part_args(source, sigma_sl, sigma_dl, sigma_dv):
    src = _c(source, (-1, 3))
    n = src.shape[0]
    z = np.zeros((n, 3))
    ssl = _c(sigma_sl, (n, 3)) if sigma_sl is not None else z
    sdl = _c(sigma_dl, (n, 3)) if sigma_dl is not None else z
    sdv = _c(sigma_dv, (n, 3)) if sigma_dv is not None else z
    return src, ssl, sdl, sdv, n


def elfmm3dparttarg(iprec, rlam, rmu, source, sigma_sl=None, sigma_dl=None, sigma_dv=None, target=None,
                    ifptfrc=1, ifstrain=1, ifptfrctarg=1, ifstraintarg=1, direct=False, halfspace=False):
    """Particle FMM in free space (src/elfmm3dpart.f:104; direct=True: the
    O(N^2) el3dpartdirecttarg, :506) or, halfspace=True, in the Mindlin half
    space z <= 0 (elhfmm3dparttarg / elh3dpartdirecttarg): point forces
    sigma_sl (n,3), point displacement discontinuities sigma_dl (n,3) with
    orientations sigma_dv (n,3).  Returns (ier, ptfrc (n,3), strain (n,3,3),
    ptfrctarg (m,3), straintarg (m,3,3))."""
    L = load()
    _need_gpu()
    src, ssl, sdl, sdv, n = _part_args(source, sigma_sl, sigma_dl, sigma_dv)
    tg = _c(target if target is not None else np.zeros((0, 3)), (-1, 3))
    m = tg.shape[0]
    pt, st = np.zeros((n, 3)), np.zeros((n, 3, 3))
    ptt, stt = np.zeros((max(m, 1), 3)), np.zeros((max(m, 1), 3, 3))
    d = lambda a: a.ctypes.data_as(_dp)
    ier = ctypes.c_int(0)
    if direct:
        f = L.elh3dpartdirecttarg_ if halfspace else L.el3dpartdirecttarg_
        f(_byref_d(rlam), _byref_d(rmu), _byref_i(n), d(src), _byref_i(sigma_sl is not None),
                              d(ssl), _byref_i(sigma_dl is not None), d(sdl), d(sdv), _byref_i(ifptfrc), d(pt),
                              _byref_i(ifstrain), d(st), _byref_i(m), d(tg), _byref_i(ifptfrctarg), d(ptt),
                              _byref_i(ifstraintarg), d(stt))
    else:
        f = L.elhfmm3dparttarg_ if halfspace else L.elfmm3dparttarg_
        f(ctypes.byref(ier), _byref_i(iprec), _byref_d(rlam), _byref_d(rmu), _byref_i(n), d(src),
                           _byref_i(sigma_sl is not None), d(ssl), _byref_i(sigma_dl is not None), d(sdl), d(sdv),
                           _byref_i(ifptfrc), d(pt), _byref_i(ifstrain), d(st), _byref_i(m), d(tg),
                           _byref_i(ifptfrctarg), d(ptt), _byref_i(ifstraintarg), d(stt))
    return ier.value, pt, st, ptt[:m], stt[:m]


def part_pair_host(rlam, rmu, x, y, sl=None, dl=None, nu=None):
    """One (point, particle) pair of the particle near field on the host
    (efmm_part_pair_host): (u (3,), strain (3,3))."""
    L = load()
    u, e6 = np.zeros(3), np.zeros(6)
    p = lambda a: _c(a, (3,)).ctypes.data_as(_dp) if a is not None else None
    L.efmm_part_pair_host.restype = ctypes.c_int
    L.efmm_part_pair_host.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
    keep = [_c(a, (3,)) if a is not None else None for a in (x, y, sl, dl, nu)]
    ier = L.efmm_part_pair_host(float(rlam), float(rmu), *[k.ctypes.data_as(_dp) if k is not None else None
                                                           for k in keep], u.ctypes.data_as(_dp),
                                e6.ctypes.data_as(_dp))
    if ier:
        raise ElfmmError(ier, "part_pair_host")
    e = np.array([[e6[0], e6[3], e6[4]], [e6[3], e6[1], e6[5]], [e6[4], e6[5], e6[2]]])
    return u, e


def batch_host(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None, target=None,
               precision=0, out=None):
    """nrhs right-hand sides in one pass from host arrays: sigma_sl/sigma_dl
    (nrhs,n,3).  Returns (ier, ptfrc (nrhs,n,3), strain (nrhs,n,3,3),
    ptfrctarg (nrhs,m,3), straintarg (nrhs,m,3,3)).  precision 0 = FP64,
    1 = mixed.  ``out`` may pass preallocated (e.g. pinned) output arrays."""
    L = load()
    _need_gpu()
    tri = _c(triangle, (-1, 3, 3))
    n = tri.shape[0]
    nrm, src = _c(trinorm, (n, 3)), _c(source, (n, 3))
    ssl = _c(sigma_sl, (-1, n, 3)) if sigma_sl is not None else None
    sdl = _c(sigma_dl, (-1, n, 3)) if sigma_dl is not None else None
    R = (ssl if ssl is not None else sdl).shape[0]
    tg = _c(target if target is not None else np.zeros((0, 3)), (-1, 3))
    m = tg.shape[0]
    if out is None:
        out = (np.zeros((R, n, 3)), np.zeros((R, n, 3, 3)), np.zeros((R, max(m, 1), 3)),
               np.zeros((R, max(m, 1), 3, 3)))
    pt, st, ptt, stt = out
    p = lambda a: a.ctypes.data_as(_dp) if a is not None else None
    ier = L.efmm_batch_host(int(iprec), float(rlam), float(rmu), n, p(tri), p(nrm), p(src), m, p(tg), R, p(ssl),
                            p(sdl), p(pt), p(st), p(ptt) if m else None, p(stt) if m else None, int(precision))
    return ier, pt, st, ptt[:, :m], stt[:, :m]


def hs_batch_host(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None, precision=1,
                  icomp_type=1, wsave=None, out=None):
    """Half-space self-evaluation (direct arrival + image part) of nrhs
    right-hand sides from host arrays through elhfmm3dtria_batch_host:
    sigma_sl/sigma_dl (nrhs,n,3).  icomp_type 1 evaluates, 2 also stores both
    near fields behind ``wsave`` (8 doubles), 3 replays them with new
    densities.  Returns (ier, ptfrc (nrhs,n,3), strain (nrhs,n,3,3)).
    ``out`` may pass preallocated (e.g. pinned) output arrays."""
    L = load()
    _need_gpu()
    tri = _c(triangle, (-1, 3, 3))
    n = tri.shape[0]
    nrm, src = _c(trinorm, (n, 3)), _c(source, (n, 3))
    ssl = _c(sigma_sl, (-1, n, 3)) if sigma_sl is not None else None
    sdl = _c(sigma_dl, (-1, n, 3)) if sigma_dl is not None else None
    R = (ssl if ssl is not None else sdl).shape[0]
    if out is None:
        out = (np.zeros((R, n, 3)), np.zeros((R, n, 3, 3)))
    pt, st = out
    ws = wsave if wsave is not None else np.zeros(8)
    p = lambda a: a.ctypes.data_as(_dp) if a is not None else None
    ier = L.elhfmm3dtria_batch_host(int(iprec), float(rlam), float(rmu), n, p(tri), p(nrm), p(src), R, p(ssl),
                                    p(sdl), p(pt), p(st), int(precision), int(icomp_type), p(ws), len(ws))
    return ier, pt, st


def read_tri(path):
    """Read a Cart3D .tri file (efmm_tri_read, the reference's atrireadchk,
    src/trilib.f:59).  Returns (verts (nverts,3) float64, ifaces (nfaces,3)
    int32, 1-based as in the file).  Raises OSError / ValueError."""
    L = load()
    nv, nf = ctypes.c_int(0), ctypes.c_int(0)
    b = os.fsencode(path)
    ier = L.efmm_tri_read(b, None, 0, ctypes.byref(nv), None, 0, ctypes.byref(nf))
    if ier == 1:
        raise OSError(f"read_tri: cannot open {path}")
    if ier not in (0, 2, 3) or (ier == 0 and (nv.value or nf.value)):
        raise ValueError(f"read_tri: malformed file {path} (ier={ier})")
    verts = np.zeros((max(nv.value, 1), 3))
    ifaces = np.zeros((max(nf.value, 1), 3), dtype=np.int32)
    ier = L.efmm_tri_read(b, verts.ctypes.data_as(_dp), nv.value, ctypes.byref(nv),
                          ifaces.ctypes.data_as(_ip), nf.value, ctypes.byref(nf))
    if ier:
        raise ValueError(f"read_tri: malformed file {path} (ier={ier})")
    return verts[:nv.value], ifaces[:nf.value]


def write_tri(path, verts, ifaces):
    """Write a Cart3D .tri file (efmm_tri_write, the reference's atriwrite);
    ifaces 1-based."""
    v = _c(verts, (-1, 3))
    f = np.ascontiguousarray(ifaces, dtype=np.int32).reshape(-1, 3)
    ier = load().efmm_tri_write(os.fsencode(path), v.ctypes.data_as(_dp), v.shape[0], f.ctypes.data_as(_ip),
                                f.shape[0])
    if ier:
        raise OSError(f"write_tri: cannot write {path} (ier={ier})")


def refine_tri(verts, ifaces):
    """Split every face in four at its edge midpoints (efmm_tri_refine, the
    reference's matlab/atrirefine.m).  Returns (verts1, ifaces1)."""
    v = _c(verts, (-1, 3))
    f = np.ascontiguousarray(ifaces, dtype=np.int32).reshape(-1, 3)
    nv, nf = v.shape[0], f.shape[0]
    v1 = np.zeros((nv + 3 * nf, 3))
    f1 = np.zeros((4 * nf, 3), dtype=np.int32)
    ier = load().efmm_tri_refine(v.ctypes.data_as(_dp), nv, f.ctypes.data_as(_ip), nf, v1.ctypes.data_as(_dp),
                                 f1.ctypes.data_as(_ip))
    if ier:
        raise ValueError(f"refine_tri: face index outside 1..{nv}")
    return v1, f1


def build_tri(verts, ifaces):
    """Triangle arrays from vertex arrays (efmm_tri_build, the reference's
    buildtri, src/trilib.f:192).  Returns (triangle (n,3,3), centroids (n,3),
    trinorm (n,3), triarea (n,)): the arguments the FMM entry points take."""
    v = _c(verts, (-1, 3))
    f = np.ascontiguousarray(ifaces, dtype=np.int32).reshape(-1, 3)
    n = f.shape[0]
    tri, cen, nrm, area = np.zeros((n, 3, 3)), np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
    ier = load().efmm_tri_build(v.ctypes.data_as(_dp), v.shape[0], n, f.ctypes.data_as(_ip), tri.ctypes.data_as(_dp),
                                cen.ctypes.data_as(_dp), nrm.ctypes.data_as(_dp), area.ctypes.data_as(_dp))
    if ier:
        raise ValueError(f"build_tri: face index outside 1..{v.shape[0]}")
    return tri, cen, nrm, area


def elhfmm3dtriatargiter(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None, target=None,
                         icomp_type=1, wsave=None, ifptfrctarg=1, ifstraintarg=1):
    """Image part of the half-space (z <= 0) layer potentials at targets
    (src/elhfmm3dtria_iter.f:46).  Returns (ier, lused, ptfrctarg (m,3),
    straintarg (m,3,3))."""
    L = load()
    _need_gpu()
    tri, nrm, src, ssl, sdl, n = _ref_args(triangle, trinorm, source, sigma_sl, sigma_dl)
    tg = _c(target if target is not None else np.zeros((0, 3)), (-1, 3))
    m = tg.shape[0]
    ws = wsave if wsave is not None else np.zeros(8)
    ptt = np.zeros((max(m, 1), 3))
    stt = np.zeros((max(m, 1), 3, 3))
    ier = ctypes.c_int(0)
    lused = ctypes.c_int(0)
    L.elhfmm3dtriatargiter_(ctypes.byref(ier), _byref_i(iprec), _byref_d(rlam), _byref_d(rmu),
                            tri.ctypes.data_as(_dp), nrm.ctypes.data_as(_dp), _byref_i(n), src.ctypes.data_as(_dp),
                            _byref_i(sigma_sl is not None), ssl.ctypes.data_as(_dp), _byref_i(sigma_dl is not None),
                            sdl.ctypes.data_as(_dp), _byref_i(m), tg.ctypes.data_as(_dp), _byref_i(ifptfrctarg),
                            ptt.ctypes.data_as(_dp), _byref_i(ifstraintarg), stt.ctypes.data_as(_dp),
                            _byref_i(icomp_type), ws.ctypes.data_as(_dp), _byref_i(ws.size), ctypes.byref(lused))
    return ier.value, lused.value, ptt[:m], stt[:m]


def hs_image_direct(rlam, rmu, triangle, trinorm, sigma_sl=None, sigma_dl=None, target=None):
    """Image part by direct summation (all pairs, refined quadrature): the
    check of the image FMM.  Returns (ier, u (m,3), e (m,3,3))."""
    L = load()
    _need_gpu()
    tri = _c(triangle, (-1, 3, 3))
    n = tri.shape[0]
    nrm = _c(trinorm, (n, 3))
    ssl = _c(sigma_sl, (n, 3)) if sigma_sl is not None else None
    sdl = _c(sigma_dl, (n, 3)) if sigma_dl is not None else None
    tg = _c(target, (-1, 3))
    m = tg.shape[0]
    u = np.zeros((max(m, 1), 3))
    e = np.zeros((max(m, 1), 3, 3))
    f = L.efmm_hs_image_direct
    f.restype = ctypes.c_int
    ier = f(ctypes.c_int(2), ctypes.c_double(rlam), ctypes.c_double(rmu), tri.ctypes.data_as(_dp),
            nrm.ctypes.data_as(_dp), ctypes.c_int(n), ssl.ctypes.data_as(_dp) if ssl is not None else None,
            sdl.ctypes.data_as(_dp) if sdl is not None else None, ctypes.c_int(m), tg.ctypes.data_as(_dp),
            u.ctypes.data_as(_dp), e.ctypes.data_as(_dp))
    return ier, u[:m], e[:m]


def elhfmm3dtria_total(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None,
                       target=None, ifptfrc=1, ifstrain=1, ifptfrctarg=1, ifstraintarg=1):
    """Half-space (z <= 0) total field, direct arrival + image part, at the
    n centroids (on-surface) and at optional targets, in one call: the sum
    the reference's drivers form from elfmm3dtriatarg and
    elhfmm3dtriatargiter (examples/elhfmm3dtria_self_iter_dr.f:331-385).
    Returns (ier, ptfrc (n,3), strain (n,3,3), ptfrctarg (m,3),
    straintarg (m,3,3))."""
    L = load()
    _need_gpu()
    tri, nrm, src, ssl, sdl, n = _ref_args(triangle, trinorm, source, sigma_sl, sigma_dl)
    tg = _c(target if target is not None else np.zeros((0, 3)), (-1, 3))
    m = tg.shape[0]
    pt = np.zeros((n, 3))
    st = np.zeros((n, 3, 3))
    ptt = np.zeros((max(m, 1), 3))
    stt = np.zeros((max(m, 1), 3, 3))
    ier = ctypes.c_int(0)
    L.elhfmm3dtria_total_(ctypes.byref(ier), _byref_i(iprec), _byref_d(rlam), _byref_d(rmu),
                          tri.ctypes.data_as(_dp), nrm.ctypes.data_as(_dp), _byref_i(n),
                          src.ctypes.data_as(_dp), _byref_i(sigma_sl is not None), ssl.ctypes.data_as(_dp),
                          _byref_i(sigma_dl is not None), sdl.ctypes.data_as(_dp), _byref_i(ifptfrc),
                          pt.ctypes.data_as(_dp), _byref_i(ifstrain), st.ctypes.data_as(_dp), _byref_i(m),
                          tg.ctypes.data_as(_dp), _byref_i(ifptfrctarg), ptt.ctypes.data_as(_dp),
                          _byref_i(ifstraintarg), stt.ctypes.data_as(_dp))
    return ier.value, pt, st, ptt[:m], stt[:m]


def halfspace_self(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None):
    """Half-space self-evaluation at the centroids: the free-space (direct
    arrival, on-surface) evaluation plus the image part with the centroids as
    targets, the sum the reference's drivers form
    (examples/elhfmm3dtria_self_iter_dr.f:331-385).  Returns (ier, ptfrc, strain)."""
    ier, pt, st = elfmm3dtria(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl, sigma_dl)
    if ier:
        return ier, pt, st
    ier, _, pti, sti = elhfmm3dtriatargiter(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl, sigma_dl,
                                            target=source)
    return ier, pt + pti, st + sti


ITER_LUSED = 8  # words of wsave the ITER handle occupies


def elfmm3dtriatargiter(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None,
                        target=None, icomp_type=1, wsave=None, ifptfrc=1, ifstrain=1, ifptfrctarg=1,
                        ifstraintarg=1):
    """Iterative-solver variant (src/elfmm3dtria_iter_1.f:160): icomp_type 2
    evaluates and stores the near-field interactions, 3 reuses them with new
    densities on the same geometry, 1 evaluates without storage, 4 builds the
    tree only, 5 stores and evaluates the near field alone.  ``wsave`` is a
    float64 array (at least ``ITER_LUSED`` words) that receives / supplies the
    handle of the device-resident store.

    Returns (ier, lused, ptfrc, strain, ptfrctarg, straintarg).
    """
    L = load()
    _need_gpu()
    tri, nrm, src, ssl, sdl, n = _ref_args(triangle, trinorm, source, sigma_sl, sigma_dl)
    tg = _c(target if target is not None else np.zeros((0, 3)), (-1, 3))
    m = tg.shape[0]
    if wsave is None:
        wsave = np.zeros(ITER_LUSED)
    if wsave.dtype != np.float64 or not wsave.flags.c_contiguous:
        raise ValueError("wsave must be a contiguous float64 array")
    pt = np.zeros((n, 3))
    st = np.zeros((n, 3, 3))
    ptt = np.zeros((max(m, 1), 3))
    stt = np.zeros((max(m, 1), 3, 3))
    ier = ctypes.c_int(0)
    lused = ctypes.c_int(0)
    L.elfmm3dtriatargiter_(ctypes.byref(ier), _byref_i(iprec), _byref_d(rlam), _byref_d(rmu),
                           tri.ctypes.data_as(_dp), nrm.ctypes.data_as(_dp), _byref_i(n),
                           src.ctypes.data_as(_dp), _byref_i(sigma_sl is not None), ssl.ctypes.data_as(_dp),
                           _byref_i(sigma_dl is not None), sdl.ctypes.data_as(_dp), _byref_i(ifptfrc),
                           pt.ctypes.data_as(_dp), _byref_i(ifstrain), st.ctypes.data_as(_dp), _byref_i(m),
                           tg.ctypes.data_as(_dp), _byref_i(ifptfrctarg), ptt.ctypes.data_as(_dp),
                           _byref_i(ifstraintarg), stt.ctypes.data_as(_dp), _byref_i(icomp_type),
                           wsave.ctypes.data_as(_dp), _byref_i(wsave.size), ctypes.byref(lused))
    return ier.value, lused.value, pt, st, ptt[:m], stt[:m]


def elfmm3dtriaiter(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl=None, sigma_dl=None,
                    icomp_type=1, wsave=None, ifptfrc=1, ifstrain=1):
    """On-surface ITER variant (src/elfmm3dtria_iter_1.f:43).
    Returns (ier, lused, ptfrc, strain)."""
    ier, lused, pt, st, _, _ = elfmm3dtriatargiter(iprec, rlam, rmu, triangle, trinorm, source, sigma_sl,
                                                   sigma_dl, None, icomp_type, wsave, ifptfrc, ifstrain, 0, 0)
    return ier, lused, pt, st


def hs_capped():
    """Sub-triangles of the image quadrature kept at the adaptive depth cap
    since the last call (and clears the count)."""
    L = load()
    L.efmm_hs_capped.restype = ctypes.c_int
    return int(L.efmm_hs_capped())


def gcr_dense_host(A, B, tol=1e-10, maxit=50):
    """The solver's iteration on the host for a dense matrix (efmm_gcr_dense_host):
    A (n,n), B (nrhs,n).  Returns (X (nrhs,n), iterations, relative
    residuals, ier per column)."""
    L = load()
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64).reshape(-1, A.shape[0])
    R, n = B.shape
    X = np.zeros((R, n))
    its = np.zeros(R, dtype=np.int32)
    rel = np.zeros(R)
    ier_c = np.zeros(R, dtype=np.int32)
    L.efmm_gcr_dense_host.restype = ctypes.c_int
    ier = L.efmm_gcr_dense_host(n, R, A.ctypes.data_as(_dp), B.ctypes.data_as(_dp), X.ctypes.data_as(_dp),
                                ctypes.c_double(tol), int(maxit), its.ctypes.data_as(_ip), rel.ctypes.data_as(_dp),
                                ier_c.ctypes.data_as(_ip))
    if ier:
        raise ElfmmError(ier, "gcr_dense_host")
    return X, its, rel, ier_c


def tune_dump():
    """The autotuner's keys and decisions, one line each:
    "knob p nbox C prec kind decided ms0 ms1" (efmm_tune_dump)."""
    L = load()
    L.efmm_tune_dump.restype = ctypes.c_int
    n = L.efmm_tune_dump(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    L.efmm_tune_dump(buf, n + 1)
    return [l for l in buf.value.decode().splitlines() if l]


def iter_release(wsave):
    """Free the device store an ITER handle names; returns ier (512 if none)."""
    return int(load().efmm_iter_release(wsave.ctypes.data_as(_dp), int(wsave.size)))


def iter_stored_bytes(wsave):
    """Device bytes held by the store an ITER handle names (-1 if none)."""
    return int(load().efmm_iter_stored_bytes(wsave.ctypes.data_as(_dp), int(wsave.size)))


class Plan:
    """Device-resident plan (native API).  Arguments are CUDA tensors (torch)
    or raw device addresses (int); float64, contiguous, user order."""

    def __init__(self, device=0):
        L = load()
        _need_gpu()
        self._L = L
        self._h = L.efmm_plan_create(int(device))
        if not self._h:
            raise ElfmmError(1024, f"cannot create plan on device {device}")

    @staticmethod
    def _ptr(t):
        if t is None:
            return None
        if isinstance(t, int):
            return t
        return t.data_ptr()

    def set_geometry(self, tri, nrm, src, tgt=None, iprec=2, iter=False, mindlin=False):
        n = int(src.shape[0]) if hasattr(src, "shape") else None
        nt = int(tgt.shape[0]) if tgt is not None else 0
        ier = self._L.efmm_plan_set_geometry(self._h, n, self._ptr(tri), self._ptr(nrm), self._ptr(src), nt,
                                             self._ptr(tgt), int(iprec), int(iter), int(mindlin))
        if ier:
            raise ElfmmError(ier, "set_geometry")
        self.n, self.nt = n, nt

    def evaluate(self, rlam, rmu, ssl=None, sdl=None, u=None, e=None, ut=None, et=None, direct=False, mode=0):
        """mode 1: store the near-field interactions (ITER first call; geometry
        set with iter=True), mode 2: reuse them."""
        if mode:
            ier = self._L.efmm_plan_evaluate_iter(self._h, float(rlam), float(rmu), self._ptr(ssl), self._ptr(sdl),
                                                  self._ptr(u), self._ptr(e), self._ptr(ut), self._ptr(et), int(mode))
            if ier:
                raise ElfmmError(ier, "evaluate (iter)")
            return
        f = self._L.efmm_plan_evaluate_direct if direct else self._L.efmm_plan_evaluate
        ier = f(self._h, float(rlam), float(rmu), self._ptr(ssl), self._ptr(sdl), self._ptr(u),
                self._ptr(e), self._ptr(ut), self._ptr(et))
        if ier:
            raise ElfmmError(ier, "evaluate")

    def evaluate_batch(self, rlam, rmu, nrhs, ssl=None, sdl=None, u=None, e=None, ut=None, et=None,
                       precision=0, mode=0, graph=False):
        """nrhs right-hand sides in one pass: ssl/sdl (nrhs,n,3); outputs
        (nrhs,n,3), (nrhs,n,3,3), (nrhs,nt,3), (nrhs,nt,3,3).  precision 0 =
        FP64, 1 = mixed (FP32 expansions and translations).  mode 1 stores the
        near-field interactions (geometry set with iter=True), mode 2 reuses
        them.  graph=True replays repeated calls (same buffers) as one CUDA
        graph (mode 0 or 2)."""
        args = (self._h, float(rlam), float(rmu), int(nrhs), self._ptr(ssl), self._ptr(sdl), self._ptr(u),
                self._ptr(e), self._ptr(ut), self._ptr(et), int(precision))
        if graph:
            ier = self._L.efmm_plan_evaluate_batch_graph(*args, int(mode))
        elif mode:
            ier = self._L.efmm_plan_evaluate_batch_iter(*args, int(mode))
        else:
            ier = self._L.efmm_plan_evaluate_batch(*args)
        if ier:
            raise ElfmmError(ier, "evaluate_batch")

    def solve(self, image, kind, rlam, rmu, nrhs, nrm, rhs, x, tol=1e-8, maxit=30, precision=0):
        """Iterative solution over the operator (efmm_plan_solve, the minimal-
        residual iteration of the reference's matlab/gmres_simple.m on the
        device): rhs (nrhs,n,3) -> x (nrhs,n,3), CUDA tensors.  image: the
        half-space image Plan or None.  kind 0: x = slip (double layer),
        operator = traction on nrm at the centroids; kind 1: x = traction
        (single layer), operator = displacement at the centroids.  Returns
        (iterations, relative residuals, ier per column) as numpy arrays."""
        R = int(nrhs)
        its = np.zeros(R, dtype=np.int32)
        rel = np.zeros(R)
        ier_c = np.zeros(R, dtype=np.int32)
        L = self._L
        L.efmm_plan_solve.restype = ctypes.c_int
        L.efmm_plan_solve.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp,
                                      _vp, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _ip, _dp, _ip]
        ier = L.efmm_plan_solve(self._h, image._h if image is not None else None, int(kind), float(rlam), float(rmu),
                                R, self._ptr(nrm), self._ptr(rhs), self._ptr(x), float(tol), int(maxit),
                                int(precision), its.ctypes.data_as(_ip), rel.ctypes.data_as(_dp),
                                ier_c.ctypes.data_as(_ip))
        if ier:
            raise ElfmmError(ier, "solve")
        return its, rel, ier_c

    def evaluate_image(self, rlam, rmu, nrhs, ssl=None, sdl=None, ut=None, et=None, precision=0, mode=0,
                       graph=False):
        """Half-space image part at the points x whose reflections (x1, x2,
        -x3) were given as this plan's targets (set_geometry(..., mindlin=True)):
        ssl/sdl (nrhs,n,3); outputs ut (nrhs,nt,3), et (nrhs,nt,3,3).
        graph=True replays repeated mode-2 calls (same buffers) as one CUDA graph."""
        if graph:
            ier = self._L.efmm_plan_evaluate_image_graph(self._h, float(rlam), float(rmu), int(nrhs),
                                                         self._ptr(ssl), self._ptr(sdl), self._ptr(ut),
                                                         self._ptr(et), int(precision))
        else:
            ier = self._L.efmm_plan_evaluate_image(self._h, float(rlam), float(rmu), int(nrhs), self._ptr(ssl),
                                                   self._ptr(sdl), self._ptr(ut), self._ptr(et), int(precision),
                                                   int(mode))
        if ier:
            raise ElfmmError(ier, "evaluate_image")

    def record(self, slot):
        """Record CUDA event `slot` (0..7) on the plan's stream."""
        if self._L.efmm_plan_record(self._h, int(slot)):
            raise ElfmmError(16, "record")

    def elapsed(self, a, b):
        """Device milliseconds between recorded slots a and b."""
        return float(self._L.efmm_plan_elapsed(self._h, int(a), int(b)))

    def timings(self):
        a = (ctypes.c_float * 8)()
        self._L.efmm_plan_timings(self._h, a)
        return dict(zip(["total", "prep", "p2m", "m2m", "m2l", "l2l", "l2t", "near"], list(a)))

    def product_stats(self):
        """(device ms, useful flops) of the P2M product stage of the last batch."""
        a = (ctypes.c_double * 2)()
        self._L.efmm_plan_product_stats(self._h, a)
        return float(a[0]), float(a[1])

    def near_stats(self):
        """(device ms, bytes) of the tensor-core product of the last mixed
        replay of the stored near field from its split (zeros otherwise)."""
        a = (ctypes.c_double * 2)()
        self._L.efmm_plan_near_stats(self._h, a)
        return float(a[0]), float(a[1])

    def evaluate_direct_subset(self, rlam, rmu, nsub, ssl=None, sdl=None, u=None, e=None):
        """Direct sum at the first nsub centroids: u (nsub,3), e (nsub,3,3)."""
        ier = self._L.efmm_plan_evaluate_direct_subset(self._h, float(rlam), float(rmu), int(nsub),
                                                       self._ptr(ssl), self._ptr(sdl), self._ptr(u), self._ptr(e))
        if ier:
            raise ElfmmError(ier, "evaluate_direct_subset")

    def stored_bytes(self):
        """Device bytes of the stored near field (ITER), 0 if none."""
        return int(self._L.efmm_plan_stored_bytes(self._h))

    def set_mixed_floor(self, eps):
        """Truncation floor of the mixed form (precision=1): its orders follow
        max(eps(iprec), eps); eps <= 0 keeps the iprec orders.  Returns the
        mixed form's expansion order."""
        order = ctypes.c_int()
        ier = self._L.efmm_plan_set_mixed_floor(self._h, float(eps), ctypes.byref(order))
        if ier:
            raise ElfmmError(ier, "set_mixed_floor")
        return order.value

    def translation_flops(self, nrhs, precision=1):
        """Flops of one pass's translation launches (M2M, M2L, L2L) for nrhs
        right-hand sides at the orders of the given form."""
        a = (ctypes.c_double * 3)()
        ier = self._L.efmm_plan_translation_flops(self._h, int(nrhs), int(precision), a)
        if ier:
            raise ElfmmError(ier, "translation_flops")
        return dict(zip(["m2m", "m2l", "l2l"], list(a)))

    def flops_per_column(self):
        """Useful flops per expansion column: P2M, M2M, M2L, L2L, L2T."""
        a = (ctypes.c_double * 5)()
        self._L.efmm_plan_flops(self._h, a)
        return dict(zip(["p2m", "m2m", "m2l", "l2l", "l2t"], list(a)))

    def setup_timings(self):
        """Host milliseconds of the last set_geometry, by phase."""
        a = (ctypes.c_float * 4)()
        self._L.efmm_plan_setup_timings(self._h, a)
        return dict(zip(["tree", "lists", "worklists", "operators"], list(a)))

    def info(self):
        a = (ctypes.c_longlong * 8)()
        self._L.efmm_plan_info(self._h, a)
        return dict(zip(["nboxes", "nlev", "p", "nbox", "near_pairs", "m2l_pairs", "launches", "far"],
                        list(a)))

    def tree(self):
        """Tree in the reference's layout (1-based ids): dict with boxes (nb,20),
        iz, iztarg, laddr (nlev+1,2), center, size, lists {1..5: [array per box]}."""
        info = self.info()
        nb, nlev = info["nboxes"], info["nlev"]
        lc = (ctypes.c_longlong * 5)()
        z = ctypes.POINTER(ctypes.c_int)()
        self._L.efmm_plan_tree_export(self._h, z, z, z, z, ctypes.POINTER(ctypes.c_double)(), z, z, lc)
        tot = int(sum(lc))
        boxes = np.zeros((nb, 20), dtype=np.int32)
        iz = np.zeros(max(self.n, 1), dtype=np.int32)
        izt = np.zeros(max(self.nt, 1), dtype=np.int32)
        laddr = np.zeros((nlev + 1, 2), dtype=np.int32)
        cs = np.zeros(4)
        lstart = np.zeros((5, nb + 1), dtype=np.int32)
        litems = np.zeros(max(tot, 1), dtype=np.int32)
        ier = self._L.efmm_plan_tree_export(self._h, boxes.ctypes.data_as(_ip), iz.ctypes.data_as(_ip),
                                            izt.ctypes.data_as(_ip), laddr.ctypes.data_as(_ip),
                                            cs.ctypes.data_as(_dp), lstart.ctypes.data_as(_ip),
                                            litems.ctypes.data_as(_ip), lc)
        if ier:
            raise ElfmmError(ier, "tree_export")
        lists = {}
        off = 0
        for t in range(5):
            items = litems[off:off + lc[t]]
            off += lc[t]
            st = lstart[t]
            lists[t + 1] = [items[st[b]:st[b + 1]].copy() for b in range(nb)]
        return dict(boxes=boxes, iz=iz[:self.n], iztarg=izt[:self.nt], laddr=laddr, center=cs[:3],
                    size=cs[3], lists=lists)

    def set_forest(self, forest):
        """Forest of independent problems for the following set_geometry
        calls (efmm_plan_set_forest): (centre x, y, z, side, level), or None."""
        f = None if forest is None else np.ascontiguousarray(forest, dtype=np.float64).reshape(5)
        ier = self._L.efmm_plan_set_forest(self._h, f.ctypes.data_as(_dp) if f is not None else None)
        if ier:
            raise ElfmmError(ier, "set_forest")

    @classmethod
    def _view(cls, L, h, n, nt):
        """A non-owning Plan over handle h (a forest's plan)."""
        v = cls.__new__(cls)
        v._L, v._h, v._owned, v.n, v.nt = L, h, False, n, nt
        return v

    def close(self):
        if getattr(self, "_h", None) and getattr(self, "_owned", True):
            self._L.efmm_plan_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def forest_layout(bb):
    """The forest placement (efmm_forest_layout, host code): bb (nprob,6)
    centroid boxes (min x, y, z, max x, y, z) -> (root (5,), shift (nprob,2))."""
    L = load()
    bb = _c(bb, (-1, 6))
    root, shift = np.zeros(5), np.zeros((bb.shape[0], 2))
    ier = L.efmm_forest_layout(bb.shape[0], bb.ctypes.data_as(_dp), root.ctypes.data_as(_dp),
                               shift.ctypes.data_as(_dp))
    if ier:
        raise ElfmmError(ier, "forest_layout")
    return root, shift


class Forest:
    """Many independent half-space problems in one pass (efmm_forest_*):
    device arrays (torch CUDA tensors or addresses) concatenated in problem
    order, counts = triangles per problem."""

    def __init__(self, device=0):
        L = load()
        _need_gpu()
        self._L = L
        self._h = L.efmm_forest_create(int(device))
        if not self._h:
            raise ElfmmError(1024, f"cannot create forest on device {device}")
        self.n = 0

    def set_mixed_floor(self, eps):
        """Tolerance floor of both plans' mixed-form orders (<= 0: the iprec
        orders)."""
        ier = self._L.efmm_forest_set_mixed_floor(self._h, float(eps))
        if ier:
            raise ElfmmError(ier, "forest set_mixed_floor")

    def set_leaf(self, nbox_free=0, nbox_image=0):
        """Leaf capacities of the two plans for the next set_geometry (<= 0:
        the default: the iprec table for the free-space plan, half of it for
        the image plan)."""
        self._L.efmm_forest_set_leaf(self._h, int(nbox_free), int(nbox_image))

    def set_geometry(self, counts, tri, nrm, cen, iprec=2, iter=False):
        c = np.ascontiguousarray(counts, dtype=np.int32)
        ier = self._L.efmm_forest_set_geometry(self._h, len(c), c.ctypes.data_as(_ip), Plan._ptr(tri),
                                               Plan._ptr(nrm), Plan._ptr(cen), int(iprec), int(iter))
        if ier:
            raise ElfmmError(ier, "forest set_geometry")
        self.n = int(c.sum())

    def evaluate(self, rlam, rmu, ssl=None, sdl=None, u=None, e=None, precision=1, mode=0):
        """Half-space u (n,3), e (n,3,3) at every problem's centroids."""
        ier = self._L.efmm_forest_evaluate(self._h, float(rlam), float(rmu), Plan._ptr(ssl), Plan._ptr(sdl),
                                           Plan._ptr(u), Plan._ptr(e), int(precision), int(mode))
        if ier:
            raise ElfmmError(ier, "forest evaluate")

    def plan(self, which):
        """The free-space (0) or image (1) plan, as a non-owning Plan."""
        h = self._L.efmm_forest_plan(self._h, int(which))
        return Plan._view(self._L, h, self.n, 0 if which == 0 else self.n)

    def close(self):
        if getattr(self, "_h", None):
            self._L.efmm_forest_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_many_host_mixed_floor(eps):
    """Tolerance floor of the mixed-form orders of the forest behind
    hs_many_host (efmm_many_host_set_mixed_floor; <= 0: the iprec orders)."""
    load().efmm_many_host_set_mixed_floor(float(eps))


def hs_many_host(iprec, rlam, rmu, counts, triangle, trinorm, centroids, sigma_sl=None, sigma_dl=None,
                 precision=1):
    """elhfmm3dtria_many_host: the half-space self-evaluation of many
    independent problems from host arrays concatenated in problem order.
    Returns (ier, u (n,3), strain (n,3,3))."""
    L = load()
    _need_gpu()
    c = np.ascontiguousarray(counts, dtype=np.int32)
    tri = _c(triangle, (-1, 3, 3))
    n = tri.shape[0]
    nrm, cen = _c(trinorm, (n, 3)), _c(centroids, (n, 3))
    ssl = _c(sigma_sl, (n, 3)) if sigma_sl is not None else None
    sdl = _c(sigma_dl, (n, 3)) if sigma_dl is not None else None
    u, e = np.zeros((n, 3)), np.zeros((n, 3, 3))
    p = lambda a: a.ctypes.data_as(_dp) if a is not None else None
    ier = L.elhfmm3dtria_many_host(int(iprec), float(rlam), float(rmu), len(c), c.ctypes.data_as(_ip), p(tri),
                                   p(nrm), p(cen), p(ssl), p(sdl), p(u), p(e), int(precision))
    return ier, u, e
