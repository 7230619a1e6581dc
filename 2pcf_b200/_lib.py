"""ctypes declarations of the C ABI in include/tpcf_b200.h.

The shared library is built in-tree (2pcf_b200/libtpcf_b200.so) by
``python -c "import __graft_entry__ as g; g.build()"`` or ``make -C
2pcf_b200/csrc``.  Loading fails loudly when it is missing: there is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtpcf_b200.so")

TPCF_OK = 0
STATUS_NAMES = {
    0: "TPCF_OK", 1: "TPCF_ERR_INVALID_ARG", 2: "TPCF_ERR_OOM", 3: "TPCF_ERR_OVERFLOW",
    4: "TPCF_ERR_TIMEOUT", 5: "TPCF_ERR_CUDA", 6: "TPCF_ERR_NOT_SUPPORTED", 7: "TPCF_ERR_NO_DEVICE",
}
globals().update({name: code for code, name in STATUS_NAMES.items()})

# Every symbol declared in include/tpcf_b200.h (checked by tests/test_abi.py).
EXPORTED = []


class Bins(C.Structure):
    _fields_ = [("n_bin", C.c_int32), ("spacing", C.c_int32), ("x_min", C.c_double),
                ("x_max", C.c_double), ("ihs_theta", C.c_double)]


class Opts(C.Structure):
    _fields_ = [("use_grid", C.c_int32), ("verbose", C.c_int32), ("cell_size", C.c_double),
                ("spherical", C.c_int32), ("shard_index", C.c_int32), ("shard_count", C.c_int32),
                ("group_size", C.c_int32), ("tile_chunks", C.c_int32), ("reserved", C.c_int32 * 3)]


class Result(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "sum_dw", "sum_gt", "sum_gx", "sum_w", "sum_K", "n_pairs",
        "theta", "mean_theta", "g_t", "g_x", "weights",
        "xi_E_marks", "xi_B_marks", "K_marks", "w_marks", "marks_weight",
        "lens_sums", "patch_sums", "lens_raw")]


class LensCat(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(n, C.c_void_p) for n in ("x", "y", "z", "val", "w", "patch")]


class ShearCat(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(n, C.c_void_p) for n in ("x", "y", "z", "e1", "e2", "w", "m")]


class KappaCat(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(n, C.c_void_p) for n in ("x", "y", "kE", "kB", "w")]


class Stats(C.Structure):
    _fields_ = [("pair_kernel_ms", C.c_double), ("call_ms", C.c_double), ("n_pairs", C.c_int64),
                ("h2d_bytes", C.c_int64), ("kernel_launches", C.c_int64), ("workspace_bytes", C.c_int64)]


class LensGrad(C.Structure):
    _fields_ = [("val", C.c_void_p), ("w", C.c_void_p)]


class ShearGrad(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("e1", "e2", "w", "m")]


class AdjointTask(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("sum_gt", "sum_gx", "sum_K", "lens_raw", "dL_dgt", "dL_dgx")]


class MarksFieldC(C.Structure):
    _fields_ = [("n", C.c_int64), ("n_bin", C.c_int64)] + [
        (n, C.c_void_p) for n in ("x", "y", "w", "xi_E", "xi_B", "K")]


class TPCFError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")


_lib = None


def _sig(L, name, restype, argtypes):
    fn = getattr(L, name)
    fn.restype = restype
    fn.argtypes = argtypes
    if name not in EXPORTED:
        EXPORTED.append(name)


def lib():
    """Load libtpcf_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                          "(the library has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, st = C.c_void_p, C.c_int32, C.c_int64, C.c_int
    _sig(L, "tpcf_abi_version", i32, [])
    _sig(L, "tpcf_create", st, [C.POINTER(vp), i32, C.POINTER(Opts)])
    _sig(L, "tpcf_destroy", st, [vp])
    _sig(L, "tpcf_last_error", C.c_char_p, [vp])
    _sig(L, "tpcf_set_stream", st, [vp, vp])
    _sig(L, "tpcf_kernel_launches", i64, [vp])
    _sig(L, "tpcf_set_timing", st, [vp, i32])
    _sig(L, "tpcf_last_stats", st, [vp, C.POINTER(Stats)])
    _sig(L, "tpcf_set_shard", st, [vp, i32, i32])
    _sig(L, "tpcf_set_cell_size", st, [vp, C.c_double])
    _sig(L, "tpcf_set_tile_shape", st, [vp, i32, i32])
    _sig(L, "tpcf_debug_inject", st, [vp, i64, i32, C.c_uint32])
    _sig(L, "tpcf_measure_fp32_peak", st, [vp, C.POINTER(C.c_double)])
    _sig(L, "tpcf_measure_fp64_peak", st, [vp, C.POINTER(C.c_double)])
    _sig(L, "tpcf_canonical_edges", st, [C.POINTER(Bins), vp, vp])
    _sig(L, "tpcf_bin_centers", st, [C.POINTER(Bins), vp])
    _sig(L, "tpcf_set_spherical", st, [vp, i32])
    _sig(L, "tpcf_chord_edges", st, [C.POINTER(Bins), vp])
    _sig(L, "tpcf_unit_vectors", st, [vp, vp, vp, i64, vp, vp])
    _sig(L, "tpcf_rotate_from_poles", st, [vp, vp, vp, i64, vp, vp, i64, C.c_float, C.POINTER(i32), vp])
    _sig(L, "tpcf_read_table", st, [C.c_char_p, i32, i32, i32, i32, vp, i64, C.POINTER(i64)])
    _sig(L, "tpcf_write_result_table", st, [C.c_char_p, i32, vp, vp, vp, vp, vp, vp, i32])
    _sig(L, "tpcf_marks_save", st, [C.c_char_p, i32, C.POINTER(MarksFieldC)])
    _sig(L, "tpcf_marks_info", st, [C.c_char_p, i32, C.POINTER(i32), vp, vp])
    _sig(L, "tpcf_marks_load", st, [C.c_char_p, i32, C.POINTER(MarksFieldC)])
    _sig(L, "tpcf_marks_bootstrap", st, [vp, i32, C.POINTER(MarksFieldC), vp, i64, vp, C.c_uint64, i32,
                                         C.c_double, i32] + [vp] * 5)
    _sig(L, "tpcf_xi_from_marks", st, [vp, i32, C.POINTER(MarksFieldC), i32, vp, vp, vp, vp] + [vp] * 6)
    _sig(L, "tpcf_shear_scalar", st, [vp] + [vp] * 5 + [i64] + [vp] * 7 + [i64] +
         [C.POINTER(Bins), vp, i32, C.POINTER(Result)])
    _sig(L, "tpcf_scalar_scalar", st, [vp] + [vp] * 4 + [i64] + [vp] * 5 + [i64] +
         [C.POINTER(Bins), vp, i32, C.POINTER(Result)])
    _sig(L, "tpcf_batch_shear_scalar", st, [vp, i32, C.POINTER(LensCat), i32, C.POINTER(ShearCat),
                                            i32, vp, vp, C.POINTER(Bins), i32, C.POINTER(Result)])
    _sig(L, "tpcf_plan_shear_scalar", st, [vp, i32, C.POINTER(LensCat), i32, C.POINTER(ShearCat),
                                           i32, vp, vp, C.POINTER(Bins), i32, C.POINTER(Result), C.POINTER(vp)])
    _sig(L, "tpcf_plan_launch", st, [vp])
    _sig(L, "tpcf_plan_results", st, [vp, C.POINTER(Result)])
    _sig(L, "tpcf_plan_set_stream", st, [vp, vp])
    _sig(L, "tpcf_plan_last_error", C.c_char_p, [vp])
    _sig(L, "tpcf_plan_destroy", st, [vp])
    _sig(L, "tpcf_shear_scalar_noalloc", st, [vp] + [vp] * 5 + [i64] + [vp] * 7 + [i64] +
         [C.POINTER(Bins), C.POINTER(Result)])
    _sig(L, "tpcf_shear_scalar_adjoint", st, [vp] + [vp] * 5 + [i64] + [vp] * 7 + [i64] +
         [C.POINTER(Bins)] + [vp] * 4 + [vp] * 2 + [vp] * 6)
    _sig(L, "tpcf_batch_scalar_scalar", st, [vp, i32, C.POINTER(LensCat), i32, C.POINTER(KappaCat),
                                             i32, vp, vp, C.POINTER(Bins), i32, C.POINTER(Result)])
    _sig(L, "tpcf_batch_shear_scalar_adjoint", st, [vp, i32, C.POINTER(LensCat), C.POINTER(LensGrad), i32,
                                                    C.POINTER(ShearCat), C.POINTER(ShearGrad), i32, vp, vp,
                                                    C.POINTER(Bins), C.POINTER(AdjointTask)])
    _sig(L, "tpcf_kmeans", st, [vp, vp, vp, vp, i64, i32, i32, C.c_float, vp, vp, C.POINTER(i32)])
    _sig(L, "tpcf_kmeans_equal", st, [vp, vp, vp, vp, i64, i32, i32, C.c_float, C.c_float, C.c_float, i32,
                                      C.c_uint64, vp, vp, C.POINTER(i32), C.POINTER(C.c_float)])
    _sig(L, "tpcf_bootstrap", st, [vp, vp, i32, i32, i32, vp, C.c_uint64, i32, C.c_double,
                                   vp, vp, vp, vp, vp, vp])
    _declare_extra(L)
    if L.tpcf_abi_version() != 1:
        raise ImportError("libtpcf_b200.so ABI version mismatch")
    _lib = L
    return L


def _declare_extra(L):
    """Entry points added after the pair sums (k-means, bootstrap, adjoint)."""
    vp, i32, i64, st = C.c_void_p, C.c_int32, C.c_int64, C.c_int
    for name, res, args in EXTRA_SIGNATURES:
        if hasattr(L, name):
            _sig(L, name, res, args)


EXTRA_SIGNATURES = []
