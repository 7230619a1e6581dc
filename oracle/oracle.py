"""ctypes front end of the CPU oracle (oracle/tpcf_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py`` as the checker.  The product library never
imports this module.

PARITY STATUS: unpinned -- the Fortran reference cannot be compiled on these
machines and its tests hold no golden vectors for the pair sums.  See the header
of tpcf_oracle.cpp for the reference lines each routine restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

LIN, LOG, IHS, SQRT = 0, 1, 2, 3
SHEAR, KAPPA = 0, 1

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liboracle.so with the committed Makefile (no-op when current)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        L.orc_create_bins_f32.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, C.c_float,
                                          _f32p, _f32p, C.POINTER(C.c_float)]
        L.orc_find_bin_f32.argtypes = [_f32p, C.c_long, C.c_float, C.c_float, C.c_int, C.c_int,
                                       C.c_float, _i32p]
        L.orc_canonical_edges.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                                          _f64p, _f64p]
        L.orc_canonical_bin.argtypes = [_f64p, C.c_long, _f64p, C.c_int, _i32p]
        for name in ("orc_ref_pairs_f32", "orc_ref_pairs_f64"):
            fn = getattr(L, name)
            fn.argtypes = ([C.c_int, C.c_long] + [vp] * 5 + [C.c_long] + [vp] * 7 +
                           ([C.c_float] * 2 if name.endswith("f32") else [C.c_double] * 2) +
                           [C.c_int, C.c_int] +
                           ([C.c_float] if name.endswith("f32") else [C.c_double]) +
                           [C.c_int, C.c_int] + [vp] * 4 + [vp] + [vp] * 5)
        L.orc_canon_pairs.argtypes = ([C.c_int, C.c_long] + [vp] * 5 + [C.c_long] + [vp] * 7 +
                                      [_f64p, C.c_int, C.c_int, _f64p, vp, C.c_long, vp])
        L.orc_kdtree_search.argtypes = [C.c_long, _f32p, _f32p, C.c_float, C.c_float, C.c_float,
                                        C.c_int, C.c_int, _i64p, C.c_long, C.POINTER(C.c_long)]
        L.orc_kmeans_ref_f32.argtypes = [C.c_long, _f32p, _f32p, _f32p, C.c_int, C.c_int,
                                         C.c_float, C.c_int, C.c_float, C.c_float, _i32p, _f32p,
                                         _f32p, C.POINTER(C.c_int)]
        L.orc_kmeans_det.argtypes = [C.c_long, _f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_float,
                                     _i32p, _f32p, _f32p, C.POINTER(C.c_int)]
        L.orc_fixed_scale.argtypes = [C.c_long, C.c_double]
        L.orc_qsort_arg_f32.argtypes = [_f32p, C.c_long, _i64p, C.c_int]
        L.orc_bootstrap_multiplicity.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, _i32p]
        L.orc_block_bootstrap.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _f64p, _f64p, _f64p,
                                          _f64p, _f64p, _f64p, _f64p]
        L.orc_covariance.argtypes = [C.c_int, C.c_int, _f64p, _f64p]
        L.orc_last_timing.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_canon_adjoint.argtypes = ([C.c_long] + [vp] * 5 + [C.c_long] + [vp] * 7 +
                                        [_f64p, C.c_int, _f64p, _f64p, C.c_int] + [_f64p] * 6)
        L.orc_canon_adjoint_sel.argtypes = ([C.c_long] + [vp] * 5 + [C.c_long] + [vp] * 7 +
                                            [_f64p, C.c_int] + [_f64p] * 5 + [vp, C.c_long, vp, C.c_long,
                                                                               C.c_int] + [vp] * 6)
        L.orc_ref_sphere_f32.argtypes = ([C.c_int, C.c_long] + [vp] * 5 + [C.c_long] + [vp] * 7 +
                                         [C.c_float, C.c_float, C.c_int, C.c_int, C.c_float, C.c_int] +
                                         [vp] * 4)
        L.orc_canon_sphere.argtypes = ([C.c_int, C.c_long] + [vp] * 5 + [C.c_long] + [vp] * 7 +
                                       [_f64p, C.c_int, C.c_int, _f64p])
        L.orc_sphere_edges_sq.argtypes = [_f64p, C.c_int, _f64p]
        L.orc_unit_vectors.argtypes = [C.c_long, vp, vp, vp, vp]
        L.orc_kmeans_equal_det.argtypes = [C.c_long, vp, vp, vp, C.c_int, C.c_int, C.c_float, C.c_float,
                                           C.c_float, C.c_int, C.c_uint64, vp, vp, vp, C.POINTER(C.c_int),
                                           C.POINTER(C.c_float)]
        L.orc_rotate_from_poles.argtypes = [vp, vp, C.c_long, vp, vp, C.c_long, C.c_float,
                                            C.POINTER(C.c_int), vp]
        _u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
        L.orc_philox4x32.argtypes = [_u32p, _u32p, _u32p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------------ binning --
def create_bins_f32(x_min, x_max, n_bin, spacing=LOG, p=1.0):
    """Reference create_bins in FP32 (src/utils.f90:139-230)."""
    edges = np.zeros(n_bin + 1, np.float32)
    centers = np.zeros(n_bin, np.float32)
    bs = C.c_float()
    rc = lib().orc_create_bins_f32(x_min, x_max, n_bin, spacing, p, edges, centers, C.byref(bs))
    if rc:
        raise ValueError("bad binning")
    return edges, centers, bs.value


def find_bin_f32(d, x_min, x_max, n_bin, spacing=LOG, p=1.0):
    """Reference find_bin_index in FP32, 0-based (-1 = no bin); src/utils.f90:101-137."""
    d = np.ascontiguousarray(d, np.float32)
    out = np.empty(d.size, np.int32)
    lib().orc_find_bin_f32(d, d.size, x_min, x_max, n_bin, spacing, p, out)
    return out


def canonical_edges(x_min, x_max, n_bin, spacing=LOG, p=1.0):
    """Canonical FP64 edges and squared edges (the library's bin rule)."""
    e = np.zeros(n_bin + 1)
    e2 = np.zeros(n_bin + 1)
    if lib().orc_canonical_edges(x_min, x_max, n_bin, spacing, p, e, e2):
        raise ValueError("bad binning")
    return e, e2


def canonical_bin(d2, e2):
    d2 = np.ascontiguousarray(d2, np.float64)
    out = np.empty(d2.size, np.int32)
    lib().orc_canonical_bin(d2, d2.size, np.ascontiguousarray(e2, np.float64), len(e2) - 1, out)
    return out


# ---------------------------------------------------------- reference loops --
def ref_pairs(mode, lens, src, x_min, x_max, n_bin, spacing=LOG, p=1.0, use_kd_tree=True,
              num_threads=1, marks=False, dtype=np.float32):
    """Restatement of tangential_shear_tpcf / scalar_kappa_tpcf (src/tpcf.f90:190-545).

    ``lens``: dict with x, y, z, val, w.  ``src``: shear dict with x, y, z, e1, e2,
    w, m, or kappa dict with x, y, kappa_E, kappa_B, w.  Returns a dict with the
    reference outputs (avg_theta, g_t, g_x, weights, n_pairs and, if asked,
    the marks arrays in [n_A][n_bin] layout)."""
    dt = np.dtype(dtype)
    cv = lambda a: None if a is None else np.ascontiguousarray(a, dt)
    nA, nB = len(lens["x"]), len(src["x"])
    xA, yA, vA, wA = (cv(lens[k]) for k in ("x", "y", "val", "w"))
    zA = cv(lens.get("z")) if mode == SHEAR else None
    if mode == SHEAR:
        xB, yB, zB, e1, e2, wB, mB = (cv(src[k]) for k in ("x", "y", "z", "e1", "e2", "w", "m"))
    else:
        xB, yB, e1, e2, wB = (cv(src[k]) for k in ("x", "y", "kappa_E", "kappa_B", "w"))
        zB = mB = None
    out = {k: np.zeros(n_bin, dt) for k in ("avg_theta", "g_t", "g_x", "weights")}
    out["n_pairs"] = np.zeros(n_bin, np.int64)
    mk = {}
    if marks:
        mk = {k: np.zeros((nA, n_bin), dt) for k in ("xi_E_marks", "xi_B_marks", "K_marks", "w_marks")}
        mk["marks_weight"] = np.zeros(nA, dt)
    fn = lib().orc_ref_pairs_f32 if dt == np.float32 else lib().orc_ref_pairs_f64
    rc = fn(mode, nA, _ptr(xA), _ptr(yA), _ptr(zA), _ptr(vA), _ptr(wA), nB, _ptr(xB), _ptr(yB),
            _ptr(zB), _ptr(e1), _ptr(e2), _ptr(wB), _ptr(mB), x_min, x_max, n_bin, spacing, p,
            int(use_kd_tree), num_threads, _ptr(out["avg_theta"]), _ptr(out["g_t"]),
            _ptr(out["g_x"]), _ptr(out["weights"]), _ptr(out["n_pairs"]),
            _ptr(mk.get("xi_E_marks")), _ptr(mk.get("xi_B_marks")), _ptr(mk.get("K_marks")),
            _ptr(mk.get("w_marks")), _ptr(mk.get("marks_weight")))
    if rc:
        raise RuntimeError(f"reference restatement failed with status {rc}")
    out.update(mk)
    return out


def last_timing():
    """(kd-tree build seconds, pair-loop seconds) of the last ref_pairs call."""
    a, b = C.c_double(), C.c_double()
    lib().orc_last_timing(C.byref(a), C.byref(b))
    return a.value, b.value


# ----------------------------------------------------------------- canonical --
# abs_*: sums of |term|; norm_*: sums of the bound on a term before its
# rotation (w_B |val_A w_A| |(e1, e2)| for shear, |term| for scalar fields), the
# scale of an FP32 evaluation's error in one rotated term.
CANON_Q = ("sum_dw", "sum_gt", "sum_gx", "sum_w", "sum_K", "n_pairs", "abs_gt", "abs_gx", "norm_gt", "norm_gx")
NQ = len(CANON_Q)


def canon_pairs(mode, lens, src, edges_sq, num_threads=None, lens_idx=None):
    """FP64 brute-force pair sums with the canonical bin rule.

    Returns a dict of per-bin FP64 arrays (CANON_Q) and, when ``lens_idx`` is
    given, ``lens`` = per-lens [n_sel][6][n_bin] sums (d*w, g_t, g_x, w, K, n)
    for those lenses (and the per-bin sums cover only those lenses), and
    ``lens_abs`` = per-lens [n_sel][2][n_bin] sums of |g_t terms|, |g_x terms|
    and ``lens_norm`` the per-lens norm_gt, norm_gx rows."""
    f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
    nA, nB = len(lens["x"]), len(src["x"])
    e2 = np.ascontiguousarray(edges_sq, np.float64)
    n_bin = len(e2) - 1
    xA, yA, vA, wA = (f(lens[k]) for k in ("x", "y", "val", "w"))
    zA = f(lens.get("z")) if mode == SHEAR else None
    if mode == SHEAR:
        xB, yB, zB, e1, e2b, wB, mB = (f(src[k]) for k in ("x", "y", "z", "e1", "e2", "w", "m"))
    else:
        xB, yB, e1, e2b, wB = (f(src[k]) for k in ("x", "y", "kappa_E", "kappa_B", "w"))
        zB = mB = None
    sums = np.zeros(NQ * n_bin)
    sel = None if lens_idx is None else np.ascontiguousarray(lens_idx, np.int64)
    lens_out = None if sel is None else np.zeros((len(sel), NQ, n_bin))
    nt = num_threads or os.cpu_count() or 1
    lib().orc_canon_pairs(mode, nA, _ptr(xA), _ptr(yA), _ptr(zA), _ptr(vA), _ptr(wA), nB, _ptr(xB),
                          _ptr(yB), _ptr(zB), _ptr(e1), _ptr(e2b), _ptr(wB), _ptr(mB), e2, n_bin,
                          nt, sums, _ptr(sel), 0 if sel is None else len(sel), _ptr(lens_out))
    sums = sums.reshape(NQ, n_bin)
    out = {k: sums[i].copy() for i, k in enumerate(CANON_Q)}
    if lens_out is not None:
        out["lens"] = np.ascontiguousarray(lens_out[:, :6])
        out["lens_abs"] = np.ascontiguousarray(lens_out[:, 6:8])  # sum|g_t terms|, sum|g_x terms|
        out["lens_norm"] = np.ascontiguousarray(lens_out[:, 8:10])
    return out


def canon_adjoint(lens, src, edges_sq, lam_t, lam_x=None, num_threads=None):
    """FP64 brute-force gradient of L = sum_b lam_t[b] xi_t,b + lam_x[b] xi_x,b
    (shear-scalar, canonical bins) w.r.t. val_A, w_A, e1_B, e2_B, w_B, m_B."""
    f = lambda a: np.ascontiguousarray(a, np.float32)
    nA, nB = len(lens["x"]), len(src["x"])
    nb = len(edges_sq) - 1
    A = [f(lens[k]) for k in ("x", "y", "z", "val", "w")]
    B = [f(src[k]) for k in ("x", "y", "z", "e1", "e2", "w", "m")]
    lt = np.ascontiguousarray(lam_t, np.float64)
    lx = np.zeros(nb) if lam_x is None else np.ascontiguousarray(lam_x, np.float64)
    out = [np.zeros(nA), np.zeros(nA)] + [np.zeros(nB) for _ in range(4)]
    lib().orc_canon_adjoint(nA, *[_ptr(a) for a in A], nB, *[_ptr(b) for b in B],
                            np.ascontiguousarray(edges_sq, np.float64), nb, lt, lx,
                            num_threads or os.cpu_count() or 1, *out)
    return dict(zip(("val_A", "w_A", "e1_B", "e2_B", "w_B", "m_B"), out))


def canon_adjoint_sel(lens, src, edges_sq, totals, lam_t, lam_x, lens_sel, src_sel, num_threads=None):
    """The FP64 brute-force gradient of canon_adjoint for selected lenses and
    sources only, given the per-bin totals ``totals`` = (sum_gt, sum_gx,
    sum_K) of the whole catalogue pair.  Returns val_A, w_A [len(lens_sel)]
    and e1_B, e2_B, w_B, m_B [len(src_sel)]."""
    f = lambda a: np.ascontiguousarray(a, np.float32)
    nA, nB = len(lens["x"]), len(src["x"])
    nb = len(edges_sq) - 1
    A = [f(lens[k]) for k in ("x", "y", "z", "val", "w")]
    B = [f(src[k]) for k in ("x", "y", "z", "e1", "e2", "w", "m")]
    d64 = lambda a: np.ascontiguousarray(a, np.float64)
    ls = np.ascontiguousarray(lens_sel, np.int64)
    ss = np.ascontiguousarray(src_sel, np.int64)
    lx = np.zeros(nb) if lam_x is None else d64(lam_x)
    out = [np.zeros(len(ls)), np.zeros(len(ls))] + [np.zeros(len(ss)) for _ in range(4)]
    lib().orc_canon_adjoint_sel(nA, *[_ptr(a) for a in A], nB, *[_ptr(b) for b in B], d64(edges_sq), nb,
                                d64(totals[0]), d64(totals[1]), d64(totals[2]), d64(lam_t), lx,
                                ls.ctypes.data, len(ls), ss.ctypes.data, len(ss),
                                num_threads or os.cpu_count() or 1, *[o.ctypes.data for o in out])
    return dict(zip(("val_A", "w_A", "e1_B", "e2_B", "w_B", "m_B"), out))


def sphere_edges_sq(edges):
    """Squared canonical chords (2 sin(e/2))^2 of FP64 angle edges (radians)."""
    e = np.ascontiguousarray(edges, np.float64)
    out = np.zeros_like(e)
    lib().orc_sphere_edges_sq(e, len(e) - 1, out)
    return out


def rotate_from_poles(xA, yA, r_max, xB=None, yB=None):
    """The reference's field rotation in FP32 (copies; returns rotated flag,
    centre and the four arrays)."""
    f = lambda a: None if a is None else np.array(a, np.float32, copy=True)
    xA, yA, xB, yB = f(xA), f(yA), f(xB), f(yB)
    r = C.c_int()
    center = np.zeros(2, np.float32)
    lib().orc_rotate_from_poles(_ptr(xA), _ptr(yA), len(xA), _ptr(xB), _ptr(yB), 0 if xB is None else len(xB),
                                r_max, C.byref(r), _ptr(center))
    return bool(r.value), center, xA, yA, xB, yB


def unit_vectors(lam, phi):
    """Canonical unit vectors (hi, lo) [n][3] of FP32 (lambda, phi) radians."""
    lam = np.ascontiguousarray(lam, np.float32)
    phi = np.ascontiguousarray(phi, np.float32)
    hi = np.zeros((len(lam), 3), np.float32)
    lo = np.zeros((len(lam), 3), np.float32)
    lib().orc_unit_vectors(len(lam), _ptr(lam), _ptr(phi), _ptr(hi), _ptr(lo))
    return hi, lo


def canon_sphere(mode, lens, src, edges_sq_chord, num_threads=None):
    """Canonical FP64 pair sums on the sphere (positions in radians)."""
    f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
    nA, nB = len(lens["x"]), len(src["x"])
    e2 = np.ascontiguousarray(edges_sq_chord, np.float64)
    nb = len(e2) - 1
    xA, yA, vA, wA = (f(lens[k]) for k in ("x", "y", "val", "w"))
    zA = f(lens.get("z")) if mode == SHEAR else None
    if mode == SHEAR:
        xB, yB, zB, e1, e2b, wB, mB = (f(src[k]) for k in ("x", "y", "z", "e1", "e2", "w", "m"))
    else:
        xB, yB, e1, e2b, wB = (f(src[k]) for k in ("x", "y", "kappa_E", "kappa_B", "w"))
        zB = mB = None
    sums = np.zeros(NQ * nb)
    lib().orc_canon_sphere(mode, nA, _ptr(xA), _ptr(yA), _ptr(zA), _ptr(vA), _ptr(wA), nB, _ptr(xB),
                           _ptr(yB), _ptr(zB), _ptr(e1), _ptr(e2b), _ptr(wB), _ptr(mB), e2, nb,
                           num_threads or os.cpu_count() or 1, sums)
    sums = sums.reshape(NQ, nb)
    return {k: sums[i].copy() for i, k in enumerate(CANON_Q)}


def ref_sphere_f32(mode, lens, src, x_min, x_max, n_bin, spacing=LOG, p=1.0, num_threads=1):
    """The reference's spherical pair loop in FP32 (distance_sphere with acos,
    angles_sphere), all pairs."""
    f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
    nA, nB = len(lens["x"]), len(src["x"])
    xA, yA, vA, wA = (f(lens[k]) for k in ("x", "y", "val", "w"))
    zA = f(lens.get("z")) if mode == SHEAR else None
    if mode == SHEAR:
        xB, yB, zB, e1, e2b, wB, mB = (f(src[k]) for k in ("x", "y", "z", "e1", "e2", "w", "m"))
    else:
        xB, yB, e1, e2b, wB = (f(src[k]) for k in ("x", "y", "kappa_E", "kappa_B", "w"))
        zB = mB = None
    out = {k: np.zeros(n_bin, np.float32) for k in ("g_t", "g_x", "weights")}
    out["n_pairs"] = np.zeros(n_bin, np.int64)
    rc = lib().orc_ref_sphere_f32(mode, nA, _ptr(xA), _ptr(yA), _ptr(zA), _ptr(vA), _ptr(wA), nB, _ptr(xB),
                                  _ptr(yB), _ptr(zB), _ptr(e1), _ptr(e2b), _ptr(wB), _ptr(mB), x_min, x_max,
                                  n_bin, spacing, p, num_threads, _ptr(out["g_t"]), _ptr(out["g_x"]),
                                  _ptr(out["weights"]), _ptr(out["n_pairs"]))
    if rc:
        raise RuntimeError("bad binning")
    return out


def normalise(s):
    """Reference normalisation (src/tpcf.f90:369-376) applied to FP64 sums."""
    with np.errstate(invalid="ignore", divide="ignore"):
        mean_theta = s["sum_dw"] / s["sum_w"]
        K = s["sum_K"]
        g_t = np.where(K > 0, s["sum_gt"] / np.where(K > 0, K, 1), 0.0)
        g_x = np.where(K > 0, s["sum_gx"] / np.where(K > 0, K, 1), 0.0)
    return {"mean_theta": mean_theta, "g_t": g_t, "g_x": g_x, "weights": s["sum_w"],
            "n_pairs": s["n_pairs"].astype(np.int64)}


# ----------------------------------------------------------------- kd-tree --
def kdtree_search(x, y, q, r, leafsize=10, brute_force=False, cap=None):
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    cap = cap or len(x)
    res = np.zeros(cap, np.int64)
    nf = C.c_long()
    rc = lib().orc_kdtree_search(len(x), x, y, q[0], q[1], r, leafsize, int(brute_force), res,
                                 cap, C.byref(nf))
    if rc:
        raise RuntimeError(f"kd-tree search failed with status {rc}")
    return res[:nf.value]


# ------------------------------------------------------------------ k-means --
def kmeans_ref_f32(x, y, w, k, equal_size=False, scaling=0.0, max_iter=1000, reassign_tol=0.0,
                   weight_tol=0.0):
    """partition_data restated in FP32 (src/kmeans.f90:12-263), fixed-grid start."""
    x, y, w = (np.ascontiguousarray(a, np.float32) for a in (x, y, w))
    lab = np.zeros(len(x), np.int32)
    cx = np.zeros(k, np.float32)
    cy = np.zeros(k, np.float32)
    it = C.c_int()
    rc = lib().orc_kmeans_ref_f32(len(x), x, y, w, k, int(equal_size), scaling, max_iter,
                                  reassign_tol, weight_tol, lab, cx, cy, C.byref(it))
    if rc:
        raise RuntimeError("partition_data failed")
    return lab, np.stack([cx, cy], 1), it.value


def kmeans_det(x, y, w, k, max_iter=1000, reassign_tol=0.0):
    """Deterministic Voronoi-mode k-means as the CUDA library defines it."""
    x, y, w = (np.ascontiguousarray(a, np.float32) for a in (x, y, w))
    lab = np.zeros(len(x), np.int32)
    cx = np.zeros(k, np.float32)
    cy = np.zeros(k, np.float32)
    it = C.c_int()
    if lib().orc_kmeans_det(len(x), x, y, w, k, max_iter, reassign_tol, lab, cx, cy, C.byref(it)):
        raise RuntimeError("kmeans_det failed")
    return lab, np.stack([cx, cy], 1), it.value


def fixed_scale(n, vmax):
    return lib().orc_fixed_scale(n, vmax)


def qsort_arg_f32(a, reverse=False):
    a = np.ascontiguousarray(a, np.float32)
    order = np.zeros(len(a), np.int64)
    lib().orc_qsort_arg_f32(a, len(a), order, int(reverse))
    return order


# --------------------------------------------------------------- bootstrap --
def philox4x32(ctr, key):
    """One Philox4x32-10 block (Salmon et al., SC'11)."""
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32(np.ascontiguousarray(ctr, np.uint32), np.ascontiguousarray(key, np.uint32), out)
    return out


def bootstrap_multiplicity(seed, n_boot, n_patch, n_draw):
    mult = np.zeros((n_boot, n_patch), np.int32)
    lib().orc_bootstrap_multiplicity(seed, n_boot, n_patch, n_draw, mult)
    return mult


def block_bootstrap(mult, St, Sx, SK, Sw):
    """Block bootstrap from patch sums (src/tpcf.f90:1166-1191) in FP64."""
    mult = np.ascontiguousarray(mult, np.int32)
    n_boot, n_patch = mult.shape
    n_bin = St.shape[1]
    gt = np.zeros((n_boot, n_bin))
    gx = np.zeros((n_boot, n_bin))
    W = np.zeros(n_boot)
    c = lambda a: np.ascontiguousarray(a, np.float64)
    lib().orc_block_bootstrap(n_boot, n_patch, n_bin, mult, c(St), c(Sx), c(SK), c(Sw), gt, gx, W)
    return gt, gx, W


def covariance(x):
    """covariance_matrix (src/utils.f90:745-764) in FP64; x is [n_samples][n_data]."""
    x = np.ascontiguousarray(x, np.float64)
    cov = np.zeros((x.shape[1], x.shape[1]))
    lib().orc_covariance(x.shape[0], x.shape[1], x, cov)
    return cov


# ------------------------------------------------------------ files, marks --
def marks_write(path, fields):
    """The binary marks stream of save_marks (src/input_formats.f90:528-560),
    restated with numpy: fields are dicts x, y, w, xi_E, xi_B, K ([n][n_bin])."""
    head = np.zeros(128, np.int64)
    head[0], head[1], head[127] = 1024, len(fields), 1024
    with open(path, "wb") as f:
        f.write(head.tobytes())
        for m in fields:
            n, nb = np.asarray(m["xi_E"]).shape
            f.write(np.array([n, nb], np.int64).tobytes())
            for k in ("x", "y", "w", "xi_E", "xi_B", "K"):
                f.write(np.ascontiguousarray(m[k], np.float32).tobytes())


def marks_read(path):
    """load_survey_marks (src/input_formats.f90:562-603) restated with numpy."""
    raw = open(path, "rb").read()
    h = np.frombuffer(raw[:1024], np.int64)
    assert h[0] == 1024 and h[127] == 1024
    off, out = 1024, []
    for _ in range(int(h[1])):
        n, nb = (int(v) for v in np.frombuffer(raw[off:off + 16], np.int64))
        off += 16
        m = {}
        for k in ("x", "y", "w"):
            m[k] = np.frombuffer(raw[off:off + 4 * n], np.float32).copy()
            off += 4 * n
        for k in ("xi_E", "xi_B", "K"):
            m[k] = np.frombuffer(raw[off:off + 4 * n * nb], np.float32).reshape(n, nb).copy()
            off += 4 * n * nb
        out.append(m)
    return out


def xi_from_marks(fields, vals, ws):
    """calculate_tpcf_from_marks (src/main.f90:1017-1139) in FP64 for one map:
    fields[i] dicts with w (marks weight), xi_E, xi_B, K; vals[i], ws[i] the
    lens values and weights.  Lenses with marks_w * w <= 0 (FP32 product, as
    the reference forms it) are removed."""
    res, E, B, K, W = [], 0.0, 0.0, 0.0, 0.0
    for m, v, w in zip(fields, vals, ws):
        mw = np.asarray(m["w"], np.float32) * np.asarray(w, np.float32)
        keep = mw > 0
        vw = (np.asarray(v, np.float64) * np.asarray(w, np.float64))[keep]
        e = (np.asarray(m["xi_E"], np.float64)[keep] * vw[:, None]).sum(0)
        b = (np.asarray(m["xi_B"], np.float64)[keep] * vw[:, None]).sum(0)
        k = (np.asarray(m["K"], np.float64)[keep] * np.asarray(w, np.float64)[keep][:, None]).sum(0)
        wsum = (np.asarray(m["w"], np.float64) * np.asarray(w, np.float64))[keep].sum()
        with np.errstate(invalid="ignore", divide="ignore"):
            res.append({"g_t": e / k, "g_x": b / k, "weights": wsum})
        E, B, K, W = E + e, B + b, K + k, W + wsum
    with np.errstate(invalid="ignore", divide="ignore"):
        return res, {"g_t": E / K, "g_x": B / K, "weights": W}


def marks_bootstrap(fields, mult, units=None, k_guard=True):
    """Resampled xi from per-lens marks (src/tpcf.f90:547-634, :844-939,
    :1194-1265) for given multiplicities [n_boot][n_units], FP64: the lens
    multiplicity is mult[unit(lens)] (the lens itself when units is None)."""
    E = np.concatenate([np.asarray(m["xi_E"], np.float64) for m in fields])
    B = np.concatenate([np.asarray(m["xi_B"], np.float64) for m in fields])
    K = np.concatenate([np.asarray(m["K"], np.float64) for m in fields])
    W = np.concatenate([np.asarray(m["w"], np.float64) for m in fields])
    mult = np.asarray(mult, np.float64)
    m = mult if units is None else mult[:, np.asarray(units)]
    e, b, k = m @ E, m @ B, m @ K
    with np.errstate(invalid="ignore", divide="ignore"):
        if k_guard:
            gt = np.where(k > 0, e / np.where(k > 0, k, 1), 0.0)
            gx = np.where(k > 0, b / np.where(k > 0, k, 1), 0.0)
        else:
            gt, gx = e / k, b / k
    return gt, gx, m @ W


def kmeans_equal(x, y, w, k, scaling=3.0, weight_tol=0.05, max_iter=1000, reassign_tol=0.01, random_init=True,
                 seed=0):
    """Equal-weight k-means restated serially (labels, centroids, iterations, max deviation)."""
    f = lambda a: np.ascontiguousarray(a, np.float32)
    x, y, w = f(x), f(y), f(w)
    n = len(x)
    lab = np.zeros(n, np.int32)
    cx = np.zeros(k, np.float32)
    cy = np.zeros(k, np.float32)
    it = C.c_int()
    dev = C.c_float()
    lib().orc_kmeans_equal_det(n, _ptr(x), _ptr(y), _ptr(w), k, max_iter, reassign_tol, scaling, weight_tol,
                               int(random_init), seed, _ptr(lab), _ptr(cx), _ptr(cy), C.byref(it), C.byref(dev))
    return lab, np.stack([cx, cy], 1), it.value, dev.value
