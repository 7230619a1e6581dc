"""File formats of the reference's driver and xi from precomputed marks.

Text catalogues (load_standard_shape_catalog, load_standard_kappa_map,
load_standard_lens_catalog, src/input_formats.f90:227-333), the per-bin result
table (src/main.f90:699-702), the binary marks stream (save_marks /
load_survey_marks, src/input_formats.f90:528-603) and
calculate_tpcf_from_marks (src/main.f90:1017-1139).  Parsing and writing are
native (libtpcf_b200, all host threads); the re-weighting of marks runs on the
GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import Context, KappaMap, LensCatalog, ShapeCatalog, _Arr, _check, _resolve_ctx
from ._lib import MarksFieldC, lib

__all__ = ["read_table", "load_standard_shape_catalog", "load_standard_kappa_map", "load_standard_lens_catalog",
           "write_result_table", "MarksField", "save_marks", "load_survey_marks", "calculate_tpcf_from_marks",
           "marks_bootstrap"]


def read_table(filename, ncols: int, keep_positive_col: int = -1, keep_nonnegative_col: int = -1,
               n_threads: int = 0) -> np.ndarray:
    """[ncols][n] float32 columns of a text table (tpcf_read_table)."""
    path = os.fsencode(filename)
    n = C.c_int64()
    _check(lib().tpcf_read_table(path, ncols, keep_positive_col, keep_nonnegative_col, n_threads, None, 0,
                                 C.byref(n)))
    cap = max(int(n.value), 1)
    cols = np.zeros((ncols, cap), np.float32)
    _check(lib().tpcf_read_table(path, ncols, keep_positive_col, keep_nonnegative_col, n_threads,
                                 cols.ctypes.data, cap, C.byref(n)))
    return np.ascontiguousarray(cols[:, :n.value])


def load_standard_shape_catalog(filename) -> ShapeCatalog:
    """Columns x y z e1 e2 w m; objects with w <= 0 dropped (input_formats.f90:227-258)."""
    x, y, z, e1, e2, w, m = read_table(filename, 7, keep_positive_col=5)
    return ShapeCatalog(x=x, y=y, e1=e1, e2=e2, w=w, z=z, m=m)


def load_standard_kappa_map(filename) -> KappaMap:
    """Columns x y kappa_E kappa_B w; pixels with w <= 0 dropped (:260-288)."""
    x, y, kE, kB, w = read_table(filename, 5, keep_positive_col=4)
    return KappaMap(x=x, y=y, kappa_E=kE, kappa_B=kB, w=w)


def load_standard_lens_catalog(filename, apply_masks: bool = True) -> LensCatalog:
    """Columns x y z val w; with apply_masks, w <= 0 and z < 0 dropped (:290-333)."""
    if apply_masks:
        x, y, z, val, w = read_table(filename, 5, keep_positive_col=4, keep_nonnegative_col=2)
    else:
        x, y, z, val, w = read_table(filename, 5)
    return LensCatalog(x=x, y=y, val=val, w=w, z=z)


def write_result_table(filename, result, spherical_coords: bool = False):
    """The driver's output table: theta, g_t, g_x, weights, n_pairs, mean_theta
    per bin (degrees when spherical_coords)."""
    f = lambda a: np.ascontiguousarray(a, np.float32)
    th, gt, gx, w, mt = (f(getattr(result, k)) for k in ("theta", "g_t", "g_x", "weights", "mean_theta"))
    npairs = np.ascontiguousarray(result.n_pairs, np.int64)
    _check(lib().tpcf_write_result_table(os.fsencode(filename), len(th), th.ctypes.data, gt.ctypes.data,
                                         gx.ctypes.data, w.ctypes.data, npairs.ctypes.data, mt.ctypes.data,
                                         int(bool(spherical_coords))))


@dataclass
class MarksField:
    """One field of a marks file: lens positions, marks weight, [n][n_bin] marks."""
    x: np.ndarray
    y: np.ndarray
    w: np.ndarray
    xi_E: np.ndarray
    xi_B: np.ndarray
    K: np.ndarray

    @property
    def n(self):
        return len(self.x)

    @property
    def n_bin(self):
        return self.xi_E.shape[1]

    @classmethod
    def from_results(cls, lenses: LensCatalog, res) -> "MarksField":
        """The marks of a tangential_shear_tpcf result (computed with val = w = 1)."""
        return cls(np.asarray(lenses.x), np.asarray(lenses.y), res.marks_weight, res.xi_E_marks, res.xi_B_marks,
                   res.K_marks)


def _host(a):
    return a.detach().cpu().numpy() if hasattr(a, "detach") else a


def _cfields(fields, host=False):
    """ctypes view of MarksField objects (numpy, or CUDA tensors unless host)."""
    keep, arr = [], (MarksFieldC * len(fields))()
    for i, m in enumerate(fields):
        vs = [(m.x, m.y, m.w, m.xi_E, m.xi_B, m.K)][0]
        if host:
            vs = [_host(v) for v in vs]
        a = [_Arr(v) for v in vs]
        keep += a
        nb = int(m.xi_E.shape[1]) if len(m.xi_E.shape) == 2 else 1
        arr[i] = MarksFieldC(int(len(m.x)), nb, *[v.ptr for v in a])
    return arr, keep


def save_marks(filename, fields: Sequence[MarksField]):
    """Binary marks stream of save_marks (src/input_formats.f90:528-560)."""
    arr, keep = _cfields(fields, host=True)
    _check(lib().tpcf_marks_save(os.fsencode(filename), len(fields), arr))


def load_survey_marks(filename):
    """load_survey_marks (src/input_formats.f90:562-603): list of MarksField."""
    path = os.fsencode(filename)
    nf = C.c_int32()
    n = np.zeros(20, np.int64)
    nb = np.zeros(20, np.int64)
    _check(lib().tpcf_marks_info(path, 20, C.byref(nf), n.ctypes.data, nb.ctypes.data))
    fields = [MarksField(np.zeros(n[i], np.float32), np.zeros(n[i], np.float32), np.zeros(n[i], np.float32),
                         np.zeros((n[i], nb[i]), np.float32), np.zeros((n[i], nb[i]), np.float32),
                         np.zeros((n[i], nb[i]), np.float32)) for i in range(nf.value)]
    arr, keep = _cfields(fields)
    _check(lib().tpcf_marks_load(path, nf.value, arr))
    return fields


def calculate_tpcf_from_marks(marks: Sequence[MarksField], val, w, lens_x=None, lens_y=None,
                              ctx: Context = None):
    """xi of foreground maps from precomputed marks (tpcf_xi_from_marks).

    ``val[i]``, ``w[i]``: the map values and weights of field i, shape [n_i]
    (one map) or [n_map][n_i].  Returns a dict with per-field ``g_t``, ``g_x``
    [n_map][n_field][n_bin], ``weights`` [n_map][n_field] and the stacked
    ``g_t_stacked``, ``g_x_stacked`` [n_map][n_bin], ``weights_stacked``
    [n_map] (FP64)."""
    ctx = _resolve_ctx(ctx)
    nf = len(marks)
    one = len(val[0].shape) == 1
    n_map = 1 if one else int(val[0].shape[0])
    V = [_Arr(v) for v in val]
    W = [_Arr(x) for x in w]
    for i, (v, x) in enumerate(zip(V, W)):
        if v.n != n_map * marks[i].n or x.n != n_map * marks[i].n:
            raise ValueError(f"field {i}: val and w must hold n_map x {marks[i].n} values")
    arr, keep = _cfields(marks)
    vp = (C.c_void_p * nf)(*[a.ptr for a in V])
    wp = (C.c_void_p * nf)(*[a.ptr for a in W])
    keep += V + W
    if lens_x is not None:
        LX = [_Arr(a) for a in lens_x]
        LY = [_Arr(a) for a in lens_y]
        keep += LX + LY
        lx = (C.c_void_p * nf)(*[a.ptr for a in LX])
        ly = (C.c_void_p * nf)(*[a.ptr for a in LY])
    else:
        lx = ly = None
    nb = marks[0].n_bin
    out = {"g_t": np.zeros((n_map, nf, nb)), "g_x": np.zeros((n_map, nf, nb)), "weights": np.zeros((n_map, nf)),
           "g_t_stacked": np.zeros((n_map, nb)), "g_x_stacked": np.zeros((n_map, nb)),
           "weights_stacked": np.zeros(n_map)}
    with np.errstate(invalid="ignore", divide="ignore"):
        _check(lib().tpcf_xi_from_marks(ctx.handle, nf, arr, n_map, vp, wp, lx, ly,
                                        *[out[k].ctypes.data for k in ("g_t", "g_x", "weights", "g_t_stacked",
                                                                       "g_x_stacked", "weights_stacked")]),
               ctx.handle)
    if one:
        out = {k: v[0] for k, v in out.items()}
    return out


def marks_bootstrap(marks: Sequence[MarksField], n_boot: int, seed: int = 0, supersampling_factor: float = 1.0,
                    units=None, n_units: int = 0, multiplicity=None, k_guard: bool = True, covariance: bool = True,
                    ctx: Context = None):
    """Point or block bootstrap from per-lens marks (tpcf_marks_bootstrap).

    ``units=None``: every lens of ``marks`` (all fields in order) is a unit --
    simple_bootstrap_foreground / survey_marked_point_bootstrap
    (src/tpcf.f90:547-634, :1194-1265).  ``units``: an int label per lens in
    [0, n_units) -- the resampling of pair_weighted_block_bootstrap (:844-939,
    with k_guard=False for its plain quotients).  Returns g_t, g_x
    [n_boot][n_bin], weights [n_boot] and the covariances."""
    ctx = _resolve_ctx(ctx)
    arr, keep = _cfields(marks)
    U = _Arr(units, np.int32)
    M = _Arr(multiplicity, np.int32)
    nb = marks[0].n_bin
    out = {"g_t": np.zeros((n_boot, nb)), "g_x": np.zeros((n_boot, nb)), "weights": np.zeros(n_boot)}
    if covariance:
        out["cov_g_t"] = np.zeros((nb, nb))
        out["cov_g_x"] = np.zeros((nb, nb))
    p = lambda k: out[k].ctypes.data if k in out else None
    with np.errstate(invalid="ignore", divide="ignore"):
        _check(lib().tpcf_marks_bootstrap(ctx.handle, len(marks), arr, U.ptr, int(n_units), M.ptr,
                                          int(seed) & 0xFFFFFFFFFFFFFFFF, int(n_boot), float(supersampling_factor),
                                          int(bool(k_guard)), p("g_t"), p("g_x"), p("weights"), p("cov_g_t"),
                                          p("cov_g_x")), ctx.handle)
    return out
