"""2pcf_b200 -- B200-native pair sums for shear-scalar and scalar-scalar
correlation functions (the hot path of tilmantroester/2pcf).

The Python names mirror the reference's Fortran interface:

    create_bins              src/utils.f90:139-230
    shear_2pcf, kappa_2pcf   src/tpcf.f90:134-188
    tangential_shear_tpcf    src/tpcf.f90:190-378
    scalar_kappa_tpcf        src/tpcf.f90:380-545

Every computation runs through libtpcf_b200.so (C ABI: include/tpcf_b200.h)
on the GPU; there is no CPU fallback.  The package directory name starts with
a digit, so import it with ``importlib.import_module("2pcf_b200")``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import Bins, KappaCat, LensCat, Opts, Result, ShearCat, Stats, TPCFError, lib

LIN_BINNING, LOG_BINNING, IHS_BINNING, SQRT_BINNING = 0, 1, 2, 3  # src/utils.f90:7
_SPACING = {"lin": 0, "log": 1, "ihs": 2, "sqrt": 3}

__all__ = [
    "Binning", "create_bins", "Context", "ShapeCatalog", "LensCatalog", "KappaMap",
    "LensingSurveyField", "Shear2pcfResults", "shear_2pcf", "kappa_2pcf",
    "tangential_shear_tpcf", "scalar_kappa_tpcf", "batch_shear_2pcf", "batch_kappa_2pcf", "partition_data",
    "partition_data_equal", "block_bootstrap", "TPCFError", "rotate_data_from_poles_and_meridian",
    "unit_vectors", "read_table", "load_standard_shape_catalog", "load_standard_kappa_map",
    "load_standard_lens_catalog", "write_result_table", "MarksField", "save_marks", "load_survey_marks",
    "calculate_tpcf_from_marks", "marks_bootstrap", "BatchPlan",
]


# --------------------------------------------------------------- arrays ------
def _is_torch(a):
    return type(a).__module__.startswith("torch")


class _Arr:
    """Holds a contiguous float32/int32 view of an input and its raw pointer."""

    def __init__(self, a, dtype=np.float32):
        self.keep = None
        self.n = 0
        if a is None:
            self.ptr = None
            return
        if _is_torch(a):
            import torch
            tdt = torch.float32 if dtype == np.float32 else torch.int32
            if a.is_cuda and a.dtype == tdt and a.is_contiguous():  # used in place
                self.keep, self.ptr, self.n = a, a.data_ptr(), a.numel()
                return
            if a.is_cuda:
                t = a.detach().to(tdt).contiguous()
                self.keep, self.ptr, self.n = t, t.data_ptr(), t.numel()
                return
            a = a.detach().cpu().numpy()
        arr = np.ascontiguousarray(a, dtype=dtype)
        self.keep, self.ptr, self.n = arr, arr.ctypes.data, arr.size


def _check(status, ctx=None):
    if status != _lib.TPCF_OK:
        msg = ""
        if ctx is not None:
            msg = (lib().tpcf_last_error(ctx) or b"").decode()
        raise TPCFError(status, msg)


# --------------------------------------------------------------- binning -----
@dataclass
class Binning:
    """type(binning) of src/utils.f90:18-24.  ``bin_edges`` are the canonical
    FP64 edges the kernels bin against; ``bin_centers`` are computed in FP32
    exactly as create_bins does."""
    x_min: float
    x_max: float
    n_bin: int
    spacing: int = LOG_BINNING
    ihs_theta: float = 1.0
    bin_edges: np.ndarray = field(default=None, repr=False)
    bin_edges_sq: np.ndarray = field(default=None, repr=False)
    bin_centers: np.ndarray = field(default=None, repr=False)

    def c_struct(self) -> Bins:
        return Bins(int(self.n_bin), int(self.spacing), float(self.x_min), float(self.x_max),
                    float(self.ihs_theta))

    @property
    def chord_edges_sq(self) -> np.ndarray:
        """Squared chords (2 sin(e/2))^2 of the edges (radians): the bin rule
        of the spherical kernels (tpcf_chord_edges)."""
        out = np.zeros(self.n_bin + 1)
        cb = self.c_struct()
        _check(lib().tpcf_chord_edges(C.byref(cb), out.ctypes.data))
        return out


def create_bins(x_min, x_max, n_bin, spacing=LOG_BINNING, p=1.0) -> Binning:
    """create_bins(x_min, x_max, n_bin, p, spacing) of src/utils.f90:139-230."""
    if isinstance(spacing, str):
        spacing = _SPACING[spacing]
    b = Binning(float(x_min), float(x_max), int(n_bin), int(spacing), float(p))
    cb = b.c_struct()
    e = np.zeros(n_bin + 1)
    e2 = np.zeros(n_bin + 1)
    _check(lib().tpcf_canonical_edges(C.byref(cb), e.ctypes.data, e2.ctypes.data))
    c = np.zeros(n_bin, np.float32)
    _check(lib().tpcf_bin_centers(C.byref(cb), c.ctypes.data))
    b.bin_edges, b.bin_edges_sq, b.bin_centers = e, e2, c
    return b


# --------------------------------------------------------------- context -----
class Context:
    """One device, one stream (tpcf_ctx).  ``use_kd_tree`` of the reference maps
    to ``use_grid`` (the device cell grid that replaces the kd-tree)."""

    def __init__(self, device: int = 0, use_grid: bool = True, cell_size: float = 0.0,
                 verbose: bool = False):
        self._h = C.c_void_p()
        o = Opts(int(use_grid), int(verbose), float(cell_size), 0, 0, 0, 0, 0, (C.c_int32 * 3)())
        _check(lib().tpcf_create(C.byref(self._h), int(device), C.byref(o)))
        self.device = device
        self.cell_size = float(cell_size)
        self.tile_shape = (0, 0)
        self.spherical = False

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().tpcf_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: Optional[int]):
        _check(lib().tpcf_set_stream(self._h, stream_ptr), self._h)

    def set_timing(self, enable: bool):
        _check(lib().tpcf_set_timing(self._h, int(enable)), self._h)

    def set_cell_size(self, cell_size: float):
        """Grid cell side for later calls (0 = theta_max/16)."""
        _check(lib().tpcf_set_cell_size(self._h, float(cell_size)), self._h)
        self.cell_size = float(cell_size)

    def set_tile_shape(self, group_size: int = 0, tile_chunks: int = 0):
        """Planar pair kernel tile shape for later calls: threads per block
        (32, 64, 128; every warp takes 32-lens work items of its own) and
        32-source sub-chunks per source tile (1, 2); 0 keeps the default.
        Changes speed only, never results."""
        _check(lib().tpcf_set_tile_shape(self._h, int(group_size), int(tile_chunks)), self._h)
        self.tile_shape = (int(group_size), int(tile_chunks))

    def set_spherical(self, on: bool):
        """Positions (longitude, latitude) and bins in radians for later calls."""
        _check(lib().tpcf_set_spherical(self._h, int(bool(on))), self._h)
        self.spherical = bool(on)

    def set_shard(self, index: int, count: int):
        """Compute only work items i % count == index (sums become partial)."""
        _check(lib().tpcf_set_shard(self._h, int(index), int(count)), self._h)

    def measure_fp32_peak(self) -> float:
        """Measured FP32 FMA throughput of this GPU in TFLOP/s."""
        v = C.c_double()
        _check(lib().tpcf_measure_fp32_peak(self._h, C.byref(v)), self._h)
        return v.value

    def measure_fp64_peak(self) -> float:
        """Measured FP64 FMA throughput of this GPU in TFLOP/s."""
        v = C.c_double()
        _check(lib().tpcf_measure_fp64_peak(self._h, C.byref(v)), self._h)
        return v.value

    def stats(self) -> dict:
        s = Stats()
        _check(lib().tpcf_last_stats(self._h, C.byref(s)), self._h)
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    @property
    def kernel_launches(self) -> int:
        return int(lib().tpcf_kernel_launches(self._h))


_default_ctx: dict = {}


def default_context(device: int = 0) -> Context:
    if device not in _default_ctx:
        _default_ctx[device] = Context(device)
    return _default_ctx[device]


# ------------------------------------------------------------- catalogues ----
@dataclass
class ShapeCatalog:  # shape_catalog, src/tpcf.f90:24-27
    x: object
    y: object
    e1: object
    e2: object
    w: object
    z: object = None
    m: object = None

    @property
    def n(self):
        return len(self.x)


@dataclass
class LensCatalog:  # lens_catalog, src/tpcf.f90:34-37
    x: object
    y: object
    val: object
    w: object
    z: object = None

    @property
    def n(self):
        return len(self.x)


@dataclass
class KappaMap:  # kappa_map, src/tpcf.f90:29-32
    x: object
    y: object
    kappa_E: object
    kappa_B: object
    w: object

    @property
    def n(self):
        return len(self.x)


@dataclass
class LensingSurveyField:  # lensing_survey_field, src/tpcf.f90:39-43
    lenses: LensCatalog
    shapes: Optional[ShapeCatalog] = None
    convergence: Optional[KappaMap] = None


@dataclass
class Shear2pcfResults:
    """shear_2pcf_results (src/tpcf.f90:17-22) plus the FP64 sums behind it."""
    n_bin: int
    theta: np.ndarray
    mean_theta: np.ndarray
    g_t: np.ndarray
    g_x: np.ndarray
    weights: np.ndarray
    n_pairs: np.ndarray
    sum_dw: np.ndarray
    sum_gt: np.ndarray
    sum_gx: np.ndarray
    sum_w: np.ndarray
    sum_K: np.ndarray
    xi_E_marks: Optional[np.ndarray] = None
    xi_B_marks: Optional[np.ndarray] = None
    K_marks: Optional[np.ndarray] = None
    w_marks: Optional[np.ndarray] = None
    marks_weight: Optional[np.ndarray] = None
    lens_sums: Optional[np.ndarray] = None
    patch_sums: Optional[np.ndarray] = None
    lens_raw: Optional[np.ndarray] = None


def _alloc_result(nb, nA, marks, lens_sums, n_patch, lens_raw=False):
    r = {k: np.zeros(nb) for k in ("sum_dw", "sum_gt", "sum_gx", "sum_w", "sum_K")}
    r["n_pairs"] = np.zeros(nb, np.int64)
    for k in ("theta", "mean_theta", "g_t", "g_x", "weights"):
        r[k] = np.zeros(nb, np.float32)
    if marks:
        for k in ("xi_E_marks", "xi_B_marks", "K_marks", "w_marks"):
            r[k] = np.zeros((nA, nb), np.float32)
        r["marks_weight"] = np.zeros(nA, np.float32)
    if lens_sums == "device":   # stays in device memory (a torch tensor on the current device)
        import torch
        r["lens_sums"] = torch.zeros((nA, 6, nb), dtype=torch.float64, device="cuda")
    elif lens_sums:
        r["lens_sums"] = np.zeros((nA, 6, nb))
    if n_patch and n_patch > 0:
        r["patch_sums"] = np.zeros((n_patch, 6, nb))
    if lens_raw:
        r["lens_raw"] = np.zeros((nA, 6, nb))
    ptr = lambda v: None if v is None else (v.data_ptr() if hasattr(v, "data_ptr") else v.ctypes.data)
    cres = Result(**{k: ptr(v) for k, v in r.items()})
    return r, cres


def _finish(r, nb):
    return Shear2pcfResults(n_bin=nb, **r)


def _resolve_ctx(ctx):
    return ctx if ctx is not None else default_context(0)


def _coords(ctx, spherical_coords):
    """spherical_coords of the reference's calls: x, y are longitude and
    latitude in radians, the bins angles in radians."""
    if bool(spherical_coords) != ctx.spherical:
        ctx.set_spherical(bool(spherical_coords))


def rotate_data_from_poles_and_meridian(x_A, y_A, r_max, verbose=False, x_B=None, y_B=None,
                                        ctx: Context = None):
    """rotate_data_from_poles_and_meridian (src/main.f90:953-1015), in place
    on float32 numpy arrays or CUDA tensors (radians).  Returns (rotated,
    (center_lambda, center_phi))."""
    ctx = _resolve_ctx(ctx)
    arrs = [_Arr(a) for a in (x_A, y_A, x_B, y_B)]
    for a, orig in zip(arrs, (x_A, y_A, x_B, y_B)):
        if orig is not None and not _is_torch(orig) and a.keep is not orig:
            raise ValueError("rotation is in place: pass contiguous float32 arrays")
    rot = C.c_int32()
    center = np.zeros(2, np.float32)
    nB = arrs[2].n if x_B is not None else 0
    _check(lib().tpcf_rotate_from_poles(ctx.handle, arrs[0].ptr, arrs[1].ptr, arrs[0].n, arrs[2].ptr,
                                        arrs[3].ptr, nB, float(r_max), C.byref(rot), center.ctypes.data),
           ctx.handle)
    if verbose and rot.value:
        print(f"Rotated field centre RA {np.degrees(center[0]):.2f} Dec {np.degrees(center[1]):.2f}")
    return bool(rot.value), (float(center[0]), float(center[1]))


def unit_vectors(lam, phi, ctx: Context = None):
    """(hi, lo) [n][3] FP32 parts of the unit vectors the spherical kernels use
    (tpcf_unit_vectors)."""
    ctx = _resolve_ctx(ctx)
    a, b = _Arr(lam), _Arr(phi)
    hi = np.zeros((a.n, 3), np.float32)
    lo = np.zeros((a.n, 3), np.float32)
    _check(lib().tpcf_unit_vectors(ctx.handle, a.ptr, b.ptr, a.n, hi.ctypes.data, lo.ctypes.data), ctx.handle)
    return hi, lo


# -------------------------------------------------------------- pair sums ----
def tangential_shear_tpcf(x_A, y_A, z_A, val_A, weight_A, x_B, y_B, z_B, e1_B, e2_B, weight_B, m_B,
                          bins: Binning, spherical_coords=False, num_threads=None,
                          use_kd_tree=True, verbose=False, calculate_marks=True,
                          patch_A=None, n_patch=0, lens_sums=False, lens_raw=False, ctx: Context = None):
    """tangential_shear_tpcf (src/tpcf.f90:190-378) on the GPU.

    Returns a Shear2pcfResults: avg_theta is ``mean_theta``; the marks arrays
    are [n_A][n_bin] (the memory layout of the reference's (n_bin, n_A)).
    ``num_threads`` is accepted and ignored; ``use_kd_tree`` selects the cell
    grid (True) or the all-pairs scan (False) when ``ctx`` is not given."""
    if ctx is None:
        ctx = default_context(0) if use_kd_tree else Context(0, use_grid=False, verbose=verbose)
    _coords(ctx, spherical_coords)
    A = [_Arr(a) for a in (x_A, y_A, z_A, val_A, weight_A)]
    B = [_Arr(a) for a in (x_B, y_B, z_B, e1_B, e2_B, weight_B, m_B)]
    P = _Arr(patch_A, np.int32)
    nA, nB = A[0].n, B[0].n
    nb = bins.n_bin
    r, cres = _alloc_result(nb, nA, calculate_marks, lens_sums, n_patch if patch_A is not None else 0,
                            lens_raw)
    cb = bins.c_struct()
    st = lib().tpcf_shear_scalar(ctx.handle, *[a.ptr for a in A], nA, *[b.ptr for b in B], nB,
                                 C.byref(cb), P.ptr, int(n_patch), C.byref(cres))
    _check(st, ctx.handle)
    return _finish(r, nb)


def scalar_kappa_tpcf(x_A, y_A, val_A, w_A, x_B, y_B, kappa_E, kappa_B, w_B, bins: Binning,
                      spherical_coords=False, num_threads=None, use_kd_tree=True, verbose=False,
                      calculate_marks=True, patch_A=None, n_patch=0, lens_sums=False,
                      ctx: Context = None):
    """scalar_kappa_tpcf (src/tpcf.f90:380-545) on the GPU."""
    if ctx is None:
        ctx = default_context(0) if use_kd_tree else Context(0, use_grid=False, verbose=verbose)
    _coords(ctx, spherical_coords)
    A = [_Arr(a) for a in (x_A, y_A, val_A, w_A)]
    B = [_Arr(a) for a in (x_B, y_B, kappa_E, kappa_B, w_B)]
    P = _Arr(patch_A, np.int32)
    nA, nB = A[0].n, B[0].n
    nb = bins.n_bin
    r, cres = _alloc_result(nb, nA, calculate_marks, lens_sums, n_patch if patch_A is not None else 0)
    cb = bins.c_struct()
    st = lib().tpcf_scalar_scalar(ctx.handle, *[a.ptr for a in A], nA, *[b.ptr for b in B], nB,
                                  C.byref(cb), P.ptr, int(n_patch), C.byref(cres))
    _check(st, ctx.handle)
    return _finish(r, nb)


def shear_2pcf(field: LensingSurveyField, bins: Binning, spherical_coords=False, num_threads=None,
               use_kd_tree=True, verbose=False, **kw):
    """shear_2pcf (src/tpcf.f90:134-160)."""
    L, S = field.lenses, field.shapes
    return tangential_shear_tpcf(L.x, L.y, L.z, L.val, L.w, S.x, S.y, S.z, S.e1, S.e2, S.w, S.m,
                                 bins, spherical_coords, num_threads, use_kd_tree, verbose, **kw)


def kappa_2pcf(field: LensingSurveyField, bins: Binning, spherical_coords=False, num_threads=None,
               use_kd_tree=True, verbose=False, **kw):
    """kappa_2pcf (src/tpcf.f90:162-188)."""
    L, K = field.lenses, field.convergence
    return scalar_kappa_tpcf(L.x, L.y, L.val, L.w, K.x, K.y, K.kappa_E, K.kappa_B, K.w, bins,
                             spherical_coords, num_threads, use_kd_tree, verbose, **kw)


def batch_shear_2pcf(lenses: Sequence[LensCatalog], shapes: Sequence[ShapeCatalog],
                     tasks: Sequence[tuple], bins: Binning, lens_patches=None, n_patch=0,
                     marks=False, lens_sums=False, spherical_coords=False, ctx: Context = None):
    """All (lens catalogue, shape catalogue) tasks in one persistent launch
    (tpcf_batch_shear_scalar).  ``lens_patches[i]`` labels lens catalogue i.
    ``lens_sums`` = True gives per-lens FP64 rows [nA][6][n_bin] as numpy
    arrays, "device" as torch tensors left in device memory."""
    ctx = _resolve_ctx(ctx)
    _coords(ctx, spherical_coords)
    keep = []
    lc = (LensCat * len(lenses))()
    for i, L in enumerate(lenses):
        arrs = [_Arr(a) for a in (L.x, L.y, L.z, L.val, L.w)]
        p = _Arr(None if lens_patches is None else lens_patches[i], np.int32)
        keep += arrs + [p]
        lc[i] = LensCat(arrs[0].n, *[a.ptr for a in arrs], p.ptr)
    sc = (ShearCat * len(shapes))()
    for i, S in enumerate(shapes):
        arrs = [_Arr(a) for a in (S.x, S.y, S.z, S.e1, S.e2, S.w, S.m)]
        keep += arrs
        sc[i] = ShearCat(arrs[0].n, *[a.ptr for a in arrs])
    tl = np.ascontiguousarray([t[0] for t in tasks], np.int32)
    ts = np.ascontiguousarray([t[1] for t in tasks], np.int32)
    nb = bins.n_bin
    outs = (Result * len(tasks))()
    pyouts = []
    for t in range(len(tasks)):
        nA = lenses[tasks[t][0]].n
        r, cres = _alloc_result(nb, nA, marks, lens_sums, n_patch if lens_patches is not None else 0)
        outs[t] = cres
        pyouts.append(r)
    cb = bins.c_struct()
    st = lib().tpcf_batch_shear_scalar(ctx.handle, len(lenses), lc, len(shapes), sc, len(tasks),
                                       tl.ctypes.data, ts.ctypes.data, C.byref(cb),
                                       int(n_patch) if lens_patches is not None else 0, outs)
    _check(st, ctx.handle)
    return [_finish(r, nb) for r in pyouts]


class BatchPlan:
    """A prepared batch_shear_2pcf call (tpcf_plan_shear_scalar): the grids,
    lens groups and sorted work items are built once; ``launch()`` enqueues
    only the persistent pair kernel and the per-patch reductions on the plan's
    stream (no host synchronisation or allocation, so it can be recorded into
    a CUDA graph, see ``capture``), ``results()`` waits and returns the same
    Shear2pcfResults list as batch_shear_2pcf (identical sums).  Device
    inputs are used in place and are kept referenced by the plan."""

    def __init__(self, lenses, shapes, tasks, bins, lens_patches=None, n_patch=0, lens_sums=False,
                 ctx: Context = None, stream=None):
        ctx = _resolve_ctx(ctx)
        self._keep = []
        lc = (LensCat * len(lenses))()
        for i, L in enumerate(lenses):
            arrs = [_Arr(a) for a in (L.x, L.y, L.z, L.val, L.w)]
            p = _Arr(None if lens_patches is None else lens_patches[i], np.int32)
            self._keep += arrs + [p]
            lc[i] = LensCat(arrs[0].n, *[a.ptr for a in arrs], p.ptr)
        sc = (ShearCat * len(shapes))()
        for i, S in enumerate(shapes):
            arrs = [_Arr(a) for a in (S.x, S.y, S.z, S.e1, S.e2, S.w, S.m)]
            self._keep += arrs
            sc[i] = ShearCat(arrs[0].n, *[a.ptr for a in arrs])
        tl = np.ascontiguousarray([t[0] for t in tasks], np.int32)
        ts = np.ascontiguousarray([t[1] for t in tasks], np.int32)
        self.n_bin = bins.n_bin
        self._n_lens = [lenses[t[0]].n for t in tasks]
        self._lens_sums = lens_sums
        self._n_patch = int(n_patch) if lens_patches is not None else 0
        shape = (Result * len(tasks))()
        for t in range(len(tasks)):
            _, shape[t] = _alloc_result(self.n_bin, 1, False, bool(lens_sums), 0)
        cb = bins.c_struct()
        h = C.c_void_p()
        st = lib().tpcf_plan_shear_scalar(ctx.handle, len(lenses), lc, len(shapes), sc, len(tasks),
                                          tl.ctypes.data, ts.ctypes.data, C.byref(cb), self._n_patch, shape,
                                          C.byref(h))
        _check(st, ctx.handle)
        self.handle = h
        self.n_task = len(tasks)
        if stream is not None:
            self.set_stream(stream)

    def _err(self, st):
        if st != 0:
            raise TPCFError(st, lib().tpcf_plan_last_error(self.handle).decode())

    def set_stream(self, stream):
        """Launch on this CUDA stream (a torch.cuda.Stream or a raw handle)."""
        raw = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        self._err(lib().tpcf_plan_set_stream(self.handle, C.c_void_p(raw)))

    def launch(self):
        self._err(lib().tpcf_plan_launch(self.handle))

    def capture(self):
        """Records launch() into a torch.cuda.CUDAGraph on the current torch
        stream (the plan launches on it) and returns the graph; graph.replay()
        then re-runs the pair kernel and the reductions."""
        import torch
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.set_stream(s)
            self.launch()  # warm-up outside the graph
            with torch.cuda.graph(g, stream=s):
                self.launch()
        torch.cuda.current_stream().wait_stream(s)
        self.set_stream(torch.cuda.current_stream())
        return g

    def results(self):
        nb = self.n_bin
        outs = (Result * self.n_task)()
        pyouts = []
        for t in range(self.n_task):
            r, cres = _alloc_result(nb, self._n_lens[t], False, self._lens_sums, self._n_patch)
            outs[t] = cres
            pyouts.append(r)
        self._err(lib().tpcf_plan_results(self.handle, outs))
        return [_finish(r, nb) for r in pyouts]

    def close(self):
        if getattr(self, "handle", None):
            lib().tpcf_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_kappa_2pcf(lenses: Sequence[LensCatalog], kappas: Sequence[KappaMap], tasks: Sequence[tuple],
                     bins: Binning, lens_patches=None, n_patch=0, marks=False, lens_sums=False,
                     spherical_coords=False, ctx: Context = None):
    """All (scalar catalogue, kappa map) tasks of the scalar-scalar estimator
    in one persistent launch (tpcf_batch_scalar_scalar)."""
    ctx = _resolve_ctx(ctx)
    _coords(ctx, spherical_coords)
    keep = []
    lc = (LensCat * len(lenses))()
    for i, L in enumerate(lenses):
        arrs = [_Arr(a) for a in (L.x, L.y, None, L.val, L.w)]
        p = _Arr(None if lens_patches is None else lens_patches[i], np.int32)
        keep += arrs + [p]
        lc[i] = LensCat(arrs[0].n, *[a.ptr for a in arrs], p.ptr)
    kc = (KappaCat * len(kappas))()
    for i, K in enumerate(kappas):
        arrs = [_Arr(a) for a in (K.x, K.y, K.kappa_E, K.kappa_B, K.w)]
        keep += arrs
        kc[i] = KappaCat(arrs[0].n, *[a.ptr for a in arrs])
    tl = np.ascontiguousarray([t[0] for t in tasks], np.int32)
    tk = np.ascontiguousarray([t[1] for t in tasks], np.int32)
    nb = bins.n_bin
    outs = (Result * len(tasks))()
    pyouts = []
    for t in range(len(tasks)):
        r, cres = _alloc_result(nb, lenses[tasks[t][0]].n, marks, lens_sums,
                                n_patch if lens_patches is not None else 0)
        outs[t] = cres
        pyouts.append(r)
    cb = bins.c_struct()
    _check(lib().tpcf_batch_scalar_scalar(ctx.handle, len(lenses), lc, len(kappas), kc, len(tasks), tl.ctypes.data,
                                          tk.ctypes.data, C.byref(cb),
                                          int(n_patch) if lens_patches is not None else 0, outs), ctx.handle)
    return [_finish(r, nb) for r in pyouts]


# ------------------------------------------------------ patches and errors ---
def partition_data(x, y, weights, k, iterations=1000, reassignment_tol=0.0, ctx: Context = None):
    """partition_data (src/kmeans.f90:12-263) for Voronoi blocks on the GPU.

    Returns (labels [n] 0-based, centroids [k][2], iterations run).  Labels are
    deterministic (fixed-point centroid sums)."""
    ctx = _resolve_ctx(ctx)
    X, Y, W = _Arr(x), _Arr(y), _Arr(weights)
    n = X.n
    lab = np.zeros(n, np.int32)
    cen = np.zeros((k, 2), np.float32)
    it = C.c_int32()
    _check(lib().tpcf_kmeans(ctx.handle, X.ptr, Y.ptr, W.ptr, n, int(k), int(iterations),
                             float(reassignment_tol), lab.ctypes.data, cen.ctypes.data, C.byref(it)),
           ctx.handle)
    return lab, cen, it.value


def partition_data_equal(x, y, weights, k, weight_equalizer_scaling=3.0, weight_tol=0.05, iterations=1000,
                         reassignment_tol=0.01, random_init=True, seed=0, ctx: Context = None):
    """partition_data with equal_size (src/kmeans.f90:12-262) on the GPU: the
    weight-penalised assignment and the post-processing rebalance that move
    boundary points out of overweight clusters.  Defaults are those of
    pair_weighted_block_bootstrap (src/tpcf.f90:892-895).  Returns (labels,
    centroids, iterations, max weight deviation (max W - min W) / mean W)."""
    ctx = _resolve_ctx(ctx)
    X, Y, W = _Arr(x), _Arr(y), _Arr(weights)
    n = X.n
    lab = np.zeros(n, np.int32)
    cen = np.zeros((k, 2), np.float32)
    it = C.c_int32()
    dev = C.c_float()
    _check(lib().tpcf_kmeans_equal(ctx.handle, X.ptr, Y.ptr, W.ptr, n, int(k), int(iterations),
                                   float(reassignment_tol), float(weight_equalizer_scaling), float(weight_tol),
                                   int(bool(random_init)), int(seed) & 0xFFFFFFFFFFFFFFFF, lab.ctypes.data,
                                   cen.ctypes.data, C.byref(it), C.byref(dev)), ctx.handle)
    return lab, cen, it.value, dev.value


def block_bootstrap(patch_sums, n_boot, seed=0, supersampling_factor=1.0, multiplicity=None,
                    covariance=True, ctx: Context = None):
    """Block bootstrap over lens patches for one or many tasks
    (survey_marked_point_block_bootstrap's resampling, src/tpcf.f90:1166-1191).

    ``patch_sums``: [n_patch][6][n_bin] (one task) or [n_task][n_patch][6][n_bin]
    as returned in Shear2pcfResults.patch_sums.  Returns a dict with g_t, g_x
    [n_boot][n_task][n_bin], weights [n_boot][n_task], multiplicity
    [n_boot][n_patch] and, if asked, cov_g_t / cov_g_x over the joint vector."""
    ctx = _resolve_ctx(ctx)
    ps = np.ascontiguousarray(patch_sums, np.float64)
    if ps.ndim == 3:
        ps = ps[None]
    n_task, n_patch, six, nb = ps.shape
    assert six == 6
    D = n_task * nb
    gt = np.zeros((n_boot, n_task, nb))
    gx = np.zeros((n_boot, n_task, nb))
    W = np.zeros((n_boot, n_task))
    mult = np.zeros((n_boot, n_patch), np.int32)
    cgt = np.zeros((D, D)) if covariance else None
    cgx = np.zeros((D, D)) if covariance else None
    M = None if multiplicity is None else np.ascontiguousarray(multiplicity, np.int32)
    p = lambda a: None if a is None else a.ctypes.data
    _check(lib().tpcf_bootstrap(ctx.handle, ps.ctypes.data, n_task, n_patch, nb, p(M), int(seed), int(n_boot),
                                float(supersampling_factor), gt.ctypes.data, gx.ctypes.data, W.ctypes.data,
                                p(cgt), p(cgx), mult.ctypes.data), ctx.handle)
    out = dict(g_t=gt, g_x=gx, weights=W, multiplicity=M if M is not None else mult)
    if covariance:
        out.update(cov_g_t=cgt, cov_g_x=cgx)
    return out



# ---------------------------------------------------------------- gradients --
def tangential_shear_adjoint(x_A, y_A, z_A, val_A, weight_A, x_B, y_B, z_B, e1_B, e2_B, weight_B, m_B,
                             bins: Binning, forward: Shear2pcfResults, dL_dg_t, dL_dg_x=None,
                             ctx: Context = None):
    """Gradient of L with dL/dg_t, dL/dg_x given per bin, through
    tpcf_shear_scalar_adjoint.  ``forward`` is the Shear2pcfResults of the same
    inputs computed with lens_raw=True.  Returns a dict of gradients w.r.t.
    val_A, w_A, e1_B, e2_B, w_B, m_B (float32 arrays)."""
    ctx = _resolve_ctx(ctx)
    _coords(ctx, False)
    A = [_Arr(a) for a in (x_A, y_A, z_A, val_A, weight_A)]
    B = [_Arr(a) for a in (x_B, y_B, z_B, e1_B, e2_B, weight_B, m_B)]
    nA, nB = A[0].n, B[0].n
    if forward.lens_raw is None:
        raise ValueError("forward must be computed with lens_raw=True")
    f64 = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
    lt, lx = f64(dL_dg_t), f64(dL_dg_x)
    raw = f64(forward.lens_raw)
    g = {k: np.zeros(nA, np.float32) for k in ("val_A", "w_A")}
    g.update({k: np.zeros(nB, np.float32) for k in ("e1_B", "e2_B", "w_B", "m_B")})
    cb = bins.c_struct()
    p = lambda a: None if a is None else a.ctypes.data
    st = lib().tpcf_shear_scalar_adjoint(
        ctx.handle, *[a.ptr for a in A], nA, *[b.ptr for b in B], nB, C.byref(cb),
        p(f64(forward.sum_gt)), p(f64(forward.sum_gx)), p(f64(forward.sum_K)), p(raw), p(lt), p(lx),
        *[g[k].ctypes.data for k in ("val_A", "w_A", "e1_B", "e2_B", "w_B", "m_B")])
    _check(st, ctx.handle)
    return g


from .files import (calculate_tpcf_from_marks, load_standard_kappa_map, load_standard_lens_catalog,  # noqa: E402
                    load_standard_shape_catalog, load_survey_marks, read_table, save_marks, write_result_table,
                    MarksField, marks_bootstrap)
