"""torch.autograd wrapper of the shear-scalar correlation function.

``xi_shear(val_A, w_A, e1_B, e2_B, w_B, geometry, bins)`` returns (xi_t, xi_x)
per bin as FP64 CUDA tensors and is differentiable w.r.t. the five per-object
inputs.  Forward: tpcf_shear_scalar with the raw per-lens sums kept on the
device; backward: tpcf_shear_scalar_adjoint (lens gradients from those sums,
source gradients from one pass over all pairs).  Positions, redshifts and m
(``geometry``) are constants.  Used for gradient tests and field-level
inference; everything runs on the GPU through the C ABI.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import Binning, Context, _check, default_context
from ._lib import Result, lib


def _f32(t):
    return t.detach().to(torch.float32).contiguous()


def _p(t):
    return None if t is None else t.data_ptr()


class ShearXi(torch.autograd.Function):
    @staticmethod
    def forward(actx, val_A, w_A, e1_B, e2_B, w_B, geometry, bins: Binning, tctx: Context):
        dev = val_A.device
        nb = bins.n_bin
        g = {k: _f32(v) for k, v in geometry.items()}
        ins = [_f32(t) for t in (val_A, w_A, e1_B, e2_B, w_B)]
        nA, nB = ins[0].numel(), ins[2].numel()
        f64 = dict(dtype=torch.float64, device=dev)
        sums = torch.zeros(5, nb, **f64)
        npairs = torch.zeros(nb, dtype=torch.int64, device=dev)
        raw = torch.zeros(nA, 6, nb, **f64)
        res = Result(sum_dw=_p(sums[0]), sum_gt=_p(sums[1]), sum_gx=_p(sums[2]), sum_w=_p(sums[3]),
                     sum_K=_p(sums[4]), n_pairs=_p(npairs), lens_raw=_p(raw))
        cb = bins.c_struct()
        tctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        st = lib().tpcf_shear_scalar(tctx.handle, _p(g["x_A"]), _p(g["y_A"]), _p(g.get("z_A")), _p(ins[0]),
                                     _p(ins[1]), nA, _p(g["x_B"]), _p(g["y_B"]), _p(g.get("z_B")), _p(ins[2]),
                                     _p(ins[3]), _p(ins[4]), _p(g.get("m_B")), nB, C.byref(cb), None, 0,
                                     C.byref(res))
        _check(st, tctx.handle)
        K = sums[4]
        pos = K > 0
        xi_t = torch.where(pos, sums[1] / torch.where(pos, K, 1.0), torch.zeros_like(K))
        xi_x = torch.where(pos, sums[2] / torch.where(pos, K, 1.0), torch.zeros_like(K))
        actx.save_for_backward(*ins, sums, raw)
        actx.geometry, actx.bins, actx.tctx, actx.npairs = g, bins, tctx, npairs
        actx.mark_non_differentiable(npairs)
        return xi_t, xi_x

    @staticmethod
    def backward(actx, d_xi_t, d_xi_x):
        val_A, w_A, e1_B, e2_B, w_B, sums, raw = actx.saved_tensors
        g, bins, tctx = actx.geometry, actx.bins, actx.tctx
        nA, nB = val_A.numel(), e1_B.numel()
        dev = val_A.device
        lt = (d_xi_t if d_xi_t is not None else torch.zeros(bins.n_bin, device=dev)).to(torch.float64).contiguous()
        lx = None if d_xi_x is None else d_xi_x.to(torch.float64).contiguous()
        outs = [torch.zeros(n, dtype=torch.float32, device=dev) for n in (nA, nA, nB, nB, nB)]
        cb = bins.c_struct()
        tctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        st = lib().tpcf_shear_scalar_adjoint(
            tctx.handle, _p(g["x_A"]), _p(g["y_A"]), _p(g.get("z_A")), _p(val_A), _p(w_A), nA, _p(g["x_B"]),
            _p(g["y_B"]), _p(g.get("z_B")), _p(e1_B), _p(e2_B), _p(w_B), _p(g.get("m_B")), nB, C.byref(cb),
            _p(sums[1]), _p(sums[2]), _p(sums[4]), _p(raw), _p(lt), _p(lx), *[_p(o) for o in outs], None)
        _check(st, tctx.handle)
        return (*outs, None, None, None)


def xi_shear(val_A, w_A, e1_B, e2_B, w_B, geometry: dict, bins: Binning, ctx: Context = None):
    """Differentiable (xi_t, xi_x) of the shear-scalar estimator.  ``geometry``
    holds x_A, y_A, x_B, y_B and optionally z_A, z_B, m_B as CUDA tensors."""
    ctx = ctx if ctx is not None else default_context(val_A.device.index or 0)
    if ctx.spherical:
        ctx.set_spherical(False)
    return ShearXi.apply(val_A, w_A, e1_B, e2_B, w_B, geometry, bins, ctx)


class ShearXiBatch(torch.autograd.Function):
    """All tasks of a tomography in one forward launch (tpcf_batch_shear_scalar
    keeping every task's raw per-lens sums on the device) and one backward
    launch (tpcf_batch_shear_scalar_adjoint); gradients of a catalogue sum over
    the tasks that use it."""

    @staticmethod
    def forward(actx, tasks, geo_L, geo_S, bins, tctx, *leaves):
        from . import _lib as L_
        n_L, n_S = len(geo_L), len(geo_S)
        vals, wAs = leaves[:n_L], leaves[n_L:2 * n_L]
        e1s, e2s, wBs = leaves[2 * n_L:2 * n_L + n_S], leaves[2 * n_L + n_S:2 * n_L + 2 * n_S], \
            leaves[2 * n_L + 2 * n_S:]
        dev = vals[0].device
        nb = bins.n_bin
        f64 = dict(dtype=torch.float64, device=dev)
        opt = lambda t: None if t is None else _f32(t)
        lv = [(_f32(g["x"]), _f32(g["y"]), opt(g.get("z")), _f32(v), _f32(w)) for g, v, w in zip(geo_L, vals, wAs)]
        sv = [(_f32(g["x"]), _f32(g["y"]), opt(g.get("z")), _f32(a), _f32(b), _f32(w), opt(g.get("m")))
              for g, a, b, w in zip(geo_S, e1s, e2s, wBs)]
        lc = (L_.LensCat * n_L)(*[L_.LensCat(t[0].numel(), *[_p(a) for a in t], None) for t in lv])
        sc = (L_.ShearCat * n_S)(*[L_.ShearCat(t[0].numel(), *[_p(a) for a in t]) for t in sv])
        nT = len(tasks)
        sums = [torch.zeros(5, nb, **f64) for _ in range(nT)]
        npairs = [torch.zeros(nb, dtype=torch.int64, device=dev) for _ in range(nT)]
        raws = [torch.zeros(lv[li][0].numel(), 6, nb, **f64) for li, _ in tasks]
        outs = (Result * nT)()
        for t in range(nT):
            s = sums[t]
            outs[t] = Result(sum_dw=_p(s[0]), sum_gt=_p(s[1]), sum_gx=_p(s[2]), sum_w=_p(s[3]), sum_K=_p(s[4]),
                             n_pairs=_p(npairs[t]), lens_raw=_p(raws[t]))
        import numpy as np
        tl = np.ascontiguousarray([a for a, _ in tasks], np.int32)
        ts = np.ascontiguousarray([b for _, b in tasks], np.int32)
        cb = bins.c_struct()
        tctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        _check(lib().tpcf_batch_shear_scalar(tctx.handle, n_L, lc, n_S, sc, nT, tl.ctypes.data, ts.ctypes.data,
                                             C.byref(cb), 0, outs), tctx.handle)
        S = torch.stack(sums)                       # [n_task][5][nb]
        K = S[:, 4]
        pos = K > 0
        xi_t = torch.where(pos, S[:, 1] / torch.where(pos, K, 1.0), torch.zeros_like(K))
        xi_x = torch.where(pos, S[:, 2] / torch.where(pos, K, 1.0), torch.zeros_like(K))
        actx.save_for_backward(S, *raws)
        actx.lv, actx.sv, actx.tasks, actx.bins, actx.tctx = lv, sv, tasks, bins, tctx
        actx.n_L, actx.n_S = n_L, n_S
        return xi_t, xi_x

    @staticmethod
    def backward(actx, d_xi_t, d_xi_x):
        S, *raws = actx.saved_tensors
        lv, sv, tasks, bins, tctx = actx.lv, actx.sv, actx.tasks, actx.bins, actx.tctx
        dev = S.device
        g_val = [torch.zeros_like(t[3]) for t in lv]
        g_wA = [torch.zeros_like(t[4]) for t in lv]
        g_e1 = [torch.zeros_like(t[3]) for t in sv]
        g_e2 = [torch.zeros_like(t[4]) for t in sv]
        g_wB = [torch.zeros_like(t[5]) for t in sv]
        cb = bins.c_struct()
        tctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        from . import _lib as L_
        nT = len(tasks)
        lts = [(d_xi_t[t] if d_xi_t is not None else torch.zeros(bins.n_bin, device=dev)).to(torch.float64)
               .contiguous() for t in range(nT)]
        lxs = [None if d_xi_x is None else d_xi_x[t].to(torch.float64).contiguous() for t in range(nT)]
        ta = (L_.AdjointTask * nT)(*[L_.AdjointTask(_p(S[t, 1]), _p(S[t, 2]), _p(S[t, 4]), _p(raws[t]), _p(lts[t]),
                                                    _p(lxs[t])) for t in range(nT)])
        lc = (L_.LensCat * len(lv))(*[L_.LensCat(t[0].numel(), *[_p(a) for a in t], None) for t in lv])
        sc = (L_.ShearCat * len(sv))(*[L_.ShearCat(t[0].numel(), *[_p(a) for a in t]) for t in sv])
        lg = (L_.LensGrad * len(lv))(*[L_.LensGrad(_p(a), _p(b)) for a, b in zip(g_val, g_wA)])
        sg = (L_.ShearGrad * len(sv))(*[L_.ShearGrad(_p(a), _p(b), _p(c), None) for a, b, c in zip(g_e1, g_e2, g_wB)])
        import numpy as np
        tl = np.ascontiguousarray([a for a, _ in tasks], np.int32)
        ts = np.ascontiguousarray([b for _, b in tasks], np.int32)
        # every task's gradient in one launch; a catalogue used by several tasks gets their sum
        _check(lib().tpcf_batch_shear_scalar_adjoint(tctx.handle, len(lv), lc, lg, len(sv), sc, sg, nT,
                                                     tl.ctypes.data, ts.ctypes.data, C.byref(cb), ta), tctx.handle)
        return (None, None, None, None, None, *g_val, *g_wA, *g_e1, *g_e2, *g_wB)


def xi_shear_batch(tasks, lens_geometry, shape_geometry, val_A, w_A, e1_B, e2_B, w_B, bins: Binning,
                   ctx: Context = None):
    """Differentiable (xi_t, xi_x) [n_task][n_bin] of every (lens catalogue,
    shape catalogue) task in one forward launch.  ``lens_geometry[i]`` holds
    x, y, z of lens catalogue i and ``shape_geometry[j]`` x, y, z, m of shape
    catalogue j (CUDA tensors); ``val_A``, ``w_A`` (per lens catalogue) and
    ``e1_B``, ``e2_B``, ``w_B`` (per shape catalogue) are lists of CUDA
    tensors that may require gradients."""
    ctx = ctx if ctx is not None else default_context(val_A[0].device.index or 0)
    if ctx.spherical:
        ctx.set_spherical(False)
    return ShearXiBatch.apply(list(tasks), lens_geometry, shape_geometry, bins, ctx, *val_A, *w_A, *e1_B, *e2_B,
                              *w_B)
