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
    return ShearXi.apply(val_A, w_A, e1_B, e2_B, w_B, geometry, bins, ctx)
