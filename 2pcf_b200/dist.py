"""Combining sharded calls across ranks (one process per GPU).

With ``Context.set_shard(rank, world)`` each rank computes a disjoint, balanced
share of the work items of a call, so its FP64 per-bin sums, n_pairs and
per-patch sums are partial.  ``combine_shards`` adds them over all ranks with
one all-reduce (NCCL on GPUs; gloo works for the same tensors on CPU) and
recomputes the reference normalisation (src/tpcf.f90:369-376).  There is no
other exchange: inputs are replicated and every rank builds its own grid.
"""
from __future__ import annotations

from typing import List

import numpy as np

SUM_FIELDS = ("sum_dw", "sum_gt", "sum_gx", "sum_w", "sum_K")


def _pack(results):
    parts = []
    for r in results:
        parts += [np.asarray(getattr(r, k), np.float64) for k in SUM_FIELDS]
        parts.append(np.asarray(r.n_pairs, np.float64))  # exact below 2^53
        if r.patch_sums is not None:
            parts.append(np.asarray(r.patch_sums, np.float64).ravel())
    return np.concatenate(parts)


def _unpack(results, flat):
    o = 0
    for r in results:
        nb = r.n_bin
        for k in SUM_FIELDS:
            setattr(r, k, flat[o:o + nb].copy())
            o += nb
        r.n_pairs = np.rint(flat[o:o + nb]).astype(np.int64)
        o += nb
        if r.patch_sums is not None:
            n = r.patch_sums.size
            r.patch_sums = flat[o:o + n].reshape(r.patch_sums.shape).copy()
            o += n
        with np.errstate(invalid="ignore", divide="ignore"):
            r.mean_theta = (r.sum_dw / r.sum_w).astype(np.float32)
            K = r.sum_K
            pos = K > 0
            r.g_t = np.where(pos, r.sum_gt / np.where(pos, K, 1), 0).astype(np.float32)
            r.g_x = np.where(pos, r.sum_gx / np.where(pos, K, 1), 0).astype(np.float32)
            r.weights = r.sum_w.astype(np.float32)
    return results


def combine_shards(results: List, group=None):
    """All-reduce (sum) the sharded results of one call over the process group,
    in place, and return them with normalised outputs recomputed."""
    import torch
    import torch.distributed as dist
    flat = _pack(results)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(flat).to(dev)
    dist.all_reduce(t, group=group)
    return _unpack(results, t.cpu().numpy())
