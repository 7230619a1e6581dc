"""Cell-size autotuner for the pair kernel.

The grid cell side trades the area scanned around each lens group (smaller
cells hug the theta_max disc more tightly) against per-row and partial-tile
overhead (more, shorter source runs).  ``autotune_cell_size`` times the pair
kernel (CUDA events on the launch stream, via tpcf_last_stats) for a list of
cell sides theta_max/d on a corner of the field that keeps the object density,
and sets the fastest on the context.  Results do not depend on the cell size
(every pair is binned by the same rule); only speed does.
"""
from __future__ import annotations

import numpy as np

from . import Context, LensCatalog, ShapeCatalog, batch_shear_2pcf

DIVISORS = (16, 24, 32, 48, 64, 96)


def _corner(cats, x_cut, y_cut):
    out = []
    for c in cats:
        x, y = np.asarray(c.x), np.asarray(c.y)
        keep = (x < x_cut) & (y < y_cut)
        fields = {k: (None if v is None else np.ascontiguousarray(np.asarray(v)[keep]))
                  for k, v in vars(c).items()}
        out.append(type(c)(**fields))
    return out


def autotune_cell_size(lenses, shapes, tasks, bins, ctx: Context, divisors=DIVISORS, corner=0.6, reps=2,
                       spherical_coords=False):
    """Pick the cell side theta_max/d (d in ``divisors``) with the shortest pair
    kernel on the lower-left ``corner`` fraction of the field, set it on ``ctx``
    and return {d: ms per 1e9 binned pairs}.  Host (numpy) catalogues."""
    xs = np.concatenate([np.asarray(c.x) for c in list(lenses) + list(shapes)])
    ys = np.concatenate([np.asarray(c.y) for c in list(lenses) + list(shapes)])
    x0, x1, y0, y1 = xs.min(), xs.max(), ys.min(), ys.max()
    L = _corner(lenses, x0 + corner * (x1 - x0), y0 + corner * (y1 - y0))
    S = _corner(shapes, x0 + corner * (x1 - x0), y0 + corner * (y1 - y0))
    timing = {}
    ctx.set_timing(True)
    for d in divisors:
        ctx.set_cell_size(bins.x_max / d)
        best = None
        for _ in range(reps):
            outs = batch_shear_2pcf(L, S, tasks, bins, spherical_coords=spherical_coords, ctx=ctx)
            st = ctx.stats()
            pairs = sum(int(o.n_pairs.sum()) for o in outs)
            cost = st["pair_kernel_ms"] / max(pairs, 1) * 1e9
            best = cost if best is None else min(best, cost)
        timing[d] = best
    d_best = min(timing, key=timing.get)
    ctx.set_cell_size(bins.x_max / d_best)
    return timing
