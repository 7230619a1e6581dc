"""Autotuner for the planar pair kernel: cell side and tile shape.

The grid cell side trades the area scanned around each lens group (smaller
cells hug the theta_max disc more tightly) against per-row overhead and
partial sub-chunks at the ends of shorter source runs.  The tile shape is the
number of threads per block (128 or 64: warps, each with its own 32-lens work
items, sharing one block's shared memory) and the number of 32-source
sub-chunks per source tile (2 or 1: fewer, larger copies against more tiles
in flight in each warp's ring).  ``autotune`` times the pair kernel
(CUDA events on the launch stream, via tpcf_last_stats) on a corner of the
field that keeps the object density: first every cell side theta_max/d with
the default shape, then every shape with the best cell side, and sets the
fastest on the context.  Results do not depend on either choice (every pair
is binned by the same rule); only speed does.
"""
from __future__ import annotations

import numpy as np

from . import Context, batch_shear_2pcf

DIVISORS = (16, 24, 32, 48, 64, 96)
SHAPES = ((128, 2), (128, 1), (64, 2))   # (threads per block, sub-chunks per tile)


def _corner(cats, x_cut, y_cut):
    out = []
    for c in cats:
        x, y = np.asarray(c.x), np.asarray(c.y)
        keep = (x < x_cut) & (y < y_cut)
        fields = {k: (None if v is None else np.ascontiguousarray(np.asarray(v)[keep]))
                  for k, v in vars(c).items()}
        out.append(type(c)(**fields))
    return out


def _cost(L, S, tasks, bins, ctx, reps, spherical_coords):
    best = None
    for _ in range(reps):
        outs = batch_shear_2pcf(L, S, tasks, bins, spherical_coords=spherical_coords, ctx=ctx)
        pairs = sum(int(o.n_pairs.sum()) for o in outs)
        cost = ctx.stats()["pair_kernel_ms"] / max(pairs, 1) * 1e9
        best = cost if best is None else min(best, cost)
    return best


def autotune(lenses, shapes, tasks, bins, ctx: Context, divisors=DIVISORS, tile_shapes=SHAPES, corner=0.5, reps=2,
             spherical_coords=False):
    """Pick the cell side theta_max/d and the tile shape with the shortest pair
    kernel per binned pair on the lower-left ``corner`` fraction of the field,
    set them on ``ctx`` and return {"cell": {d: ms per 1e9 pairs}, "tile":
    {"GxT": ms per 1e9 pairs}, "choice": {"cell_divisor", "group_size",
    "tile_chunks"}}.  Host (numpy) catalogues."""
    xs = np.concatenate([np.asarray(c.x) for c in list(lenses) + list(shapes)])
    ys = np.concatenate([np.asarray(c.y) for c in list(lenses) + list(shapes)])
    x0, x1, y0, y1 = xs.min(), xs.max(), ys.min(), ys.max()
    L = _corner(lenses, x0 + corner * (x1 - x0), y0 + corner * (y1 - y0))
    S = _corner(shapes, x0 + corner * (x1 - x0), y0 + corner * (y1 - y0))
    ctx.set_timing(True)
    shape0 = tile_shapes[0] if not spherical_coords else (0, 0)
    ctx.set_tile_shape(*shape0)
    cell = {}
    for d in divisors:
        ctx.set_cell_size(bins.x_max / d)
        cell[d] = _cost(L, S, tasks, bins, ctx, reps, spherical_coords)
    d_best = min(cell, key=cell.get)
    ctx.set_cell_size(bins.x_max / d_best)
    tile = {}
    if not spherical_coords:   # the spherical kernel has one shape
        for g, t in tile_shapes:
            ctx.set_tile_shape(g, t)
            tile[f"{g}x{t}"] = _cost(L, S, tasks, bins, ctx, reps, spherical_coords)
    best = min(tile, key=tile.get) if tile else None
    g_best, t_best = (int(v) for v in best.split("x")) if best else (0, 0)
    ctx.set_tile_shape(g_best, t_best)
    return {"cell": cell, "tile": tile,
            "choice": {"cell_divisor": d_best, "group_size": g_best, "tile_chunks": t_best}}


def autotune_cell_size(lenses, shapes, tasks, bins, ctx: Context, divisors=DIVISORS, corner=0.6, reps=2,
                       spherical_coords=False):
    """The cell side alone (default tile shape): sets it on ``ctx`` and returns
    {d: ms per 1e9 binned pairs}."""
    r = autotune(lenses, shapes, tasks, bins, ctx, divisors=divisors, tile_shapes=((0, 0),), corner=corner,
                 reps=reps, spherical_coords=spherical_coords)
    return r["cell"]
