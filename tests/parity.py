"""Parity measures shared by the GPU tests.

Every comparison against the FP64 oracle goes through ``check_sums`` (per-bin
sums of one call) or ``check_lens_sums`` (per-lens sums), which assert the bar
and return -- and print, and append to the JSON-lines file named by the
environment variable TPCF_PARITY_LOG when it is set -- what was observed:

- n_pairs: bit-exact with the canonical FP64 bin rule (asserted);
- every FP64 sum: |got - oracle| <= RTOL * sum|terms| of its bin (asserted),
  reported as the margin = max |got - oracle| / (RTOL * sum|terms|), so a
  margin of 0.01 means the error used 1% of the allowed band;
- xi = sum_gt / sum_K (and xi_x): the relative error |dxi| / |xi| per bin
  against the oracle's FP64 xi, with the bins whose relative error exceeds
  RTOL listed together with the ratio |sum_gt| / sum|g_t terms| of those bins
  (how much the terms cancel: a bin whose xi is a small remainder of a large
  cancelling sum carries the absolute error of that sum in a small number).
  Asserted: every bin is within RTOL relative in xi, or within RTOL of
  sum|g_t terms| / K in absolute terms (the scale of the cancelling sum).
"""
from __future__ import annotations

import json
import os

import numpy as np

RTOL = 1e-6
_SUMS = (("sum_gt", "abs_gt"), ("sum_gx", "abs_gx"), ("sum_w", "sum_w"), ("sum_K", "sum_K"),
         ("sum_dw", "sum_dw"))


def _log(rec):
    print("PARITY " + json.dumps(rec), flush=True)
    path = os.environ.get("TPCF_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(rec) + "\n")


def _xi(sg, sK):
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(sK > 0, sg / np.where(sK > 0, sK, 1.0), 0.0)


def check_sums(name, res, can, rtol=RTOL):
    """Per-bin parity of one result (Shear2pcfResults or a dict with the same
    keys) against canon_pairs output ``can``."""
    get = (lambda k: getattr(res, k)) if not isinstance(res, dict) else (lambda k: res[k])
    np_got = np.asarray(get("n_pairs"), np.int64)
    np_ref = can["n_pairs"].astype(np.int64)
    rec = {"case": name, "n_bin": int(len(np_ref)), "binned_pairs": int(np_ref.sum()),
           "n_pairs_exact": bool(np.array_equal(np_got, np_ref))}
    margins = {}
    for q, sc in _SUMS:
        got, exp, scale = np.asarray(get(q), np.float64), can[q], np.abs(can[sc]) + 1e-300
        m = np.abs(got - exp) / (rtol * scale)
        margins[q] = float(np.max(m)) if m.size else 0.0
    rec["margin"] = margins
    K_ref, K_got = can["sum_K"], np.asarray(get("sum_K"), np.float64)
    xt_ref, xt_got = _xi(can["sum_gt"], K_ref), _xi(np.asarray(get("sum_gt"), np.float64), K_got)
    xx_ref, xx_got = _xi(can["sum_gx"], K_ref), _xi(np.asarray(get("sum_gx"), np.float64), K_got)
    with np.errstate(invalid="ignore", divide="ignore"):
        rel_t = np.where(xt_ref != 0, np.abs(xt_got - xt_ref) / np.abs(xt_ref), np.abs(xt_got))
        rel_x = np.where(xx_ref != 0, np.abs(xx_got - xx_ref) / np.abs(xx_ref), np.abs(xx_got))
        cancel = np.abs(can["sum_gt"]) / (np.abs(can["abs_gt"]) + 1e-300)
    rec["xi_t_rel_err_max"] = float(rel_t.max())
    rec["xi_t_rel_err_median"] = float(np.median(rel_t))
    rec["xi_x_rel_err_max"] = float(rel_x.max())
    over = np.nonzero(rel_t > rtol)[0]
    rec["xi_t_bins_over_rtol"] = [{"bin": int(b), "rel_err": float(rel_t[b]),
                                   "sum_over_sum_abs": float(cancel[b])} for b in over]
    _log(rec)
    assert rec["n_pairs_exact"], f"{name}: n_pairs {np_got} expected {np_ref}"
    for q, m in margins.items():
        assert m <= 1.0, f"{name}: {q} off by {m:.3g} x the {rtol} sum|terms| band"
    with np.errstate(invalid="ignore", divide="ignore"):
        band = rtol * np.where(K_ref > 0, can["abs_gt"] / np.where(K_ref > 0, K_ref, 1.0), 0.0)
    ok = (rel_t <= rtol) | (np.abs(xt_got - xt_ref) <= band + 1e-300)
    assert ok.all(), f"{name}: xi_t bins {np.nonzero(~ok)[0]} rel err {rel_t[~ok]}"
    return rec


def check_lens_sums(name, got, can, rtol=RTOL, extra=None):
    """Per-lens parity.  ``got`` is [n][6][n_bin] (d*w, g_t, g_x, w, K, n) from
    the library, ``can`` the canon_pairs output for the same lenses (its
    ``lens`` rows and ``lens_norm`` = per-lens sums of w_B |val w| |(e1, e2)|).
    n bit-exact; d*w, w, K within rtol of the oracle's value (their terms are
    positive); g_t, g_x within rtol of the lens's sum of term bounds in that
    bin.  One lens-bin holds few pairs, and a rotated term that nearly cancels
    (e1 cos 2phi ~ -e2 sin 2phi) carries an FP32 error of a few ulps of
    w |val w| |e|, not of the term: the per-lens band is set on that bound."""
    got = np.asarray(got, np.float64)
    ref, ab = can["lens"], can["lens_norm"]
    rec = {"case": name, "lenses": int(ref.shape[0]), "binned_pairs": int(ref[:, 5].sum()),
           "n_pairs_exact": bool(np.array_equal(got[:, 5], ref[:, 5]))}
    if extra:
        rec.update(extra)
    scales = {"sum_dw": (0, np.abs(ref[:, 0])), "sum_gt": (1, ab[:, 0]), "sum_gx": (2, ab[:, 1]),
              "sum_w": (3, np.abs(ref[:, 3])), "sum_K": (4, np.abs(ref[:, 4]))}
    margins = {}
    for q, (row, sc) in scales.items():
        m = np.abs(got[:, row] - ref[:, row]) / (rtol * sc + 1e-300)
        margins[q] = float(m.max()) if m.size else 0.0
    rec["margin"] = margins
    _log(rec)
    assert rec["n_pairs_exact"], f"{name}: per-lens n_pairs differ"
    for q, m in margins.items():
        assert m <= 1.0, f"{name}: per-lens {q} off by {m:.3g} x the {rtol} band"
    return rec


def log_record(rec):
    _log(rec)
