"""tpcf_shear_scalar_noalloc: the pair sum for callers that cannot allocate
device memory (their GPU memory belongs to a framework allocator or a fixed
pool, or they cannot afford cudaMalloc/cudaFree's device-wide synchronisation).
It takes all scratch from one static device array instead.

Called through the C ABI and checked against tpcf_shear_scalar on two calls in
a row (the second, smaller call runs over the first call's leftover scratch),
with the tolerance of the other parity tests: n_pairs identical, sums within
1e-6 of the oracle's sum of |terms|.  This file sorts last so that a run
stopping at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from conftest import uniform_shear

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def call_noalloc(tpcf, ctx, L, S, bins):
    lib = tpcf._lib.lib()
    nb = bins.n_bin
    out = {k: np.zeros(nb) for k in ("sum_dw", "sum_gt", "sum_gx", "sum_w", "sum_K")}
    out["n_pairs"] = np.zeros(nb, np.int64)
    for k in ("theta", "mean_theta", "g_t", "g_x", "weights"):
        out[k] = np.zeros(nb, np.float32)
    res = tpcf._lib.Result(**{k: v.ctypes.data for k, v in out.items()})
    cb = bins.c_struct()
    ptr = lambda a: a.ctypes.data
    st = lib.tpcf_shear_scalar_noalloc(ctx.handle, ptr(L["x"]), ptr(L["y"]), ptr(L["z"]), ptr(L["val"]),
                                       ptr(L["w"]), len(L["x"]), ptr(S["x"]), ptr(S["y"]), ptr(S["z"]),
                                       ptr(S["e1"]), ptr(S["e2"]), ptr(S["w"]), ptr(S["m"]), len(S["x"]),
                                       C.byref(cb), C.byref(res))
    return st, out


def compare(got, ref, can, name):
    np.testing.assert_array_equal(got["n_pairs"], ref.n_pairs)
    for q, scale in (("sum_gt", "abs_gt"), ("sum_gx", "abs_gx"), ("sum_w", "sum_w"),
                     ("sum_K", "sum_K"), ("sum_dw", "sum_dw")):
        assert np.all(np.abs(got[q] - getattr(ref, q)) <= RTOL * np.abs(can[scale]) + 1e-300), (name, q)
    np.testing.assert_array_equal(got["theta"], ref.theta)
    K = can["sum_K"]
    with np.errstate(invalid="ignore", divide="ignore"):
        for q, scale in (("g_t", "abs_gt"), ("g_x", "abs_gx")):
            band = RTOL * np.where(K > 0, can[scale] / np.where(K > 0, K, 1), 0) + 2e-7 * np.abs(getattr(ref, q))
            assert np.all(np.abs(got[q].astype(np.float64) - getattr(ref, q)) <= band + 1e-30), (name, q)
        np.testing.assert_allclose(got["weights"], ref.weights, rtol=2e-7)
        np.testing.assert_allclose(got["mean_theta"], ref.mean_theta, rtol=2e-6)   # NaN where no pair


def test_noalloc_matches_regular_entry_point_twice(tpcf, oracle):
    """On a fresh context the no-allocation entry point runs first (twice) and
    the context still holds no device workspace; then the regular entry point
    on the same inputs gives the same results within the tolerance."""
    ctx = tpcf.Context(0)
    bins = tpcf.create_bins(1.0, 60.0, 14)
    cases = []
    for seed, n_lens, n_src in ((41, 7000, 9000), (42, 2500, 3100)):
        L, S = uniform_shear(n_lens, n_src, 300.0, seed, w="uniform")
        L["w"][::61] = 0.0
        st, got = call_noalloc(tpcf, ctx, L, S, bins)
        assert st == 0, tpcf._lib.lib().tpcf_last_error(ctx.handle)
        assert ctx.stats()["workspace_bytes"] == 0
        cases.append((L, S, got))
    for i, (L, S, got) in enumerate(cases):
        ref = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                         S["z"], S["e1"], S["e2"], S["w"], S["m"], bins,
                                         calculate_marks=False, ctx=ctx)
        can = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq)
        compare(got, ref, can, f"call {i}")
    assert ctx.stats()["workspace_bytes"] > 0    # the regular entry point does allocate
    ctx.close()


def test_noalloc_small_theta_over_wide_field(tpcf, oracle):
    """theta_max = 10' over a 20000' field: the cell table would need more than
    the whole scratch at the regular cell side, so this entry point coarsens the
    cells; the results stay those of the regular entry point."""
    rng = np.random.default_rng(45)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    centres = rng.uniform(0, 20000, (12, 2))

    def clumps(n):
        c = centres[rng.integers(0, 12, n)]
        return f(c[:, 0] + rng.normal(0, 6, n)), f(c[:, 1] + rng.normal(0, 6, n))

    xl, yl = clumps(3000)
    xs, ys = clumps(4000)
    L = dict(x=xl, y=yl, z=np.zeros(3000, np.float32), val=f(rng.normal(0, .02, 3000)),
             w=f(rng.uniform(.5, 1.5, 3000)))
    S = dict(x=xs, y=ys, z=np.ones(4000, np.float32), e1=f(rng.normal(0, .26, 4000)),
             e2=f(rng.normal(0, .26, 4000)), w=f(rng.uniform(.5, 1.5, 4000)), m=np.zeros(4000, np.float32))
    bins = tpcf.create_bins(0.5, 10.0, 8)
    ctx = tpcf.Context(0)
    st, got = call_noalloc(tpcf, ctx, L, S, bins)
    assert st == 0, tpcf._lib.lib().tpcf_last_error(ctx.handle)
    assert got["n_pairs"].sum() > 100000
    ref = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"], S["e1"],
                                     S["e2"], S["w"], S["m"], bins, calculate_marks=False, ctx=ctx)
    compare(got, ref, oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq), "wide field")
    ctx.close()


def test_noalloc_rejects_oversized_call(tpcf):
    ctx = tpcf.Context(0)
    bins = tpcf.create_bins(1.0, 60.0, 14)
    L, S = uniform_shear(1000, 3_000_000, 300.0, 43)
    st, _ = call_noalloc(tpcf, ctx, L, S, bins)
    assert st == 3  # TPCF_ERR_OVERFLOW: beyond the static scratch
    assert b"static scratch" in tpcf._lib.lib().tpcf_last_error(ctx.handle)
    ctx.close()
