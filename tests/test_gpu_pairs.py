"""GPU parity of the pair kernels (through the C ABI) against the CPU oracle.

Bar: n_pairs bit-exact with the canonical FP64 bin rule; every FP64 sum within
RTOL = 1e-6 of the oracle relative to the sum of |terms| of that bin (the
natural error scale of a cancelling sum); xi within 1e-6 of the oracle
relative to sum|g terms| / K.
"""
import numpy as np
import pytest

from conftest import uniform_shear
from parity import check_sums

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def canon(oracle, mode, L, S, bins, **kw):
    return oracle.canon_pairs(mode, L, S, bins.bin_edges_sq, **kw)


def assert_parity(res, can, rtol=RTOL, kappa=False, name=None):
    import inspect
    check_sums(name or inspect.stack()[1].function, res, can, rtol=rtol)


def test_shear_uniform(tpcf, oracle, ctx):
    L, S = uniform_shear(4000, 5000, 600.0, 11)
    bins = tpcf.create_bins(1.0, 100.0, 15)
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                     S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, ctx=ctx)
    assert_parity(res, canon(oracle, oracle.SHEAR, L, S, bins))
    assert res.n_pairs.sum() > 100000


def test_kappa_uniform(tpcf, oracle, ctx):
    rng = np.random.default_rng(12)
    n = 6000
    f = lambda a: np.ascontiguousarray(a, np.float32)
    L = dict(x=f(rng.uniform(0, 300, n)), y=f(rng.uniform(0, 300, n)), val=f(rng.normal(0, .02, n)),
             w=f(rng.uniform(.5, 1.5, n)))
    K = dict(x=f(rng.uniform(0, 300, n)), y=f(rng.uniform(0, 300, n)),
             kappa_E=f(rng.normal(0, .02, n)), kappa_B=f(rng.normal(0, .01, n)),
             w=f(rng.uniform(.5, 1.5, n)))
    bins = tpcf.create_bins(0.5, 80.0, 30)
    res = tpcf.scalar_kappa_tpcf(L["x"], L["y"], L["val"], L["w"], K["x"], K["y"], K["kappa_E"],
                                 K["kappa_B"], K["w"], bins, ctx=ctx)
    can = canon(oracle, oracle.KAPPA, L, K, bins)
    assert_parity(res, can)
    np.testing.assert_array_equal(res.sum_K, res.sum_w)


def test_masks_z_cut_and_m(tpcf, oracle, ctx):
    L, S = uniform_shear(3000, 4000, 300.0, 13, w="uniform")
    rng = np.random.default_rng(14)
    L["w"][rng.random(3000) < 0.05] = 0.0                 # skipped lenses (tpcf.f90:285)
    L["z"][:] = rng.uniform(-0.2, 1.0, 3000).astype(np.float32)  # z < 0 masked, z order cut
    S["z"][:] = rng.uniform(-0.2, 1.2, 4000).astype(np.float32)
    S["m"][:] = rng.normal(0, 0.05, 4000).astype(np.float32)
    bins = tpcf.create_bins(1.0, 60.0, 12)
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                     S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, ctx=ctx)
    can = canon(oracle, oracle.SHEAR, L, S, bins)
    assert_parity(res, can)
    assert not np.allclose(res.sum_K, res.sum_w)


def test_exact_edges_lin_and_log(tpcf, oracle, ctx):
    # lens at the origin, sources at exact integer distances: d2 equals a squared
    # edge exactly, including d == x_max (last bin) and d > x_max (no bin)
    xs = np.arange(0, 13, dtype=np.float32)
    L = dict(x=np.zeros(1, np.float32), y=np.zeros(1, np.float32), z=np.zeros(1, np.float32),
             val=np.ones(1, np.float32), w=np.ones(1, np.float32))
    S = dict(x=xs, y=np.zeros_like(xs), z=np.ones_like(xs), e1=np.full_like(xs, 0.1),
             e2=np.zeros_like(xs), w=np.ones_like(xs), m=np.zeros_like(xs))
    for bins in (tpcf.create_bins(0.0, 10.0, 10, spacing="lin"),
                 tpcf.create_bins(1.0, 10.0, 1, spacing="log"),
                 tpcf.create_bins(1.0, 100.0, 2, spacing="log")):
        res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                         S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, ctx=ctx)
        can = canon(oracle, oracle.SHEAR, L, S, bins)
        np.testing.assert_array_equal(res.n_pairs, can["n_pairs"].astype(np.int64))
    lin = tpcf.create_bins(0.0, 10.0, 10, spacing="lin")
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                     S["z"], S["e1"], S["e2"], S["w"], S["m"], lin, ctx=ctx)
    # d = 0 (lin x_min = 0) is in bin 0; 1..9 in bins 1..9; 10 == x_max in bin 9
    np.testing.assert_array_equal(res.n_pairs, [1, 1, 1, 1, 1, 1, 1, 1, 1, 2])


def test_near_edge_guard_band(tpcf, oracle, ctx):
    # many pairs within a few ulp of log edges: the FP64 re-binning path
    bins = tpcf.create_bins(1.0, 100.0, 20)
    rng = np.random.default_rng(15)
    e = bins.bin_edges
    n = 20000
    k = rng.integers(0, 21, n)
    d = e[k] * (1.0 + rng.integers(-40, 41, n) * 1e-8)
    ang = rng.uniform(0, 2 * np.pi, n)
    S = dict(x=(300 + d * np.cos(ang)).astype(np.float32), y=(300 + d * np.sin(ang)).astype(np.float32),
             z=np.ones(n, np.float32), e1=rng.normal(0, .26, n).astype(np.float32),
             e2=rng.normal(0, .26, n).astype(np.float32), w=np.ones(n, np.float32),
             m=np.zeros(n, np.float32))
    L = dict(x=np.full(3, 300, np.float32), y=np.full(3, 300, np.float32), z=np.zeros(3, np.float32),
             val=np.ones(3, np.float32), w=np.ones(3, np.float32))
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                     S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, ctx=ctx)
    can = canon(oracle, oracle.SHEAR, L, S, bins)
    np.testing.assert_array_equal(res.n_pairs, can["n_pairs"].astype(np.int64))


@pytest.mark.parametrize("spacing", ["lin", "sqrt", "ihs"])
def test_other_spacings(tpcf, oracle, ctx, spacing):
    L, S = uniform_shear(2000, 3000, 200.0, 16)
    bins = tpcf.create_bins(0.5 if spacing != "lin" else 0.0, 50.0, 17, spacing=spacing, p=0.3)
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                     S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, ctx=ctx)
    assert_parity(res, canon(oracle, oracle.SHEAR, L, S, bins))


def test_marks_and_lens_sums(tpcf, oracle, ctx):
    L, S = uniform_shear(2500, 3000, 400.0, 17, w="uniform")
    L["w"][::97] = 0.0
    bins = tpcf.create_bins(1.0, 100.0, 15)
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                     S["z"], S["e1"], S["e2"], S["w"], S["m"], bins,
                                     calculate_marks=True, lens_sums=True, ctx=ctx)
    idx = np.arange(0, 2500, 7)
    can = canon(oracle, oracle.SHEAR, L, S, bins, lens_idx=idx)
    lens = can["lens"]                       # [n_sel][6][n_bin]: dw, gt, gx, w, K, n
    got = res.lens_sums[idx]
    np.testing.assert_array_equal(got[:, 5], lens[:, 5])
    scale = np.abs(lens).sum(axis=2, keepdims=True) + 1e-300
    assert np.all(np.abs(got[:, :5] - lens[:, :5]) <= 1e-6 * scale[:, :5])
    # marks are FP32 (as in the reference): within FP32 rounding of the FP64 sums
    assert np.all(np.abs(res.xi_E_marks[idx] - lens[:, 1]) <= 2e-6 * scale[:, 1] + 1e-7 * np.abs(lens[:, 1]))
    np.testing.assert_allclose(res.w_marks[idx], lens[:, 3], rtol=2e-6)
    np.testing.assert_allclose(res.marks_weight[idx], lens[:, 3].sum(1), rtol=2e-6)
    assert np.all(res.xi_E_marks[::97] == 0) and np.all(res.marks_weight[::97] == 0)


def test_grid_equals_all_pairs(tpcf, oracle):
    L, S = uniform_shear(1500, 2500, 300.0, 18)
    bins = tpcf.create_bins(1.0, 40.0, 10)
    a = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                   S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, use_kd_tree=False)
    b = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                   S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, use_kd_tree=True)
    np.testing.assert_array_equal(a.n_pairs, b.n_pairs)
    can = canon(oracle, oracle.SHEAR, L, S, bins)
    assert_parity(a, can)
    assert_parity(b, can)


def test_patches_and_determinism(tpcf, oracle, ctx):
    L, S = uniform_shear(3000, 3000, 300.0, 19)
    rng = np.random.default_rng(20)
    patch = rng.integers(0, 7, 3000).astype(np.int32)
    bins = tpcf.create_bins(1.0, 50.0, 12)
    kw = dict(patch_A=patch, n_patch=7, ctx=ctx)
    r1 = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                    S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, **kw)
    r2 = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"],
                                    S["z"], S["e1"], S["e2"], S["w"], S["m"], bins, **kw)
    for k in ("sum_gt", "sum_gx", "sum_w", "sum_dw", "n_pairs", "patch_sums"):
        np.testing.assert_array_equal(getattr(r1, k), getattr(r2, k))
    for p in range(7):
        can = canon(oracle, oracle.SHEAR, L, S, bins, lens_idx=np.nonzero(patch == p)[0])
        ps = r1.patch_sums[p]
        np.testing.assert_array_equal(ps[5], can["n_pairs"])
        assert np.all(np.abs(ps[1] - can["sum_gt"]) <= 1e-6 * can["abs_gt"] + 1e-300)
    np.testing.assert_allclose(r1.patch_sums.sum(0)[1], r1.sum_gt, rtol=1e-12, atol=1e-15)


def test_empty_and_masked(tpcf, ctx):
    bins = tpcf.create_bins(1.0, 10.0, 5)
    e = np.zeros(0, np.float32)
    one = np.ones(4, np.float32)
    r = tpcf.tangential_shear_tpcf(e, e, e, e, e, one, one, one, one, one, one, one * 0, bins, ctx=ctx)
    assert r.n_pairs.sum() == 0 and np.all(np.isnan(r.mean_theta)) and np.all(r.g_t == 0)
    r = tpcf.tangential_shear_tpcf(one, one, one, one, one * 0, one, one, one, one, one, one,
                                   one * 0, bins, ctx=ctx)
    assert r.n_pairs.sum() == 0


def test_batch_matches_single_calls(tpcf, oracle, ctx):
    cats = [uniform_shear(1500 + 300 * i, 2000 + 500 * i, 300.0, 30 + i) for i in range(2)]
    lenses = [tpcf.LensCatalog(x=L["x"], y=L["y"], val=L["val"], w=L["w"], z=L["z"]) for L, _ in cats]
    shapes = [tpcf.ShapeCatalog(x=S["x"], y=S["y"], e1=S["e1"], e2=S["e2"], w=S["w"], z=S["z"],
                                m=S["m"]) for _, S in cats]
    tasks = [(i, j) for i in range(2) for j in range(2)]
    bins = tpcf.create_bins(1.0, 60.0, 14)
    outs = tpcf.batch_shear_2pcf(lenses, shapes, tasks, bins, ctx=ctx)
    for (i, j), r in zip(tasks, outs):
        can = canon(oracle, oracle.SHEAR, cats[i][0], cats[j][1], bins)
        assert_parity(r, can)


def test_cell_size_autotune_keeps_results(tpcf, oracle):
    at = __import__("importlib").import_module("2pcf_b200.autotune")
    L, S = uniform_shear(3000, 4000, 400.0, 88)
    lens = [tpcf.LensCatalog(x=L["x"], y=L["y"], val=L["val"], w=L["w"], z=L["z"])]
    shp = [tpcf.ShapeCatalog(x=S["x"], y=S["y"], e1=S["e1"], e2=S["e2"], w=S["w"], z=S["z"], m=S["m"])]
    bins = tpcf.create_bins(1.0, 80.0, 12)
    ctx = tpcf.Context(0)
    timing = at.autotune_cell_size(lens, shp, [(0, 0)], bins, ctx, divisors=(8, 16, 48))
    assert set(timing) == {8, 16, 48} and ctx.cell_size == bins.x_max / min(timing, key=timing.get)
    can = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq)
    for d in (5, 16, 64):
        ctx.set_cell_size(bins.x_max / d)
        r = tpcf.batch_shear_2pcf(lens, shp, [(0, 0)], bins, ctx=ctx)[0]
        assert_parity(r, can)
    # every tile shape the tuner can pick gives the same pair sums
    for g, t in ((128, 2), (128, 1), (64, 2), (32, 2)):
        ctx.set_tile_shape(g, t)
        r = tpcf.batch_shear_2pcf(lens, shp, [(0, 0)], bins, ctx=ctx)[0]
        assert_parity(r, can, name=f"tile shape {g} threads x {t} sub-chunks")
    tuned = at.autotune(lens, shp, [(0, 0)], bins, ctx, divisors=(16, 48))
    assert set(tuned["tile"]) == {"128x2", "128x1", "64x2"}
    assert ctx.tile_shape == (tuned["choice"]["group_size"], tuned["choice"]["tile_chunks"])
    ctx.close()


def test_batched_scalar_scalar_equals_single_calls(tpcf, oracle, ctx):
    """tpcf_batch_scalar_scalar: every (scalar catalogue, kappa map) task of one
    launch against the FP64 oracle and against tpcf_scalar_scalar."""
    rng = np.random.default_rng(96)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    lens, kap, raw = [], [], []
    for n, box in ((3000, 300.0), (1500, 250.0)):
        L = dict(x=f(rng.uniform(0, box, n)), y=f(rng.uniform(0, box, n)), val=f(rng.normal(0, .02, n)),
                 w=f(rng.uniform(.5, 1.5, n)))
        K = dict(x=f(rng.uniform(0, box, 2 * n)), y=f(rng.uniform(0, box, 2 * n)),
                 kappa_E=f(rng.normal(0, .02, 2 * n)), kappa_B=f(rng.normal(0, .01, 2 * n)),
                 w=f(rng.uniform(.5, 1.5, 2 * n)))
        raw.append((L, K))
        lens.append(tpcf.LensCatalog(x=L["x"], y=L["y"], val=L["val"], w=L["w"]))
        kap.append(tpcf.KappaMap(**K))
    bins = tpcf.create_bins(0.5, 60.0, 16)
    tasks = [(0, 0), (0, 1), (1, 0), (1, 1)]
    outs = tpcf.batch_kappa_2pcf(lens, kap, tasks, bins, ctx=ctx)
    for (i, j), r in zip(tasks, outs):
        L, _ = raw[i]
        _, K = raw[j]
        can = oracle.canon_pairs(oracle.KAPPA, L, K, bins.bin_edges_sq)
        assert_parity(r, can, name=f"batched scalar-scalar task ({i}, {j})")
        one = tpcf.scalar_kappa_tpcf(L["x"], L["y"], L["val"], L["w"], K["x"], K["y"], K["kappa_E"], K["kappa_B"],
                                     K["w"], bins, calculate_marks=False, ctx=ctx)
        np.testing.assert_array_equal(one.n_pairs, r.n_pairs)
        np.testing.assert_allclose(one.sum_gt, r.sum_gt, rtol=1e-13, atol=1e-13 * np.abs(one.sum_gt).max())
