"""GPU xi from precomputed marks (tpcf_xi_from_marks, calculate_tpcf_from_marks
src/main.f90:1017-1139) against the oracle's FP64 restatement, and the
marks route against the direct pair sum: marks computed once with val = w = 1
and re-weighted by a map give that map's g_t (to the FP32 rounding of the
per-lens marks, 1e-6 of sum|terms|/K)."""
import numpy as np
import pytest

from conftest import uniform_shear

pytestmark = pytest.mark.gpu


def rand_marks(rng, n, nb):
    return {"x": rng.normal(size=n).astype(np.float32), "y": rng.normal(size=n).astype(np.float32),
            "w": np.where(rng.random(n) < 0.1, 0.0, rng.uniform(0.1, 2, n)).astype(np.float32),
            "xi_E": rng.normal(size=(n, nb)).astype(np.float32), "xi_B": rng.normal(size=(n, nb)).astype(np.float32),
            "K": rng.uniform(0.5, 1.5, (n, nb)).astype(np.float32)}


@pytest.mark.parametrize("nb,n_map", [(15, 6), (20, 11), (32, 16), (40, 6)])
def test_matches_oracle_for_several_maps(tpcf, oracle, ctx, nb, n_map):
    """n_bin <= 32 sums on the FP64 tensor cores (20, 32: whole 16-byte marks
    rows; 15: 4-byte copies), wider binnings on the FP64 FMA form; one map
    tile (6 maps) or two (11, 16)."""
    rng = np.random.default_rng(nb)
    raw = [rand_marks(rng, n, nb) for n in (5000, 0, 12345)]
    marks = [tpcf.MarksField(**m) for m in raw]
    vals = [rng.normal(0, 0.02, (n_map, len(m["x"]))).astype(np.float32) for m in raw]
    ws = [np.where(rng.random((n_map, len(m["x"]))) < 0.05, 0.0,
                   rng.uniform(0.5, 1.5, (n_map, len(m["x"])))).astype(np.float32) for m in raw]
    out = tpcf.calculate_tpcf_from_marks(marks, vals, ws, ctx=ctx)
    for m in range(n_map):
        per, st = oracle.xi_from_marks(raw, [v[m] for v in vals], [w[m] for w in ws])
        for i, p in enumerate(per):
            np.testing.assert_allclose(out["g_t"][m, i], p["g_t"], rtol=1e-9, equal_nan=True)
            np.testing.assert_allclose(out["g_x"][m, i], p["g_x"], rtol=1e-9, equal_nan=True)
            np.testing.assert_allclose(out["weights"][m, i], p["weights"], rtol=1e-12)
        np.testing.assert_allclose(out["g_t_stacked"][m], st["g_t"], rtol=1e-9)
        np.testing.assert_allclose(out["weights_stacked"][m], st["weights"], rtol=1e-12)


def test_marks_route_equals_direct_pair_sum(tpcf, ctx):
    L, S = uniform_shear(4000, 6000, 400.0, 21, w="uniform")
    bins = tpcf.create_bins(1.0, 60.0, 10)
    ones = np.ones_like(L["val"])
    m = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], ones, ones, S["x"], S["y"], S["z"], S["e1"], S["e2"],
                                   S["w"], S["m"], bins, calculate_marks=True, ctx=ctx)
    mf = tpcf.MarksField.from_results(tpcf.LensCatalog(x=L["x"], y=L["y"], val=ones, w=ones), m)
    direct = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                        S["e1"], S["e2"], S["w"], S["m"], bins, calculate_marks=True, ctx=ctx)
    out = tpcf.calculate_tpcf_from_marks([mf], [L["val"]], [L["w"]], lens_x=[L["x"]], lens_y=[L["y"]], ctx=ctx)
    scale = np.abs(direct.xi_E_marks).sum(0, dtype=np.float64) / direct.sum_K
    assert np.all(np.abs(out["g_t"][0] - direct.sum_gt / direct.sum_K) <= 1e-6 * scale)
    # the reference's weights output is sum_j marks_w_j w_j (one number per field)
    np.testing.assert_allclose(out["weights"][0], (m.marks_weight.astype(np.float64) * L["w"]).sum(), rtol=1e-9)


def test_position_mismatch_is_rejected(tpcf, ctx):
    rng = np.random.default_rng(3)
    raw = rand_marks(rng, 100, 5)
    mf = tpcf.MarksField(**raw)
    bad = raw["x"].copy()
    bad[17] += 1e-3
    with pytest.raises(tpcf.TPCFError):
        tpcf.calculate_tpcf_from_marks([mf], [np.ones(100, np.float32)], [np.ones(100, np.float32)],
                                       lens_x=[bad], lens_y=[raw["y"]], ctx=ctx)


def test_device_tensors(tpcf, oracle, ctx):
    import torch
    rng = np.random.default_rng(4)
    raw = [rand_marks(rng, 3000, 12)]
    marks = [tpcf.MarksField(**{k: torch.from_numpy(v).cuda() for k, v in raw[0].items()})]
    v = rng.normal(size=(2, 3000)).astype(np.float32)
    w = rng.uniform(0.5, 1.5, (2, 3000)).astype(np.float32)
    out = tpcf.calculate_tpcf_from_marks(marks, [torch.from_numpy(v).cuda()], [torch.from_numpy(w).cuda()], ctx=ctx)
    per, _ = oracle.xi_from_marks(raw, [v[1]], [w[1]])
    np.testing.assert_allclose(out["g_t"][1, 0], per[0]["g_t"], rtol=1e-9)


def test_point_bootstrap_matches_oracle(tpcf, oracle, ctx):
    """Per-lens resampling over two fields: the drawn multiplicities are those
    of the patch bootstrap's Philox stream with the lenses as units."""
    rng = np.random.default_rng(11)
    raw = [rand_marks(rng, n, 9) for n in (3000, 1234)]
    marks = [tpcf.MarksField(**m) for m in raw]
    n_boot, n_units = 37, 4234
    out = tpcf.marks_bootstrap(marks, n_boot, seed=77, supersampling_factor=1.3, ctx=ctx)
    mult = oracle.bootstrap_multiplicity(77, n_boot, n_units, int(n_units * 1.3))
    gt, gx, W = oracle.marks_bootstrap(raw, mult)
    np.testing.assert_allclose(out["g_t"], gt, rtol=1e-10)
    np.testing.assert_allclose(out["g_x"], gx, rtol=1e-10)
    np.testing.assert_allclose(out["weights"], W, rtol=1e-12)
    np.testing.assert_allclose(out["cov_g_t"], np.cov(gt.T), rtol=1e-8, atol=1e-300)


def test_block_bootstrap_from_labels(tpcf, oracle, ctx):
    rng = np.random.default_rng(12)
    raw = [rand_marks(rng, 5000, 12)]
    marks = [tpcf.MarksField(**m) for m in raw]
    labels = rng.integers(0, 50, 5000).astype(np.int32)
    mult = rng.integers(0, 3, (20, 50)).astype(np.int32)
    out = tpcf.marks_bootstrap(marks, 20, units=labels, n_units=50, multiplicity=mult, k_guard=False,
                               covariance=False, ctx=ctx)
    gt, gx, W = oracle.marks_bootstrap(raw, mult, units=labels, k_guard=False)
    np.testing.assert_allclose(out["g_t"], gt, rtol=1e-10)
    np.testing.assert_allclose(out["weights"], W, rtol=1e-12)
    with pytest.raises(tpcf.TPCFError):
        tpcf.marks_bootstrap(marks, 2, units=labels, n_units=40, ctx=ctx)
