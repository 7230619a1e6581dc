"""GPU parity of the k-means patches and the batched bootstrap (through the C
ABI) against the oracle: labels, centroids and iteration counts bit-exact
with the deterministic oracle; multiplicities from Philox identical to the
host replica; resampled xi and covariances bit-exact (same FP64 summation
order)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_kmeans_golden(tpcf, ctx):
    g = dict(np.load(os.path.join(GOLD, "kmeans_small.npz")))
    lab, cen, it = tpcf.partition_data(g["x"], g["y"], g["w"], int(g["k"]), ctx=ctx)
    np.testing.assert_array_equal(lab, g["det_labels"])
    np.testing.assert_array_equal(cen, g["det_centroids"])
    assert it == int(g["det_iters"])


def test_kmeans_clustered_100_patches(tpcf, oracle, synth, ctx):
    w = synth.make_workload(3, scale=0.05)
    L = w["lenses"]
    wt = (0.01 + L["w"] / L["w"].max()).astype(np.float32)   # src/tpcf.f90:1104
    lab, cen, it = tpcf.partition_data(L["x"], L["y"], wt, 100, ctx=ctx)
    lab_o, cen_o, it_o = oracle.kmeans_det(L["x"], L["y"], wt, 100)
    np.testing.assert_array_equal(lab, lab_o)
    np.testing.assert_array_equal(cen, cen_o)
    assert it == it_o
    lab2, _, _ = tpcf.partition_data(L["x"], L["y"], wt, 100, ctx=ctx)
    np.testing.assert_array_equal(lab, lab2)   # deterministic
    ref, _, _ = oracle.kmeans_ref_f32(L["x"], L["y"], wt, 100)
    assert np.mean(ref == lab) > 0.98           # vs the FP32-serial restatement


def test_bootstrap_golden(tpcf, ctx):
    g = dict(np.load(os.path.join(GOLD, "bootstrap_small.npz")))
    n_patch, nb = g["St"].shape
    ps = np.zeros((n_patch, 6, nb))
    ps[:, 1], ps[:, 2], ps[:, 4] = g["St"], g["Sx"], g["SK"]
    ps[:, 3, 0] = g["Sw"]
    n_boot = g["mult"].shape[0]
    out = tpcf.block_bootstrap(ps, n_boot, seed=int(g["seed"]), supersampling_factor=1.0, ctx=ctx)
    np.testing.assert_array_equal(out["multiplicity"], g["mult"])
    np.testing.assert_array_equal(out["g_t"][:, 0], g["gt"])
    np.testing.assert_array_equal(out["g_x"][:, 0], g["gx"])
    np.testing.assert_array_equal(out["weights"][:, 0], g["W"])
    np.testing.assert_array_equal(out["cov_g_t"], g["cov_gt"])
    out2 = tpcf.block_bootstrap(ps, n_boot, multiplicity=g["mult"], ctx=ctx)
    np.testing.assert_array_equal(out2["g_t"][:, 0], g["gt"])


def test_pairs_kmeans_bootstrap_chain(tpcf, oracle, ctx):
    """Patch sums from the pair kernel with device k-means labels, resampled on
    the device, against the oracle chain (per-patch oracle sums, same
    multiplicities)."""
    from conftest import uniform_shear
    L, S = uniform_shear(3000, 4000, 300.0, 77, w="uniform")
    wt = (0.01 + L["w"] / L["w"].max()).astype(np.float32)
    lab, _, _ = tpcf.partition_data(L["x"], L["y"], wt, 9, ctx=ctx)
    bins = tpcf.create_bins(1.0, 60.0, 10)
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                     S["e1"], S["e2"], S["w"], S["m"], bins, patch_A=lab, n_patch=9,
                                     calculate_marks=False, ctx=ctx)
    boot = tpcf.block_bootstrap(res.patch_sums, 200, seed=99, ctx=ctx)
    mult = oracle.bootstrap_multiplicity(99, 200, 9, 9)
    np.testing.assert_array_equal(boot["multiplicity"], mult)
    St = np.zeros((9, 10)); SK = np.zeros((9, 10)); Sx = np.zeros((9, 10)); Sw = np.zeros(9)
    for p in range(9):
        c = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq, lens_idx=np.nonzero(lab == p)[0])
        St[p], Sx[p], SK[p], Sw[p] = c["sum_gt"], c["sum_gx"], c["sum_K"], c["sum_w"].sum()
        np.testing.assert_array_equal(res.patch_sums[p, 5], c["n_pairs"])
    gt, gx, W = oracle.block_bootstrap(mult, St, Sx, SK, Sw)
    scale = np.abs(gt).max()
    assert np.all(np.abs(boot["g_t"][:, 0] - gt) <= 1e-6 * scale)
    cov = oracle.covariance(gt)
    assert np.all(np.abs(boot["cov_g_t"] - cov) <= 1e-5 * np.abs(cov).max())


@pytest.mark.parametrize("random_init", [True, False])
def test_equal_weight_kmeans_bit_exact(tpcf, oracle, ctx, random_init):
    """partition_data with equal_size (src/kmeans.f90:12-262): labels and
    centroids bit-exact with the oracle's serial restatement (chunked sweep,
    fixed-point weights, rebalance), and far more even cluster weights than
    plain k-means."""
    rng = np.random.default_rng(31)
    n = 60000
    x = np.concatenate([rng.normal(200, 20, n // 2), rng.uniform(0, 1000, n - n // 2)]).astype(np.float32)
    y = np.concatenate([rng.normal(300, 20, n // 2), rng.uniform(0, 800, n - n // 2)]).astype(np.float32)
    w = rng.uniform(0.01, 1.01, n).astype(np.float32)
    lab, cen, it, dev = tpcf.partition_data_equal(x, y, w, 40, random_init=random_init, seed=9, ctx=ctx)
    olab, ocen, oit, odev = oracle.kmeans_equal(x, y, w, 40, random_init=random_init, seed=9)
    assert it == oit
    np.testing.assert_array_equal(lab, olab)
    np.testing.assert_array_equal(cen, ocen)
    assert dev == odev
    W = np.bincount(lab, weights=w.astype(np.float64), minlength=40)
    assert abs((W.max() - W.min()) / W.mean() - dev) < 1e-5
    plab, _, _ = tpcf.partition_data(x, y, w, 40, ctx=ctx)
    Wp = np.bincount(plab, weights=w.astype(np.float64), minlength=40)
    assert dev < 0.5 * (Wp.max() - Wp.min()) / Wp.mean()
