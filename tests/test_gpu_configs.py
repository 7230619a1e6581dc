"""Parity of the benchmark configurations at their stated sizes against the
FP64 oracle, through the C ABI.

- Configuration 1 (20k x 20k uniform, 15 log bins 1-100', shear-scalar and
  scalar-scalar): every pair against the FP64 brute force -- n_pairs
  bit-exact, every sum, xi -- and against the FP64 restatement of the
  reference loop (kd-tree, log10 binning: the reference compiled with 8-byte
  reals).
- Configuration 3 (2 M shear x 500 k scalar, clustered, 100 k-means patches,
  1000 resamples, 20 log bins 1-200'): k-means labels bit-exact with the
  deterministic oracle; per-lens sums of 5 lenses in every patch (500) against
  the FP64 brute force of those lenses over all 2 M sources; the per-patch
  sums add up to the totals and equal the sums of the per-lens rows of their
  patches; the resampled xi and covariance equal the oracle's bootstrap of the
  same patch sums with the same multiplicities.
- Configuration 4 (the clustered 2 M x 500 k data, chi^2 of xi_t against a
  seeded target with the diagonal bootstrap variance): the adjoint's
  gradients of 500 lenses and 500 sources against the FP64 brute-force
  gradient and against central finite differences (step 1e-3) of the FP64
  loss.

Each case prints (and appends to $TPCF_PARITY_LOG) its observed margins and xi
errors (tests/parity.py).
"""
import os

import numpy as np
import pytest

from parity import check_lens_sums, check_sums, log_record

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def w1(synth):
    return synth.make_workload(1)


@pytest.fixture(scope="module")
def w3(synth):
    return synth.make_workload(3)


def test_config1_shear_all_pairs(tpcf, oracle, ctx, w1):
    L, S = w1["lenses"], w1["shapes"]
    bins = tpcf.create_bins(*w1["bins"])
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                     S["e1"], S["e2"], S["w"], S["m"], bins, calculate_marks=False, ctx=ctx)
    can = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq)
    check_sums("config1 shear-scalar 20k x 20k vs FP64 brute force", res, can)
    # the reference loop restated in FP64 (kd-tree, find_bin_index on log10 d)
    ref = oracle.ref_pairs(oracle.SHEAR, L, S, *w1["bins"], num_threads=os.cpu_count(), dtype=np.float64)
    np.testing.assert_array_equal(res.n_pairs, ref["n_pairs"])
    rel = np.abs(res.g_t.astype(np.float64) - ref["g_t"]) / np.abs(ref["g_t"])
    log_record({"case": "config1 shear-scalar vs FP64 reference restatement", "n_pairs_exact": True,
                "g_t_rel_err_max": float(rel.max()), "g_t_rel_err_median": float(np.median(rel))})


def test_config1_kappa_all_pairs(tpcf, oracle, ctx, w1):
    L, K = w1["lenses"], w1["kappa_map"]
    bins = tpcf.create_bins(*w1["bins"])
    res = tpcf.scalar_kappa_tpcf(L["x"], L["y"], L["val"], L["w"], K["x"], K["y"], K["kappa_E"], K["kappa_B"],
                                 K["w"], bins, calculate_marks=False, ctx=ctx)
    can = oracle.canon_pairs(oracle.KAPPA, L, K, bins.bin_edges_sq)
    check_sums("config1 scalar-scalar 20k x 20k vs FP64 brute force", res, can)
    ref = oracle.ref_pairs(oracle.KAPPA, L, K, *w1["bins"], num_threads=os.cpu_count(), dtype=np.float64)
    np.testing.assert_array_equal(res.n_pairs, ref["n_pairs"])


def _kmeans_weights(L):
    return (0.01 + L["w"] / L["w"].max()).astype(np.float32)  # src/tpcf.f90:1104


def test_config3_patches_lenses_bootstrap(tpcf, oracle, ctx, w3):
    L, S = w3["lenses"], w3["shapes"]
    bins = tpcf.create_bins(*w3["bins"])
    n_patch, n_boot = w3["n_patch"], w3["n_boot"]
    wt = _kmeans_weights(L)
    lab, cen, it = tpcf.partition_data(L["x"], L["y"], wt, n_patch, ctx=ctx)
    lab_o, cen_o, it_o = oracle.kmeans_det(L["x"], L["y"], wt, n_patch)
    np.testing.assert_array_equal(lab, lab_o)
    np.testing.assert_array_equal(cen, cen_o)
    assert it == it_o
    res = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                     S["e1"], S["e2"], S["w"], S["m"], bins, patch_A=lab, n_patch=n_patch,
                                     calculate_marks=False, lens_sums=True, ctx=ctx)
    ps = res.patch_sums
    np.testing.assert_array_equal(ps[:, 5].sum(0), res.n_pairs)
    np.testing.assert_allclose(ps[:, 1].sum(0), res.sum_gt, rtol=1e-12, atol=1e-12 * np.abs(res.sum_gt).max())
    # each patch's sums are the sums of its lenses' rows (lens_sums rows: d*w, g_t, g_x, w, K, n)
    for p in range(n_patch):
        rows = res.lens_sums[lab == p].sum(0)
        np.testing.assert_array_equal(rows[5], ps[p, 5])
        np.testing.assert_allclose(rows[1], ps[p, 1], rtol=1e-10, atol=1e-10 * np.abs(ps[p, 1]).max())
    # 5 lenses of every patch against the FP64 brute force over all sources
    rng = np.random.default_rng(33)
    idx = np.sort(np.concatenate([rng.choice(np.nonzero(lab == p)[0], 5, replace=False)
                                  for p in range(n_patch)]))
    can = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq, lens_idx=idx)
    check_lens_sums("config3 per-lens, 5 lenses in each of 100 patches, all 2 M sources", res.lens_sums[idx],
                    can)
    assert res.n_pairs.sum() > 5e10
    # resampling: same multiplicities (Philox) and the oracle's estimator
    boot = tpcf.block_bootstrap(ps, n_boot, seed=1003, ctx=ctx)
    mult = oracle.bootstrap_multiplicity(1003, n_boot, n_patch, n_patch)
    np.testing.assert_array_equal(boot["multiplicity"], mult)
    gt, gx, W = oracle.block_bootstrap(mult, ps[:, 1], ps[:, 2], ps[:, 4], ps[:, 3].sum(1))
    np.testing.assert_allclose(boot["g_t"][:, 0], gt, rtol=1e-12, atol=1e-15 * np.abs(gt).max())
    np.testing.assert_allclose(boot["g_x"][:, 0], gx, rtol=1e-12, atol=1e-15 * np.abs(gx).max())
    cov = oracle.covariance(gt)
    np.testing.assert_allclose(boot["cov_g_t"], cov, rtol=1e-9, atol=1e-12 * np.abs(cov).max())
    log_record({"case": "config3 pairs -> k-means -> bootstrap chain", "kmeans_labels_exact": True,
                "kmeans_iterations": int(it), "multiplicities_exact": True, "n_boot": n_boot,
                "binned_pairs": int(res.n_pairs.sum())})


def test_config4_gradients_fp64_and_finite_differences(tpcf, oracle, ctx, synth):
    w = synth.make_workload(4)
    L, S = w["lenses"], w["shapes"]
    bins = tpcf.create_bins(*w["bins"])
    nb = bins.n_bin
    lab, _, _ = tpcf.partition_data(L["x"], L["y"], _kmeans_weights(L), 100, ctx=ctx)
    fwd = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                     S["e1"], S["e2"], S["w"], S["m"], bins, patch_A=lab, n_patch=100,
                                     calculate_marks=False, lens_raw=True, ctx=ctx)
    # diagonal covariance from the block bootstrap, seeded target around xi
    boot = tpcf.block_bootstrap(fwd.patch_sums, 1000, seed=1004, covariance=False, ctx=ctx)
    sig = boot["g_t"][:, 0].std(0, ddof=1)
    xi = fwd.sum_gt / fwd.sum_K
    target = np.random.default_rng(1004).normal(xi, sig)
    lam = 2.0 * (xi - target) / sig ** 2                  # dL/dxi_t of L = sum ((xi - t)/sig)^2
    g = tpcf.tangential_shear_adjoint(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                      S["e1"], S["e2"], S["w"], S["m"], bins, fwd, lam, None, ctx=ctx)
    rng = np.random.default_rng(44)
    ls = np.sort(rng.choice(len(L["x"]), 500, replace=False))
    ss = np.sort(rng.choice(len(S["x"]), 500, replace=False))
    tot = (fwd.sum_gt, fwd.sum_gx, fwd.sum_K)
    ref = oracle.canon_adjoint_sel(L, S, bins.bin_edges_sq, tot, lam, None, ls, ss)
    rec = {"case": "config4 adjoint vs FP64 brute-force gradient, 500 lenses + 500 sources"}
    for k, sel in (("val_A", ls), ("w_A", ls), ("e1_B", ss), ("e2_B", ss), ("w_B", ss)):
        got, exp = g[k][sel], ref[k]
        scale = np.abs(exp).max()
        err = np.abs(got - exp)
        rec[k] = {"max_err_over_max": float(err.max() / scale),
                  "median_rel_err": float(np.median(err / (np.abs(exp) + 1e-300)))}
        assert np.all(err <= 1e-4 * scale + 1e-4 * np.abs(exp)), (k, err.max() / scale)
    log_record(rec)

    # central finite differences of the FP64 loss, step h = 1e-3, on the same
    # 1000 objects: the totals move by the object's own contribution, taken
    # from the FP64 brute force at the perturbed value (lenses: their rows are
    # linear in val_A and in w_A; sources: one oracle call per perturbed copy)
    h = 1e-3
    St, SK = fwd.sum_gt.astype(np.float64), fwd.sum_K.astype(np.float64)

    def dloss(dgt, dK):
        # L(S + d) - L(S) without cancellation: (xi' - xi)(xi' + xi - 2t)/sig^2
        x1 = (St + dgt) / (SK + dK)
        dx = (dgt * SK - St * dK) / (SK * (SK + dK))
        return float(np.sum(dx * (x1 + xi - 2 * target) / sig ** 2))

    can = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq, lens_idx=ls)
    rows = can["lens"]                                      # d*w, g_t, g_x, w, K, n
    fd, an = [], []
    for k, i in enumerate(ls):
        gt_i, K_i = rows[k, 1], rows[k, 4]
        v, wa = float(L["val"][i]), float(L["w"][i])
        if v != 0.0:   # g_t rows scale with val_A
            fd.append((dloss(gt_i * h / v, 0 * K_i) - dloss(-gt_i * h / v, 0 * K_i)) / (2 * h))
            an.append(g["val_A"][i])
        # every row scales with w_A
        fd.append((dloss(gt_i * h / wa, K_i * h / wa) - dloss(-gt_i * h / wa, -K_i * h / wa)) / (2 * h))
        an.append(g["w_A"][i])
    for j in ss:
        one = {q: S[q][j:j + 1].copy() for q in ("x", "y", "z", "e1", "e2", "w", "m")}
        base = oracle.canon_pairs(oracle.SHEAR, L, one, bins.bin_edges_sq)
        for q, key in (("e1", "e1_B"), ("e2", "e2_B")):
            vals = []
            for sgn in (1, -1):
                p = dict(one)
                p[q] = np.array([one[q][0] + sgn * h], np.float32)
                c = oracle.canon_pairs(oracle.SHEAR, L, p, bins.bin_edges_sq)
                vals.append((float(p[q][0]), dloss(c["sum_gt"] - base["sum_gt"], c["sum_K"] - base["sum_K"])))
            fd.append((vals[0][1] - vals[1][1]) / (vals[0][0] - vals[1][0]))
            an.append(g[key][j])
        wb = float(one["w"][0])   # every source row scales with w_B
        fd.append((dloss(base["sum_gt"] * h / wb, base["sum_K"] * h / wb)
                   - dloss(-base["sum_gt"] * h / wb, -base["sum_K"] * h / wb)) / (2 * h))
        an.append(g["w_B"][j])
    fd, an = np.array(fd), np.array(an)
    scale = np.abs(fd).max()
    err = np.abs(fd - an)
    log_record({"case": "config4 adjoint vs central FD (h = 1e-3) of the FP64 loss", "objects": 1000,
                "derivatives": int(len(fd)), "max_err_over_max": float(err.max() / scale),
                "median_rel_err": float(np.median(err / (np.abs(fd) + 1e-300)))})
    assert np.all(err <= 2e-3 * scale + 1e-3 * np.abs(fd)), err.max() / scale
