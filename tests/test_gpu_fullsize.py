"""Full-size checks on the 10.0 M-object tomography workload (5 shear bins x 5
scalar bins, 25 tasks, 100 patches, 20 log bins over 1-300 arcmin) and the
1 M-point scalar auto-correlation, through properties that hold at any size:

- per-lens parity in every one of the 25 tasks: the per-lens FP64 sums of 20
  random lenses per task, computed inside the full batched launch, against
  the oracle's FP64 brute force of those lenses over the task's whole source
  catalogue (n_pairs bit-exact, sums to 1e-6 of the lens's sum|terms| per
  bin; margins printed, tests/parity.py);
- the per-patch sums add up to the totals (n_pairs exactly);
- the batched launch equals single-task calls (n_pairs exactly);
- two shards add up to the unsharded result (n_pairs exactly, sums to 1e-12);
- linearity: doubling every lens value doubles the g_t and g_x sums exactly
  (the lens factor val*w enters in FP64, so a factor 2 is exact).
"""
import numpy as np
import pytest

from parity import check_lens_sums

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tomo(synth):
    return synth.make_workload(5)


def cats(tpcf, w):
    L = [tpcf.LensCatalog(**{k: l[k] for k in ("x", "y", "val", "w", "z")}) for l in w["lens_bins"]]
    S = [tpcf.ShapeCatalog(**{k: s[k] for k in ("x", "y", "e1", "e2", "w", "z", "m")}) for s in w["shape_bins"]]
    return L, S


def test_tomography_patches_batch_and_lens_parity(tpcf, oracle, tomo):
    import torch
    ctx = tpcf.Context(0)
    ctx.set_cell_size(tomo["bins"][1] / 64)
    bins = tpcf.create_bins(*tomo["bins"])
    L, S = cats(tpcf, tomo)
    ux = np.concatenate([l["x"] for l in tomo["lens_bins"]])
    uy = np.concatenate([l["y"] for l in tomo["lens_bins"]])
    uw = np.concatenate([l["w"] for l in tomo["lens_bins"]])
    lab, _, _ = tpcf.partition_data(ux, uy, (0.01 + uw / uw.max()).astype(np.float32), 100, ctx=ctx)
    offs = np.cumsum([0] + [len(l["x"]) for l in tomo["lens_bins"]])
    P = [lab[offs[i]:offs[i + 1]] for i in range(5)]
    # one 25-task launch with per-lens FP64 rows kept in device memory
    out = tpcf.batch_shear_2pcf(L, S, tomo["tasks"], bins, lens_patches=P, n_patch=100, lens_sums="device",
                                ctx=ctx)
    total = sum(int(o.n_pairs.sum()) for o in out)
    assert total > 1.0e12
    rng = np.random.default_rng(5)
    for t, (li, si) in enumerate(tomo["tasks"]):
        o = out[t]
        np.testing.assert_array_equal(o.patch_sums[:, 5].sum(0), o.n_pairs)
        np.testing.assert_allclose(o.patch_sums[:, 1].sum(0), o.sum_gt, rtol=1e-12, atol=1e-9)
        # 20 random lenses of this task against every source of its shear bin
        Ld, Sd = tomo["lens_bins"][li], tomo["shape_bins"][si]
        idx = np.sort(rng.choice(len(Ld["x"]), 20, replace=False))
        got = o.lens_sums.index_select(0, torch.as_tensor(idx, device=o.lens_sums.device)).cpu().numpy()
        can = oracle.canon_pairs(oracle.SHEAR, Ld, Sd, bins.bin_edges_sq, lens_idx=idx)
        check_lens_sums(f"config5 task {t} (scalar bin {li + 1} x shear bin {si + 1}), 20 lenses", got, can,
                        extra={"sources": int(len(Sd["x"]))})
        o.lens_sums = None
    # the same task launched alone (same patches and per-lens rows: the same
    # lens groups and FP32 fold interval) gives the batched launch's sums bit
    # for bit: the tasks of a batch do not interact
    t = tomo["tasks"].index((0, 4))
    alone = tpcf.batch_shear_2pcf([L[0]], [S[4]], [(0, 0)], bins, lens_patches=[P[0]], n_patch=100,
                                  lens_sums="device", ctx=ctx)[0]
    for q in ("n_pairs", "sum_gt", "sum_gx", "sum_w", "sum_K"):
        np.testing.assert_array_equal(getattr(alone, q), getattr(out[t], q))
    np.testing.assert_array_equal(alone.patch_sums, out[t].patch_sums)
    alone.lens_sums = None
    # the plain single call groups its lenses without patches and folds its
    # FP32 partials every 4096 sources instead of 1024: the same pairs, sums
    # that agree to the FP32 accumulation error
    Ld, Sd = tomo["lens_bins"][0], tomo["shape_bins"][4]
    one = tpcf.tangential_shear_tpcf(Ld["x"], Ld["y"], Ld["z"], Ld["val"], Ld["w"], Sd["x"], Sd["y"], Sd["z"],
                                     Sd["e1"], Sd["e2"], Sd["w"], Sd["m"], bins, calculate_marks=False, ctx=ctx)
    np.testing.assert_array_equal(one.n_pairs, out[t].n_pairs)
    np.testing.assert_allclose(one.sum_gt, out[t].sum_gt, rtol=1e-5, atol=1e-6 * np.abs(one.sum_gt).max())
    np.testing.assert_allclose(one.sum_w, out[t].sum_w, rtol=1e-6)
    ctx.close()


def test_tomography_shards_and_linearity(tpcf, tomo):
    bins = tpcf.create_bins(*tomo["bins"])
    L, S = cats(tpcf, tomo)
    tasks = tomo["tasks"][18:]  # the densest seven tasks
    full_ctx = tpcf.Context(0)
    full = tpcf.batch_shear_2pcf(L, S, tasks, bins, ctx=full_ctx)
    parts = []
    for r in range(2):
        c = tpcf.Context(0)
        c.set_shard(r, 2)
        parts.append(tpcf.batch_shear_2pcf(L, S, tasks, bins, ctx=c))
        c.close()
    for i, f in enumerate(full):
        np.testing.assert_array_equal(parts[0][i].n_pairs + parts[1][i].n_pairs, f.n_pairs)
        np.testing.assert_allclose(parts[0][i].sum_gt + parts[1][i].sum_gt, f.sum_gt, rtol=1e-12, atol=1e-9)
    L2 = [tpcf.LensCatalog(x=l.x, y=l.y, val=(2 * l.val).astype(np.float32), w=l.w, z=l.z) for l in L]
    dbl = tpcf.batch_shear_2pcf(L2, S, tasks, bins, ctx=full_ctx)
    for f, d in zip(full, dbl):
        np.testing.assert_array_equal(d.sum_gt, 2 * f.sum_gt)
        np.testing.assert_array_equal(d.sum_gx, 2 * f.sum_gx)
        np.testing.assert_array_equal(d.n_pairs, f.n_pairs)
    full_ctx.close()


def test_kappa_auto_1M_lens_parity(tpcf, oracle, synth):
    w = synth.make_workload(2)
    L, K = w["lenses"], w["kappa_map"]
    bins = tpcf.create_bins(*w["bins"])
    ctx = tpcf.Context(0)
    res = tpcf.scalar_kappa_tpcf(L["x"], L["y"], L["val"], L["w"], K["x"], K["y"], K["kappa_E"], K["kappa_B"],
                                 K["w"], bins, calculate_marks=False, lens_sums=True, ctx=ctx)
    assert res.n_pairs.sum() > 1e11
    idx = np.sort(np.random.default_rng(6).choice(len(L["x"]), 120, replace=False))
    can = oracle.canon_pairs(oracle.KAPPA, L, K, bins.bin_edges_sq, lens_idx=idx)
    check_lens_sums("config2 kappa-kappa 1M auto, 120 lenses", res.lens_sums[idx], can)
    ctx.close()
