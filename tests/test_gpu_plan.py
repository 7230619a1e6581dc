"""Prepared batches (tpcf_plan_shear_scalar): a plan launched directly, and
its launch recorded into a CUDA graph and replayed, give the sums of the
plain batched call bit for bit; the context the plan was made from stays
usable meanwhile."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

QS = ("n_pairs", "sum_dw", "sum_gt", "sum_gx", "sum_w", "sum_K", "g_t", "g_x", "mean_theta", "weights")


def catalogues(tpcf, rng, n_lens, n_src, box, device):
    import torch
    dev = (lambda a: torch.from_numpy(a).cuda()) if device else (lambda a: a)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    L = tpcf.LensCatalog(x=dev(f32(rng.uniform(0, box, n_lens))), y=dev(f32(rng.uniform(0, box, n_lens))),
                         val=dev(f32(rng.normal(0, 0.02, n_lens))), w=dev(f32(rng.uniform(0.5, 1.5, n_lens))),
                         z=dev(f32(rng.uniform(0, 0.5, n_lens))))
    S = tpcf.ShapeCatalog(x=dev(f32(rng.uniform(0, box, n_src))), y=dev(f32(rng.uniform(0, box, n_src))),
                          e1=dev(f32(rng.normal(0, 0.26, n_src))), e2=dev(f32(rng.normal(0, 0.26, n_src))),
                          w=dev(f32(rng.uniform(0.5, 1.5, n_src))), z=dev(f32(rng.uniform(0.3, 1.2, n_src))),
                          m=dev(f32(rng.normal(0, 0.02, n_src))))
    return L, S


def same(a, b):
    for x, y in zip(a, b):
        for q in QS:
            np.testing.assert_array_equal(getattr(x, q), getattr(y, q), err_msg=q)
        if x.patch_sums is not None:
            np.testing.assert_array_equal(x.patch_sums, y.patch_sums)


@pytest.mark.parametrize("device", [False, True])
def test_plan_and_graph_replay_match_the_batched_call(tpcf, device):
    import torch
    rng = np.random.default_rng(31)
    L0, S0 = catalogues(tpcf, rng, 30_000, 60_000, 300.0, device)
    L1, S1 = catalogues(tpcf, rng, 20_000, 80_000, 300.0, device)
    tasks = [(0, 0), (0, 1), (1, 1), (1, 0)]
    bins = tpcf.create_bins(1.0, 60.0, 12)
    patches = [rng.integers(0, 7, 30_000).astype(np.int32), rng.integers(0, 7, 20_000).astype(np.int32)]
    ctx = tpcf.Context(0)
    ctx.set_cell_size(60.0 / 24)
    direct = tpcf.batch_shear_2pcf([L0, L1], [S0, S1], tasks, bins, lens_patches=patches, n_patch=7, ctx=ctx)
    plan = tpcf.BatchPlan([L0, L1], [S0, S1], tasks, bins, lens_patches=patches, n_patch=7, ctx=ctx)
    plan.launch()
    same(plan.results(), direct)
    plan.launch()  # a second launch clears the queue itself
    same(plan.results(), direct)
    # the plan keeps its own workspace: the context serves other calls meanwhile
    other = tpcf.batch_shear_2pcf([L1], [S0], [(0, 0)], bins, ctx=ctx)
    assert other[0].n_pairs.sum() > 0
    g = plan.capture()
    same(plan.results(), direct)  # the warm-up launch of the capture
    for _ in range(3):
        g.replay()
        torch.cuda.synchronize()
        same(plan.results(), direct)
    del g
    plan.close()
    ctx.close()


def test_plan_per_lens_rows_and_misuse(tpcf):
    rng = np.random.default_rng(32)
    L0, S0 = catalogues(tpcf, rng, 10_000, 30_000, 200.0, True)
    bins = tpcf.create_bins(1.0, 40.0, 10)
    ctx = tpcf.Context(0)
    direct = tpcf.batch_shear_2pcf([L0], [S0], [(0, 0)], bins, lens_sums=True, ctx=ctx)
    plan = tpcf.BatchPlan([L0], [S0], [(0, 0)], bins, lens_sums=True, ctx=ctx)
    plan.launch()
    got = plan.results()
    same(got, direct)
    np.testing.assert_array_equal(got[0].lens_sums, direct[0].lens_sums)
    plan.close()
    ctx.set_spherical(True)
    with pytest.raises(tpcf.TPCFError):
        tpcf.BatchPlan([L0], [S0], [(0, 0)], bins, ctx=ctx)
    ctx.close()
