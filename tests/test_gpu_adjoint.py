"""GPU checks of the adjoint (tpcf_shear_scalar_adjoint) and the
torch.autograd wrapper: against the FP64 brute-force gradient of the oracle,
and against central finite differences (step 1e-3, FP64 oracle loss) on 1000
random objects.

Tolerance: FP32 pair arithmetic with FP64 accumulation, so each gradient is
compared relative to the largest gradient of its kind: 1e-4 of max|g| (the
bar of the FP32 per-pair products) plus 1e-4 of |g| itself."""
import importlib

import numpy as np
import pytest

from conftest import uniform_shear

pytestmark = pytest.mark.gpu


def catalogue(n_lens, n_src, box, seed):
    L, S = uniform_shear(n_lens, n_src, box, seed, w="uniform")
    rng = np.random.default_rng(seed + 1)
    S["m"][:] = rng.normal(0, 0.05, n_src).astype(np.float32)
    return L, S


def close(got, ref, rtol=1e-4, name=""):
    scale = np.abs(ref).max() + 1e-300
    bad = np.abs(got - ref) > rtol * scale + rtol * np.abs(ref)
    assert not bad.any(), (name, np.nonzero(bad)[0][:10], got[bad][:5], ref[bad][:5])


def forward_and_adjoint(tpcf, ctx, L, S, bins, lt, lx):
    fwd = tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                     S["e1"], S["e2"], S["w"], S["m"], bins, calculate_marks=False,
                                     lens_raw=True, ctx=ctx)
    g = tpcf.tangential_shear_adjoint(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                      S["e1"], S["e2"], S["w"], S["m"], bins, fwd, lt, lx, ctx=ctx)
    return fwd, g


def test_adjoint_matches_fp64_bruteforce_gradient(tpcf, oracle, ctx):
    L, S = catalogue(3000, 4000, 300.0, 60)
    bins = tpcf.create_bins(1.0, 80.0, 12)
    rng = np.random.default_rng(61)
    lt, lx = rng.normal(size=12), rng.normal(size=12)
    _, g = forward_and_adjoint(tpcf, ctx, L, S, bins, lt, lx)
    ref = oracle.canon_adjoint(L, S, bins.bin_edges_sq, lt, lx)
    for k in ("val_A", "w_A", "e1_B", "e2_B", "w_B", "m_B"):
        close(g[k], ref[k], name=k)


def test_adjoint_with_z_cut_and_generic_spacing(tpcf, oracle, ctx):
    L, S = catalogue(1500, 2000, 200.0, 62)
    rng = np.random.default_rng(63)
    L["z"][:] = rng.uniform(0, 1, 1500).astype(np.float32)
    S["z"][:] = rng.uniform(-0.1, 1.2, 2000).astype(np.float32)
    bins = tpcf.create_bins(0.5, 50.0, 9, spacing="sqrt")
    lt = rng.normal(size=9)
    _, g = forward_and_adjoint(tpcf, ctx, L, S, bins, lt, None)
    ref = oracle.canon_adjoint(L, S, bins.bin_edges_sq, lt, None)
    for k in ("val_A", "w_A", "e1_B", "e2_B", "w_B", "m_B"):
        close(g[k], ref[k], name=k)


def test_adjoint_central_finite_differences(tpcf, oracle, ctx):
    """Central FD (step 1e-3 on the FP32 inputs, loss in FP64 by the oracle) on
    1000 random objects."""
    L, S = catalogue(500, 700, 150.0, 64)
    bins = tpcf.create_bins(1.0, 60.0, 8)
    rng = np.random.default_rng(65)
    lt, lx = rng.normal(size=8), rng.normal(size=8)
    _, g = forward_and_adjoint(tpcf, ctx, L, S, bins, lt, lx)

    def loss(Lc, Sc):
        c = oracle.canon_pairs(oracle.SHEAR, Lc, Sc, bins.bin_edges_sq)
        K = c["sum_K"]
        xt = np.where(K > 0, c["sum_gt"] / np.where(K > 0, K, 1), 0)
        xx = np.where(K > 0, c["sum_gx"] / np.where(K > 0, K, 1), 0)
        return float(lt @ xt + lx @ xx)

    picks = [("lens", k, i) for k in ("val", "w") for i in rng.choice(500, 125, replace=False)]
    picks += [("src", k, i) for k in ("e1", "e2", "w", "m") for i in rng.choice(700, 188, replace=False)]
    key = {"val": "val_A", "w": None, "e1": "e1_B", "e2": "e2_B", "m": "m_B"}
    fd, an = [], []
    for side, k, i in picks[:1000]:
        cat = L if side == "lens" else S
        x0 = cat[k][i]
        vals = []
        for sgn in (1, -1):
            cat[k][i] = np.float32(x0 + sgn * 1e-3)
            vals.append((cat[k][i], loss(L, S)))
        cat[k][i] = x0
        fd.append((vals[0][1] - vals[1][1]) / (float(vals[0][0]) - float(vals[1][0])))
        name = key[k] if k != "w" else ("w_A" if side == "lens" else "w_B")
        an.append(float(g[name][i]))
    fd, an = np.array(fd), np.array(an)
    scale = np.abs(fd).max()
    assert np.all(np.abs(fd - an) <= 2e-3 * scale + 1e-3 * np.abs(fd)), np.max(np.abs(fd - an) / scale)


def test_autograd_chi2_loss(tpcf, oracle):
    import torch
    ag = importlib.import_module("2pcf_b200.autograd")
    L, S = catalogue(2000, 3000, 250.0, 66)
    bins = tpcf.create_bins(1.0, 70.0, 10)
    d = lambda a: torch.from_numpy(a).cuda()
    geo = dict(x_A=d(L["x"]), y_A=d(L["y"]), z_A=d(L["z"]), x_B=d(S["x"]), y_B=d(S["y"]), z_B=d(S["z"]),
               m_B=d(S["m"]))
    leaves = [d(a).requires_grad_(True) for a in (L["val"], L["w"], S["e1"], S["e2"], S["w"])]
    xi_t, xi_x = ag.xi_shear(*leaves, geo, bins)
    rng = np.random.default_rng(67)
    target = torch.from_numpy(rng.normal(0, 1e-4, 10)).cuda()
    sigma = torch.full((10,), 1e-3, dtype=torch.float64, device="cuda")
    loss = (((xi_t - target) / sigma) ** 2).sum()
    loss.backward()
    lt = (2 * (xi_t - target) / sigma ** 2).detach().cpu().numpy()
    ref = oracle.canon_adjoint(L, S, bins.bin_edges_sq, lt, None)
    for leaf, k in zip(leaves, ("val_A", "w_A", "e1_B", "e2_B", "w_B")):
        close(leaf.grad.cpu().numpy(), ref[k], name=k)
    can = oracle.normalise(oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq))
    np.testing.assert_allclose(xi_t.detach().cpu().numpy(), can["g_t"], rtol=1e-5, atol=1e-9)


def test_batched_autograd_equals_per_task(tpcf, oracle):
    """xi_shear_batch (one forward launch for all tasks) gives the values and
    gradients of per-task xi_shear calls; a catalogue used by two tasks gets
    the sum of its gradients."""
    import torch
    ag = importlib.import_module("2pcf_b200.autograd")
    cats = [catalogue(1500, 2000, 200.0, 70 + k) for k in range(2)]
    bins = tpcf.create_bins(1.0, 60.0, 8)
    d = lambda a: torch.from_numpy(a).cuda()
    geo_L = [dict(x=d(L["x"]), y=d(L["y"]), z=d(L["z"])) for L, _ in cats]
    geo_S = [dict(x=d(S["x"]), y=d(S["y"]), z=d(S["z"]), m=d(S["m"])) for _, S in cats]
    tasks = [(0, 0), (0, 1), (1, 1)]
    leaves = lambda: ([d(L["val"]).requires_grad_(True) for L, _ in cats], [d(L["w"]).requires_grad_(True) for L, _ in cats],
                      [d(S["e1"]).requires_grad_(True) for _, S in cats], [d(S["e2"]).requires_grad_(True) for _, S in cats],
                      [d(S["w"]).requires_grad_(True) for _, S in cats])
    v, wa, e1, e2, wb = leaves()
    xt, xx = ag.xi_shear_batch(tasks, geo_L, geo_S, v, wa, e1, e2, wb, bins)
    rng = np.random.default_rng(71)
    ct = torch.from_numpy(rng.normal(size=(3, 8))).cuda()
    cx = torch.from_numpy(rng.normal(size=(3, 8))).cuda()
    ((xt * ct).sum() + (xx * cx).sum()).backward()
    v2, wa2, e12, e22, wb2 = leaves()
    loss = 0
    for t, (li, si) in enumerate(tasks):
        geo = dict(x_A=geo_L[li]["x"], y_A=geo_L[li]["y"], z_A=geo_L[li]["z"], x_B=geo_S[si]["x"],
                   y_B=geo_S[si]["y"], z_B=geo_S[si]["z"], m_B=geo_S[si]["m"])
        a, b = ag.xi_shear(v2[li], wa2[li], e12[si], e22[si], wb2[si], geo, bins)
        np.testing.assert_array_equal(a.detach().cpu().numpy(), xt[t].detach().cpu().numpy())
        loss = loss + (a * ct[t]).sum() + (b * cx[t]).sum()
    loss.backward()
    for p1, p2 in zip(v + wa + e1 + e2 + wb, v2 + wa2 + e12 + e22 + wb2):
        close(p1.grad.cpu().numpy(), p2.grad.cpu().numpy(), rtol=1e-6, name="batched grad")
