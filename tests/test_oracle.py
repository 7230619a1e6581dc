"""CPU tests of the oracle: the reference's own pinned behaviour, the golden
fixtures, known answers, and agreement between the FP32 restatement of the
reference loop and the canonical FP64 rule.  No GPU needed."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, f"{name}.npz")))


def split(d, prefix):
    return {k[len(prefix):]: v for k, v in d.items() if k.startswith(prefix)}


# -------------------------------------------------- pinned by the reference --
def test_kdtree_search_equals_brute_force(oracle):
    """src/test_kdtree.f90:96-104: the tree search returns the same sorted index
    set as the brute-force scan (100k uniform points, leafsize 10)."""
    rng = np.random.default_rng(100)
    n = 100_000
    x = (rng.random(n) * 2 * np.pi).astype(np.float32)
    y = (-np.pi / 2 + rng.random(n) * np.pi).astype(np.float32)
    queries = [(2.5, 0.25, 1.1)] + [(rng.uniform(0, 6.3), rng.uniform(-1.5, 1.5), rng.uniform(0.01, 0.8))
                                    for _ in range(20)]
    for qx, qy, r in queries:
        a = np.sort(oracle.kdtree_search(x, y, (qx, qy), r))
        b = np.sort(oracle.kdtree_search(x, y, (qx, qy), r, brute_force=True))
        np.testing.assert_array_equal(a, b)


# ------------------------------------------------------------ golden files --
def test_golden_shear(oracle):
    g = load("shear_small")
    L, S = split(g, "L_"), split(g, "S_")
    lo, hi, nb = g["bins"]
    can = oracle.canon_pairs(oracle.SHEAR, L, S, g["edges_sq"], num_threads=3)
    pinned = [k for k in oracle.CANON_Q if f"canon_{k}" in g]
    assert len(pinned) >= 8
    for k in pinned:
        np.testing.assert_array_equal(can[k], g[f"canon_{k}"])
    ref = oracle.ref_pairs(oracle.SHEAR, L, S, lo, hi, int(nb), num_threads=1, marks=True)
    for k, v in ref.items():
        np.testing.assert_array_equal(v, g[f"ref_{k}"])


def test_golden_kappa(oracle):
    g = load("kappa_small")
    L, K = split(g, "L_"), split(g, "K_")
    lo, hi, nb = g["bins"]
    can = oracle.canon_pairs(oracle.KAPPA, L, K, g["edges_sq"], num_threads=2)
    pinned = [k for k in oracle.CANON_Q if f"canon_{k}" in g]
    assert len(pinned) >= 8
    for k in pinned:
        np.testing.assert_array_equal(can[k], g[f"canon_{k}"])
    ref = oracle.ref_pairs(oracle.KAPPA, L, K, lo, hi, int(nb), num_threads=1)
    for k, v in ref.items():
        np.testing.assert_array_equal(v, g[f"ref_{k}"])


def test_golden_kmeans(oracle):
    g = load("kmeans_small")
    lab, cen, it = oracle.kmeans_det(g["x"], g["y"], g["w"], int(g["k"]))
    np.testing.assert_array_equal(lab, g["det_labels"])
    np.testing.assert_array_equal(cen, g["det_centroids"])
    lab, cen, it = oracle.kmeans_ref_f32(g["x"], g["y"], g["w"], int(g["k"]))
    np.testing.assert_array_equal(lab, g["ref_labels"])


def test_golden_bootstrap(oracle):
    g = load("bootstrap_small")
    mult = oracle.bootstrap_multiplicity(int(g["seed"]), *g["mult"].shape, g["mult"].shape[1])
    np.testing.assert_array_equal(mult, g["mult"])
    gt, gx, W = oracle.block_bootstrap(mult, g["St"], g["Sx"], g["SK"], g["Sw"])
    np.testing.assert_array_equal(gt, g["gt"])
    np.testing.assert_array_equal(oracle.covariance(gt), g["cov_gt"])


# -------------------------------------------- reference restatement vs rule --
def test_fp32_restatement_agrees_with_canonical_rule(oracle):
    """The reference bins in FP32 (sqrt, log10, int); the canonical rule bins the
    FP64 d^2 against FP64 squared edges.  They may differ only for pairs within
    FP32 rounding of an edge: count those."""
    g = load("shear_small")
    L, S = split(g, "L_"), split(g, "S_")
    ref_np = g["ref_n_pairs"]
    can_np = g["canon_n_pairs"].astype(np.int64)
    moved = np.abs(ref_np - can_np).sum()
    assert moved <= 4, (ref_np, can_np)
    # the FP64 build of the reference loop agrees exactly on random data
    lo, hi, nb = g["bins"]
    ref64 = oracle.ref_pairs(oracle.SHEAR, L, S, lo, hi, int(nb), num_threads=2, dtype=np.float64)
    np.testing.assert_array_equal(ref64["n_pairs"], can_np)
    K = g["canon_sum_K"]
    np.testing.assert_allclose(ref64["g_t"], np.where(K > 0, g["canon_sum_gt"] / K, 0), rtol=1e-10, atol=1e-16)


def test_kd_tree_and_all_pairs_restatement_agree(oracle):
    g = load("kappa_small")
    L, K = split(g, "L_"), split(g, "K_")
    lo, hi, nb = g["bins"]
    a = oracle.ref_pairs(oracle.KAPPA, L, K, lo, hi, int(nb), use_kd_tree=True)
    b = oracle.ref_pairs(oracle.KAPPA, L, K, lo, hi, int(nb), use_kd_tree=False)
    np.testing.assert_array_equal(a["n_pairs"], b["n_pairs"])


def test_find_bin_index_reference_semantics(oracle):
    # x < x_min or x > x_max -> none; x == x_max -> last bin (src/utils.f90:109-115)
    d = np.array([0.5, 1.0, 1.5, 99.9, 100.0, 100.1], np.float32)
    np.testing.assert_array_equal(oracle.find_bin_f32(d, 1.0, 100.0, 2), [-1, 0, 0, 1, 1, -1])
    e2 = oracle.canonical_edges(1.0, 100.0, 2)[1]
    np.testing.assert_array_equal(oracle.canonical_bin(d.astype(np.float64) ** 2, e2), [-1, 0, 0, 1, 1, -1])


# --------------------------------------------------------------- analytic ----
def test_pure_tangential_shear_known_answer(oracle):
    """Sources on rings around one lens with e = -gamma (cos 2phi, sin 2phi):
    g_t = gamma exactly and g_x = 0 (the estimator of src/tpcf.f90:343-352)."""
    gamma = 0.05
    r = np.repeat(np.geomspace(1.5, 90, 40), 36)
    phi = np.tile(np.linspace(0, 2 * np.pi, 36, endpoint=False), 40)
    n = r.size
    S = dict(x=(r * np.cos(phi)).astype(np.float32), y=(r * np.sin(phi)).astype(np.float32),
             z=np.ones(n, np.float32), w=np.ones(n, np.float32), m=np.zeros(n, np.float32))
    dx, dy = -S["x"].astype(np.float64), -S["y"].astype(np.float64)  # lens minus source
    ang = np.arctan2(dy, dx)
    S["e1"] = (-gamma * np.cos(2 * ang)).astype(np.float32)
    S["e2"] = (-gamma * np.sin(2 * ang)).astype(np.float32)
    L = dict(x=np.zeros(1, np.float32), y=np.zeros(1, np.float32), z=np.zeros(1, np.float32),
             val=np.ones(1, np.float32), w=np.ones(1, np.float32))
    _, e2 = oracle.canonical_edges(1.0, 100.0, 10)
    c = oracle.normalise(oracle.canon_pairs(oracle.SHEAR, L, S, e2))
    np.testing.assert_allclose(c["g_t"], gamma, rtol=1e-6)
    np.testing.assert_allclose(c["g_x"], 0, atol=1e-7)
    ref = oracle.ref_pairs(oracle.SHEAR, L, S, 1.0, 100.0, 10)
    np.testing.assert_allclose(ref["g_t"], gamma, rtol=1e-5)


def test_constant_kappa_known_answer(oracle):
    rng = np.random.default_rng(5)
    n = 3000
    L = dict(x=rng.uniform(0, 100, n).astype(np.float32), y=rng.uniform(0, 100, n).astype(np.float32),
             val=np.full(n, 2.0, np.float32), w=rng.uniform(0.5, 1.5, n).astype(np.float32))
    K = dict(x=rng.uniform(0, 100, n).astype(np.float32), y=rng.uniform(0, 100, n).astype(np.float32),
             kappa_E=np.full(n, 0.25, np.float32), kappa_B=np.zeros(n, np.float32),
             w=rng.uniform(0.5, 1.5, n).astype(np.float32))
    _, e2 = oracle.canonical_edges(1.0, 50.0, 8)
    c = oracle.normalise(oracle.canon_pairs(oracle.KAPPA, L, K, e2))
    np.testing.assert_allclose(c["g_t"], 0.5, rtol=1e-12)


# --------------------------------------------------------- RNG / bootstrap --
def test_philox_known_answer_vectors(oracle):
    """Random123 known-answer vectors of Philox4x32-10."""
    kat = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
           ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
           ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, want in kat:
        np.testing.assert_array_equal(oracle.philox4x32(ctr, key), np.array(want, np.uint32))


def test_bootstrap_identity_and_covariance(oracle):
    rng = np.random.default_rng(6)
    St, Sx = rng.normal(size=(10, 5)), rng.normal(size=(10, 5))
    SK, Sw = rng.uniform(1, 2, (10, 5)), rng.uniform(1, 2, 10)
    mult = np.ones((3, 10), np.int32)          # every patch exactly once
    gt, gx, W = oracle.block_bootstrap(mult, St, Sx, SK, Sw)
    np.testing.assert_allclose(gt, np.broadcast_to(St.sum(0) / SK.sum(0), gt.shape), rtol=1e-14)
    np.testing.assert_allclose(W, Sw.sum(), rtol=1e-14)
    x = rng.normal(size=(200, 6))
    np.testing.assert_allclose(oracle.covariance(x), np.cov(x, rowvar=False, ddof=1), rtol=1e-12)
    m = oracle.bootstrap_multiplicity(7, 50, 13, 13)
    assert np.all(m.sum(1) == 13)


def test_kmeans_deterministic_vs_reference_fraction(oracle):
    """The deterministic (fixed-point) Lloyd iteration and the FP32-serial
    restatement of partition_data agree on all but a tiny fraction of labels."""
    g = load("kmeans_small")
    agree = np.mean(g["det_labels"] == g["ref_labels"])
    assert agree > 0.99
    assert len(np.unique(g["det_labels"])) == int(g["k"])


def test_equal_weight_kmeans_restatement_balances(oracle):
    """The equal-weight restatement gives valid labels, cluster weights that
    match its reported deviation, and a much smaller spread than plain k-means."""
    rng = np.random.default_rng(7)
    n = 20000
    x = np.concatenate([rng.normal(0, 5, n // 2), rng.uniform(0, 100, n // 2)]).astype(np.float32)
    y = np.concatenate([rng.normal(0, 5, n // 2), rng.uniform(0, 100, n // 2)]).astype(np.float32)
    w = rng.uniform(0.5, 1.5, n).astype(np.float32)
    lab, cen, it, dev = oracle.kmeans_equal(x, y, w, 20, random_init=False)
    assert lab.min() >= 0 and lab.max() < 20
    W = np.bincount(lab, weights=w.astype(np.float64), minlength=20)
    assert abs((W.max() - W.min()) / W.mean() - dev) < 1e-5
    _, _, _, dev0 = oracle.kmeans_equal(x, y, w, 20, scaling=0.0, weight_tol=1e9, random_init=False)
    assert dev < 0.3 * dev0


def test_subset_adjoint_equals_full_adjoint(oracle):
    """canon_adjoint_sel (gradients of selected objects from given totals, used
    at full sizes) equals the full brute-force gradient on those objects."""
    rng = np.random.default_rng(1)
    n = 400
    f = lambda a: np.ascontiguousarray(a, np.float32)
    L = dict(x=f(rng.uniform(0, 100, n)), y=f(rng.uniform(0, 100, n)), z=f(rng.uniform(0, 1, n)),
             val=f(rng.normal(0, 1, n)), w=f(rng.uniform(.5, 1.5, n)))
    S = dict(x=f(rng.uniform(0, 100, n)), y=f(rng.uniform(0, 100, n)), z=f(rng.uniform(0.2, 1.2, n)),
             e1=f(rng.normal(0, .3, n)), e2=f(rng.normal(0, .3, n)), w=f(rng.uniform(.5, 1.5, n)),
             m=f(rng.normal(0, .05, n)))
    _, e2 = oracle.canonical_edges(1.0, 50.0, 8)
    lt, lx = rng.normal(size=8), rng.normal(size=8)
    full = oracle.canon_adjoint(L, S, e2, lt, lx)
    c = oracle.canon_pairs(oracle.SHEAR, L, S, e2)
    ls, ss = np.array([3, 50, 399]), np.array([0, 7, 123, 250])
    sel = oracle.canon_adjoint_sel(L, S, e2, (c["sum_gt"], c["sum_gx"], c["sum_K"]), lt, lx, ls, ss)
    for k, idx in (("val_A", ls), ("w_A", ls), ("e1_B", ss), ("e2_B", ss), ("w_B", ss), ("m_B", ss)):
        np.testing.assert_allclose(sel[k], full[k][idx], rtol=1e-12, atol=1e-15 * np.abs(full[k]).max())
