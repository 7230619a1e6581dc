"""GPU parity of the spherical pair kernels (spherical_coords, src/tpcf.f90:297-359)
against the canonical spherical oracle, through the C ABI.

Bar (as for the planar kernels): n_pairs bit-exact with the canonical FP64 rule
(squared chords of the unit vectors against (2 sin(e/2))^2); every FP64 sum
within RTOL = 1e-6 of the oracle relative to the sum of |terms| of its bin;
unit vectors bit-exact with the oracle's.
"""
import numpy as np
import pytest

from test_gpu_pairs import assert_parity

pytestmark = pytest.mark.gpu

D2R = np.pi / 180.0
ARCMIN = D2R / 60.0


def f32(a):
    return np.ascontiguousarray(a, np.float32)


@pytest.fixture(scope="module")
def sctx(tpcf):
    c = tpcf.Context(0)
    yield c
    c.close()


def cap(rng, n, lam0, lam1, phi0, phi1):
    lam = rng.uniform(lam0, lam1, n) * D2R
    phi = np.arcsin(rng.uniform(np.sin(phi0 * D2R), np.sin(phi1 * D2R), n))
    return f32(lam), f32(phi)


def shear_cats(rng, nL, nS, box, w="ones"):
    xa, ya = cap(rng, nL, *box)
    xb, yb = cap(rng, nS, *box)
    wl = np.ones(nL) if w == "ones" else rng.uniform(0.5, 1.5, nL)
    ws = np.ones(nS) if w == "ones" else rng.uniform(0.5, 1.5, nS)
    L = dict(x=xa, y=ya, z=f32(np.zeros(nL)), val=f32(rng.normal(0, 0.02, nL)), w=f32(wl))
    S = dict(x=xb, y=yb, z=f32(np.ones(nS)), e1=f32(rng.normal(0, 0.26, nS)), e2=f32(rng.normal(0, 0.26, nS)),
             w=f32(ws), m=f32(np.zeros(nS)))
    return L, S


def run_shear(tpcf, ctx, L, S, bins, **kw):
    return tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                      S["e1"], S["e2"], S["w"], S["m"], bins, spherical_coords=True,
                                      ctx=ctx, **kw)


def test_unit_vectors_bit_exact(tpcf, oracle, sctx):
    rng = np.random.default_rng(1)
    lam = f32(rng.uniform(-7, 13, 200000))
    phi = f32(rng.uniform(-1.5707964, 1.5707964, 200000))
    hi, lo = tpcf.unit_vectors(lam, phi, ctx=sctx)
    ohi, olo = oracle.unit_vectors(lam, phi)
    np.testing.assert_array_equal(hi, ohi)
    np.testing.assert_array_equal(lo, olo)


def test_shear_patch_log_bins(tpcf, oracle, sctx):
    """KiDS-like patch away from the equator, 1'..100' log bins (series path)."""
    rng = np.random.default_rng(2)
    L, S = shear_cats(rng, 5000, 7000, (35, 47, -36, -26), w="uniform")
    bins = tpcf.create_bins(1 * ARCMIN, 100 * ARCMIN, 15)
    res = run_shear(tpcf, sctx, L, S, bins)
    can = oracle.canon_sphere(oracle.SHEAR, L, S, bins.chord_edges_sq)
    assert_parity(res, can)
    assert res.n_pairs.sum() > 100000
    np.testing.assert_allclose(res.mean_theta, oracle.normalise(can)["mean_theta"], rtol=1e-6)


def test_shear_generic_spacing_z_cut_and_m(tpcf, oracle, sctx):
    rng = np.random.default_rng(3)
    L, S = shear_cats(rng, 3000, 4000, (100, 108, 10, 17), w="uniform")
    L["z"][:] = f32(rng.uniform(-0.1, 1.0, 3000))
    S["z"][:] = f32(rng.uniform(-0.1, 1.2, 4000))
    S["m"][:] = f32(rng.normal(0, 0.05, 4000))
    L["w"][rng.random(3000) < 0.05] = 0.0
    for sp in ("lin", "sqrt"):
        bins = tpcf.create_bins(2 * ARCMIN, 80 * ARCMIN, 11, spacing=sp)
        res = run_shear(tpcf, sctx, L, S, bins)
        assert_parity(res, oracle.canon_sphere(oracle.SHEAR, L, S, bins.chord_edges_sq))


def test_poles_wrap_and_wide_bins(tpcf, oracle, sctx):
    """Whole-sky sparse catalogues with negative longitudes, longitudes past
    2 pi and points at the poles; bins up to 40 degrees (asin path, chords
    above 0.25)."""
    rng = np.random.default_rng(4)
    n = 3000
    L = dict(x=f32(rng.uniform(-np.pi, 3 * np.pi, n)), y=f32(np.arcsin(rng.uniform(-1, 1, n))),
             z=f32(np.zeros(n)), val=f32(rng.normal(0, 0.02, n)), w=f32(np.ones(n)))
    S = dict(x=f32(rng.uniform(-np.pi, 3 * np.pi, n)), y=f32(np.arcsin(rng.uniform(-1, 1, n))),
             z=f32(np.ones(n)), e1=f32(rng.normal(0, 0.26, n)), e2=f32(rng.normal(0, 0.26, n)),
             w=f32(np.ones(n)), m=f32(np.zeros(n)))
    L["y"][:5] = f32([np.pi / 2, -np.pi / 2, 1.5707, -1.5707, 1.57079])
    S["y"][:5] = f32([np.pi / 2, -np.pi / 2, 1.5706, -1.57079, 1.57])
    S["x"][5:20] = f32(np.linspace(-1e-3, 1e-3, 15))        # straddle lambda = 0
    L["x"][5:20] = f32(2 * np.pi - np.linspace(0, 2e-3, 15))
    for lo, hi, nb, sp in ((1 * D2R, 40 * D2R, 12, "log"), (0.0, 30 * D2R, 10, "lin")):
        bins = tpcf.create_bins(lo, hi, nb, spacing=sp)
        res = run_shear(tpcf, sctx, L, S, bins)
        assert_parity(res, oracle.canon_sphere(oracle.SHEAR, L, S, bins.chord_edges_sq))


def test_kappa_patch(tpcf, oracle, sctx):
    rng = np.random.default_rng(5)
    n = 5000
    xa, ya = cap(rng, n, 200, 210, 50, 58)
    xb, yb = cap(rng, n, 200, 210, 50, 58)
    L = dict(x=xa, y=ya, val=f32(rng.normal(0, 0.02, n)), w=f32(rng.uniform(0.5, 1.5, n)))
    K = dict(x=xb, y=yb, kappa_E=f32(rng.normal(0, 0.02, n)), kappa_B=f32(rng.normal(0, 0.01, n)),
             w=f32(rng.uniform(0.5, 1.5, n)))
    bins = tpcf.create_bins(0.5 * ARCMIN, 60 * ARCMIN, 20)
    res = tpcf.scalar_kappa_tpcf(L["x"], L["y"], L["val"], L["w"], K["x"], K["y"], K["kappa_E"], K["kappa_B"],
                                 K["w"], bins, spherical_coords=True, ctx=sctx)
    assert_parity(res, oracle.canon_sphere(oracle.KAPPA, L, K, bins.chord_edges_sq))


def test_all_pairs_equals_grid_and_marks(tpcf, oracle, sctx):
    rng = np.random.default_rng(6)
    L, S = shear_cats(rng, 1500, 2500, (10, 16, -5, 3))
    bins = tpcf.create_bins(1 * ARCMIN, 90 * ARCMIN, 10)
    g = run_shear(tpcf, sctx, L, S, bins, calculate_marks=True)
    brute = tpcf.Context(0, use_grid=False)
    try:
        a = run_shear(tpcf, brute, L, S, bins, calculate_marks=True)
    finally:
        brute.close()
    can = oracle.canon_sphere(oracle.SHEAR, L, S, bins.chord_edges_sq)
    assert_parity(a, can)
    assert_parity(g, can)
    # per-lens marks (FP32 per lens) sum to the totals
    scale = np.abs(g.xi_E_marks).sum(0, dtype=np.float64)
    assert np.all(np.abs(g.xi_E_marks.sum(0, dtype=np.float64) - g.sum_gt) <= 1e-6 * scale + 1e-12)
    np.testing.assert_allclose(g.w_marks.sum(0, dtype=np.float64), g.sum_w, rtol=1e-6)


def test_batch_with_patches_matches_oracle(tpcf, oracle, sctx):
    rng = np.random.default_rng(7)
    box = (300, 310, -12, -4)
    lens, shapes = [], []
    for _ in range(2):
        L, S = shear_cats(rng, 2000, 3000, box)
        lens.append(tpcf.LensCatalog(x=L["x"], y=L["y"], z=L["z"], val=L["val"], w=L["w"]))
        shapes.append(tpcf.ShapeCatalog(x=S["x"], y=S["y"], z=S["z"], e1=S["e1"], e2=S["e2"], w=S["w"],
                                        m=S["m"]))
    bins = tpcf.create_bins(1 * ARCMIN, 60 * ARCMIN, 8)
    tasks = [(0, 0), (0, 1), (1, 1)]
    patches = [(np.arange(2000) % 5).astype(np.int32) for _ in range(2)]
    out = tpcf.batch_shear_2pcf(lens, shapes, tasks, bins, lens_patches=patches, n_patch=5,
                                spherical_coords=True, ctx=sctx)
    for (li, si), r in zip(tasks, out):
        Lc, Sc = lens[li], shapes[si]
        Ld = dict(x=Lc.x, y=Lc.y, z=Lc.z, val=Lc.val, w=Lc.w)
        Sd = dict(x=Sc.x, y=Sc.y, z=Sc.z, e1=Sc.e1, e2=Sc.e2, w=Sc.w, m=Sc.m)
        assert_parity(r, oracle.canon_sphere(oracle.SHEAR, Ld, Sd, bins.chord_edges_sq))
        np.testing.assert_array_equal(r.patch_sums.sum(0)[5], r.n_pairs)


def test_latitude_out_of_range_is_rejected(tpcf, sctx):
    L = dict(x=f32([0.1]), y=f32([1.7]), z=f32([0.0]), val=f32([1.0]), w=f32([1.0]))
    S = dict(x=f32([0.1]), y=f32([0.2]), z=f32([1.0]), e1=f32([0.1]), e2=f32([0.1]), w=f32([1.0]),
             m=f32([0.0]))
    bins = tpcf.create_bins(1 * ARCMIN, 60 * ARCMIN, 4)
    with pytest.raises(tpcf.TPCFError):
        run_shear(tpcf, sctx, L, S, bins)
