"""CPU checks of the spherical oracle (test infrastructure) and of the host-only
spherical entry points of the C ABI.

The reference has no spherical test data, so the canonical spherical rule is
pinned by analytic cases: unit vectors against libm in FP64, separations
along the equator that are exact multiples of the input angles, and a pure
tangential shear pattern whose g_t is 1 by construction.  The FP32
restatement of the reference's loop (acos of the dot product) is compared at
separations where FP32 acos is accurate to ~1e-3.
"""
import numpy as np
import pytest

D2R = np.pi / 180.0


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def cap_catalogue(rng, n, lam0, lam1, phi0, phi1):
    """Points uniform on the sphere inside a longitude/latitude box (degrees)."""
    lam = rng.uniform(lam0, lam1, n) * D2R
    phi = np.arcsin(rng.uniform(np.sin(phi0 * D2R), np.sin(phi1 * D2R), n))
    return f32(lam), f32(phi)


def test_unit_vectors_against_libm(oracle):
    rng = np.random.default_rng(0)
    lam = f32(rng.uniform(-7, 13, 100000))
    phi = f32(rng.uniform(-1.5707964, 1.5707964, 100000))
    hi, lo = oracle.unit_vectors(lam, phi)
    u = hi.astype(np.float64) + lo
    l, p = lam.astype(np.float64), phi.astype(np.float64)
    ref = np.stack([np.cos(p) * np.cos(l), np.cos(p) * np.sin(l), np.sin(p)], 1)
    assert np.abs(u - ref).max() < 4e-15
    # hi is the FP32 rounding of u; lo the FP32 rounding of the remainder
    np.testing.assert_array_equal(hi, u.astype(np.float32))
    assert np.all(np.abs(lo) <= np.spacing(np.abs(hi)) / 2 + 1e-45)


def test_chord_edges_match_the_library(tpcf, oracle):
    for (lo, hi, n, sp) in ((1 / 60 * D2R, 100 / 60 * D2R, 15, "log"), (0.0, 0.5, 7, "lin"),
                            (0.01, 3.1, 20, "sqrt")):
        b = tpcf.create_bins(lo, hi, n, spacing=sp)
        ref = oracle.sphere_edges_sq(b.bin_edges)
        np.testing.assert_array_equal(b.chord_edges_sq, ref)
        np.testing.assert_allclose(ref, (2 * np.sin(b.bin_edges / 2)) ** 2, rtol=1e-15, atol=1e-300)


def test_chord_edges_reject_beyond_pi(tpcf):
    b = tpcf.create_bins(0.1, 3.5, 4, spacing="lin")
    with pytest.raises(tpcf.TPCFError):
        b.chord_edges_sq


def test_equator_separations_are_exact(oracle):
    """Lens at (0, 0); sources on the equator at longitudes k * 2^-10 rad: the
    chord is 2 sin(dlam/2), so every source falls in the bin of its exact
    angle (bins with edges strictly between the sample angles)."""
    k = np.arange(1, 200)
    lamB = f32(k * 2.0 ** -10)
    S = dict(x=lamB, y=f32(np.zeros_like(lamB)), z=f32(np.ones_like(lamB)), e1=f32(np.zeros_like(lamB)),
             e2=f32(np.zeros_like(lamB)), w=f32(np.ones_like(lamB)), m=f32(np.zeros_like(lamB)))
    L = dict(x=f32([0.0]), y=f32([0.0]), z=f32([0.0]), val=f32([1.0]), w=f32([1.0]))
    edges = (np.array([0.5, 10.5, 50.5, 120.5, 199.5]) * 2.0 ** -10)
    can = oracle.canon_sphere(oracle.SHEAR, L, S, oracle.sphere_edges_sq(edges))
    np.testing.assert_array_equal(can["n_pairs"], [10, 40, 70, 79])
    ang = k * 2.0 ** -10
    expect = [ang[(ang > a) & (ang < b)].sum() for a, b in zip(edges[:-1], edges[1:])]
    np.testing.assert_allclose(can["sum_dw"], expect, rtol=1e-13)


def test_pure_tangential_pattern(oracle):
    """Sources around a lens at (40 deg, -30 deg) with e = -(cos 2a, sin 2a),
    a the bearing at the lens (east of north measured as in angles_sphere):
    g_t = 1, g_x = 0 for every bin."""
    rng = np.random.default_rng(3)
    lam1, phi1 = 40 * D2R, -30 * D2R
    n = 4000
    d = rng.uniform(2, 90, n) / 60 * D2R
    alpha = rng.uniform(0, 2 * np.pi, n)  # angle of the direction from the north axis
    # destination point of an initial great-circle direction (east = sin, north = cos)
    phi2 = np.arcsin(np.sin(phi1) * np.cos(d) + np.cos(phi1) * np.sin(d) * np.cos(alpha))
    lam2 = lam1 + np.arctan2(np.sin(alpha) * np.sin(d) * np.cos(phi1),
                             np.cos(d) - np.sin(phi1) * np.sin(phi2))
    lamB, phiB = f32(lam2), f32(phi2)
    # bearing recomputed from the rounded positions: A = east, B = north components
    l2, p2 = lamB.astype(np.float64), phiB.astype(np.float64)
    l1, p1 = float(np.float32(lam1)), float(np.float32(phi1))
    A = np.cos(p2) * np.sin(l2 - l1)
    B = np.cos(p1) * np.sin(p2) - np.sin(p1) * np.cos(p2) * np.cos(l2 - l1)
    c2, s2 = (A * A - B * B) / (A * A + B * B), 2 * A * B / (A * A + B * B)
    S = dict(x=lamB, y=phiB, z=f32(np.ones(n)), e1=f32(-c2), e2=f32(-s2), w=f32(np.ones(n)),
             m=f32(np.zeros(n)))
    L = dict(x=f32([lam1]), y=f32([phi1]), z=f32([0.0]), val=f32([1.0]), w=f32([1.0]))
    edges = np.geomspace(1 / 60 * D2R, 100 / 60 * D2R, 11)
    can = oracle.normalise(oracle.canon_sphere(oracle.SHEAR, L, S, oracle.sphere_edges_sq(edges)))
    assert can["n_pairs"].sum() == n
    full = can["n_pairs"] > 0
    assert full.sum() >= 9
    np.testing.assert_allclose(can["g_t"][full], 1.0, atol=2e-7)
    np.testing.assert_allclose(can["g_x"][full], 0.0, atol=2e-7)


def test_reference_restatement_at_large_separations(oracle):
    """FP32 acos (the reference's distance_sphere) against the canonical rule:
    counts agree to 0.5% per bin and xi to 2e-3 of its noise scale at
    separations of 0.5 to 5 degrees."""
    rng = np.random.default_rng(5)
    n = 2500
    xa, ya = cap_catalogue(rng, n, 30, 50, -40, -20)
    xb, yb = cap_catalogue(rng, n, 30, 50, -40, -20)
    L = dict(x=xa, y=ya, z=f32(np.zeros(n)), val=f32(rng.normal(0, 0.02, n)), w=f32(np.ones(n)))
    S = dict(x=xb, y=yb, z=f32(np.ones(n)), e1=f32(rng.normal(0, 0.26, n)), e2=f32(rng.normal(0, 0.26, n)),
             w=f32(np.ones(n)), m=f32(np.zeros(n)))
    lo, hi = 0.5 * D2R, 5 * D2R
    edges, _ = oracle.canonical_edges(lo, hi, 8)
    raw = oracle.canon_sphere(oracle.SHEAR, L, S, oracle.sphere_edges_sq(edges))
    can = oracle.normalise(raw)
    ref = oracle.ref_sphere_f32(oracle.SHEAR, L, S, lo, hi, 8, num_threads=8)
    np.testing.assert_allclose(ref["n_pairs"], can["n_pairs"], rtol=5e-3)
    scale = raw["abs_gt"] / raw["sum_K"]
    assert np.all(np.abs(ref["g_t"] - can["g_t"]) <= 2e-3 * scale)


def test_field_rotation_restatement(oracle):
    """rotation_sphere as written in src/utils.f90:483-509 rotates about the y
    axis by +phi_c after moving the field centre (median) to longitude pi, so
    the centre's latitude is doubled rather than removed; the
    restatement keeps that (the centre at x = -cos 2phi_c, z = sin 2phi_c).  A field near the pole is rotated, a field far
    from poles and meridian is not."""
    rng = np.random.default_rng(9)
    n = 1001
    x = f32(rng.uniform(10, 50, n) * D2R)
    y = f32(rng.uniform(75, 85, n) * D2R)
    x[0], y[0] = np.median(x), np.median(y)
    rot, center, xr, yr, _, _ = oracle.rotate_from_poles(x, y, np.float32(10 * D2R))
    assert rot
    assert center[0] == x[0] and center[1] == y[0]
    # the centre lands at x = -cos(2 phi_c), y = 0, z = sin(2 phi_c)
    c2 = np.cos(2 * float(y[0]))
    assert abs(xr[0] - (np.pi if c2 > 0 else 0.0)) < 1e-6
    assert abs(yr[0] - np.arcsin(np.sin(2 * float(y[0])))) < 1e-5
    x2 = f32(rng.uniform(110, 130, n) * D2R)
    y2 = f32(rng.uniform(-30, -10, n) * D2R)
    rot2, _, xr2, yr2, _, _ = oracle.rotate_from_poles(x2, y2, np.float32(1 * D2R))
    assert not rot2
    np.testing.assert_array_equal(xr2, x2)
    np.testing.assert_array_equal(yr2, y2)
