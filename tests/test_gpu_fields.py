"""GPU field rotation (tpcf_rotate_from_poles) against the FP32 restatement of
rotate_data_from_poles_and_meridian (src/main.f90:953-1015).

The decisions (rotate or not, the wrap) and the medians must be identical; the
rotated coordinates agree to 5e-6 rad (the reference evaluates the rotation
in FP32, the library in FP64 rounded to FP32)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

D2R = np.pi / 180.0


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def wrapdiff(a, b):
    d = (a.astype(np.float64) - b.astype(np.float64)) % (2 * np.pi)
    return np.minimum(d, 2 * np.pi - d)


@pytest.mark.parametrize("case", ["pole", "meridian", "none", "south_even"])
def test_rotation_matches_restatement(tpcf, oracle, ctx, case):
    rng = np.random.default_rng({"pole": 1, "meridian": 2, "none": 3, "south_even": 4}[case])
    nA, nB = (20001, 30000) if case != "south_even" else (20000, 25000)
    if case == "pole":
        lam = lambda n: rng.uniform(10, 50, n); phi = lambda n: rng.uniform(75, 85, n); r = 10.0
    elif case == "meridian":
        lam = lambda n: (rng.uniform(-10, 10, n) % 360); phi = lambda n: rng.uniform(-20, 20, n); r = 1.0
    elif case == "none":
        lam = lambda n: rng.uniform(110, 130, n); phi = lambda n: rng.uniform(-30, -10, n); r = 1.0
    else:
        lam = lambda n: rng.uniform(200, 240, n); phi = lambda n: rng.uniform(-88, -70, n); r = 3.0
    xA, yA, xB, yB = f32(lam(nA) * D2R), f32(phi(nA) * D2R), f32(lam(nB) * D2R), f32(phi(nB) * D2R)
    r_max = np.float32(r * D2R)
    o_rot, o_c, oxA, oyA, oxB, oyB = oracle.rotate_from_poles(xA, yA, r_max, xB, yB)
    gxA, gyA, gxB, gyB = xA.copy(), yA.copy(), xB.copy(), yB.copy()
    rot, center = tpcf.rotate_data_from_poles_and_meridian(gxA, gyA, r_max, x_B=gxB, y_B=gyB, ctx=ctx)
    assert rot == o_rot == (case != "none")
    assert center == (float(o_c[0]), float(o_c[1]))
    for g, o in ((gxA, oxA), (gxB, oxB)):
        assert wrapdiff(g, o).max() < 5e-6
    for g, o in ((gyA, oyA), (gyB, oyB)):
        ok = np.abs(o) < 1.5  # FP32 acos loses precision next to the poles
        assert np.abs(g[ok].astype(np.float64) - o[ok]).max() < 5e-6


def test_rotation_on_device_tensors(tpcf, oracle, ctx):
    import torch
    rng = np.random.default_rng(5)
    xA, yA = f32(rng.uniform(0, 20, 5000) * D2R), f32(rng.uniform(80, 89, 5000) * D2R)
    r_max = np.float32(5 * D2R)
    o_rot, o_c, oxA, oyA, _, _ = oracle.rotate_from_poles(xA, yA, r_max)
    tx, ty = torch.from_numpy(xA.copy()).cuda(), torch.from_numpy(yA.copy()).cuda()
    rot, center = tpcf.rotate_data_from_poles_and_meridian(tx, ty, r_max, ctx=ctx)
    assert rot and o_rot
    assert wrapdiff(tx.cpu().numpy(), oxA).max() < 5e-6
