"""Seeded synthetic catalogues for the five benchmark workloads.

No public survey is used.  Positions are in arcmin on a flat patch, so the
angular bins are in arcmin directly.  Every draw comes from numpy's PCG64 with
seed 1000 + workload number, in a fixed order, so the same call always gives
the same catalogue.  ``scale`` shrinks object counts (areas stay) for tests.

  1  shear-scalar + scalar-scalar, 20k x 20k uniform on [0,600]^2, 15 log bins 1-100'
  2  scalar-scalar auto-correlation, 1M uniform on [0,600]^2, Gaussian random
     kappa field (2048^2, P(k) ~ k^-1.5, sigma 0.02), w ~ U(0.5,1.5), 30 log bins 0.5-250'
  3  shear-scalar with errors, 2M shear x 500k scalar on [0,1200]^2, clustered
     (half in Gaussian blobs of sigma 18' at 1 blob/deg^2, half Poisson),
     tangential shear around the 400 highest kappa peaks plus N(0,0.26) noise,
     100 k-means patches, 1000 resamples, 20 log bins 1-200'
  4  workload 3 without bootstrap, with a seeded chi^2 target
  5  tomography: 5 shear bins (0.2,0.5,1.0,1.9,4.0 M) x 5 scalar bins
     (0.1,0.2,0.4,0.7,1.0 M) on [0,1897.4]^2 drawn as workload 3, 25 pairs,
     100 patches, 1000 resamples, 20 log bins 1-300'
"""
from __future__ import annotations

import numpy as np

SIGMA_BLOB = 18.0     # 0.3 deg in arcmin
SIGMA_PEAK = 18.0
BLOB_AREA = 3600.0    # one blob per deg^2 (arcmin^2)

WORKLOADS = {
    1: dict(box=600.0, n_lens=20_000, n_src=20_000, bins=(1.0, 100.0, 15), clustered=False),
    2: dict(box=600.0, n_lens=1_000_000, bins=(0.5, 250.0, 30), clustered=False),
    3: dict(box=1200.0, n_lens=500_000, n_src=2_000_000, bins=(1.0, 200.0, 20), clustered=True,
            n_patch=100, n_boot=1000),
    4: dict(box=1200.0, n_lens=500_000, n_src=2_000_000, bins=(1.0, 200.0, 20), clustered=True),
    5: dict(box=1897.4, n_lens=(100_000, 200_000, 400_000, 700_000, 1_000_000),
            n_src=(200_000, 500_000, 1_000_000, 1_900_000, 4_000_000), bins=(1.0, 300.0, 20),
            clustered=True, n_patch=100, n_boot=1000),
}


def grf_kappa(rng, box, n_grid=2048, slope=-1.5, sigma=0.02):
    """Gaussian random field with P(k) ~ k^slope on an n_grid^2 grid, zero mean,
    standard deviation ``sigma`` (FFT of white noise times sqrt(P))."""
    white = rng.standard_normal((n_grid, n_grid))
    f = np.fft.rfft2(white)
    kx = np.fft.fftfreq(n_grid)[:, None]
    ky = np.fft.rfftfreq(n_grid)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    amp = np.zeros_like(k)
    nz = k > 0
    amp[nz] = k[nz] ** (slope / 2.0)
    field = np.fft.irfft2(f * amp, s=(n_grid, n_grid))
    field -= field.mean()
    field *= sigma / field.std()
    return field.astype(np.float64)


def sample_grid(field, box, x, y):
    """Nearest-grid-point sample of a periodic grid covering [0, box)^2."""
    n = field.shape[0]
    ix = np.clip((x / box * n).astype(np.int64), 0, n - 1)
    iy = np.clip((y / box * n).astype(np.int64), 0, n - 1)
    return field[iy, ix]


def positions(rng, n, box, clustered):
    if not clustered:
        return rng.uniform(0, box, n), rng.uniform(0, box, n)
    n_blob_pts = n // 2
    n_blobs = max(1, int(round(box * box / BLOB_AREA)))
    cx = rng.uniform(0, box, n_blobs)
    cy = rng.uniform(0, box, n_blobs)
    which = rng.integers(0, n_blobs, n_blob_pts)
    bx = np.mod(cx[which] + rng.normal(0, SIGMA_BLOB, n_blob_pts), box)
    by = np.mod(cy[which] + rng.normal(0, SIGMA_BLOB, n_blob_pts), box)
    px = rng.uniform(0, box, n - n_blob_pts)
    py = rng.uniform(0, box, n - n_blob_pts)
    return np.concatenate([bx, px]), np.concatenate([by, py])


def peak_shear_grid(kappa, box, n_peaks=400, amp=0.05, sigma_p=SIGMA_PEAK):
    """gamma1, gamma2 grids of the tangential pattern gamma_t = amp*exp(-r^2/2s^2)
    around the ``n_peaks`` highest local maxima of kappa:
    (gamma1, gamma2) = -gamma_t (cos 2phi, sin 2phi)."""
    n = kappa.shape[0]
    k = kappa
    is_max = np.ones_like(k, dtype=bool)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dx or dy:
                is_max &= k > np.roll(np.roll(k, dy, 0), dx, 1)
    iy, ix = np.nonzero(is_max)
    order = np.argsort(-k[iy, ix], kind="stable")[:n_peaks]
    iy, ix = iy[order], ix[order]
    pix = box / n
    half = int(np.ceil(5 * sigma_p / pix))
    off = np.arange(-half, half + 1)
    dxg, dyg = np.meshgrid(off * pix, off * pix)
    r2 = dxg * dxg + dyg * dyg
    gt = amp * np.exp(-r2 / (2 * sigma_p * sigma_p))
    with np.errstate(invalid="ignore", divide="ignore"):
        c2 = np.where(r2 > 0, (dxg * dxg - dyg * dyg) / r2, 0.0)
        s2 = np.where(r2 > 0, 2 * dxg * dyg / r2, 0.0)
    g1w, g2w = -gt * c2, -gt * s2
    g1 = np.zeros_like(k)
    g2 = np.zeros_like(k)
    for y0, x0 in zip(iy, ix):
        rows = (y0 + off) % n
        cols = (x0 + off) % n
        g1[np.ix_(rows, cols)] += g1w
        g2[np.ix_(rows, cols)] += g2w
    return g1, g2


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def shear_catalog(rng, n, box, clustered, g1=None, g2=None, noise=0.26, weights="uniform"):
    x, y = positions(rng, n, box, clustered)
    e1 = rng.normal(0, noise, n)
    e2 = rng.normal(0, noise, n)
    if g1 is not None:
        e1 = e1 + sample_grid(g1, box, x, y)
        e2 = e2 + sample_grid(g2, box, x, y)
    w = np.ones(n) if weights == "ones" else rng.uniform(0.5, 1.5, n)
    return dict(x=_f32(x), y=_f32(y), z=np.ones(n, np.float32), e1=_f32(e1), e2=_f32(e2),
                w=_f32(w), m=np.zeros(n, np.float32))


def lens_catalog(rng, n, box, clustered, kappa=None, weights="uniform"):
    x, y = positions(rng, n, box, clustered)
    val = sample_grid(kappa, box, x, y) if kappa is not None else rng.normal(0, 0.02, n)
    w = np.ones(n) if weights == "ones" else rng.uniform(0.5, 1.5, n)
    return dict(x=_f32(x), y=_f32(y), z=np.zeros(n, np.float32), val=_f32(val), w=_f32(w))


def make_workload(k: int, scale: float = 1.0, n_grid: int = 2048):
    """Catalogues of workload ``k`` (1..5) with object counts times ``scale``."""
    cfg = WORKLOADS[k]
    rng = np.random.default_rng(1000 + k)
    box = cfg["box"]
    s = lambda n: max(1, int(round(n * scale)))
    out = dict(workload=k, box=box, bins=cfg["bins"], scale=scale)
    if k == 1:
        x, y = rng.uniform(0, box, s(cfg["n_lens"])), rng.uniform(0, box, s(cfg["n_lens"]))
        nA = len(x)
        lens = dict(x=_f32(x), y=_f32(y), z=np.zeros(nA, np.float32),
                    val=_f32(rng.normal(0, 0.02, nA)), w=np.ones(nA, np.float32))
        nB = s(cfg["n_src"])
        xb, yb = rng.uniform(0, box, nB), rng.uniform(0, box, nB)
        src = dict(x=_f32(xb), y=_f32(yb), z=np.ones(nB, np.float32),
                   e1=_f32(rng.normal(0, 0.26, nB)), e2=_f32(rng.normal(0, 0.26, nB)),
                   w=np.ones(nB, np.float32), m=np.zeros(nB, np.float32))
        out.update(lenses=lens, shapes=src)
        # scalar-scalar leg of workload 1: kappa at the shape positions
        out["kappa_map"] = dict(x=src["x"], y=src["y"], kappa_E=_f32(rng.normal(0, 0.02, nB)),
                                kappa_B=np.zeros(nB, np.float32), w=np.ones(nB, np.float32))
        return out
    kappa = grf_kappa(rng, box, n_grid)
    if k == 2:
        n = s(cfg["n_lens"])
        x, y = rng.uniform(0, box, n), rng.uniform(0, box, n)
        kv = sample_grid(kappa, box, x, y)
        w = rng.uniform(0.5, 1.5, n)
        lens = dict(x=_f32(x), y=_f32(y), z=np.zeros(n, np.float32), val=_f32(kv), w=_f32(w))
        kmap = dict(x=lens["x"], y=lens["y"], kappa_E=lens["val"], kappa_B=np.zeros(n, np.float32),
                    w=lens["w"])
        out.update(lenses=lens, kappa_map=kmap)
        return out
    g1, g2 = peak_shear_grid(kappa, box)
    if k in (3, 4):
        src = shear_catalog(rng, s(cfg["n_src"]), box, True, g1, g2)
        lens = lens_catalog(rng, s(cfg["n_lens"]), box, True, kappa)
        out.update(lenses=lens, shapes=src)
        if k == 3:
            out.update(n_patch=cfg["n_patch"], n_boot=cfg["n_boot"])
        return out
    srcs = [shear_catalog(rng, s(n), box, True, g1, g2) for n in cfg["n_src"]]
    lenses = [lens_catalog(rng, s(n), box, True, kappa) for n in cfg["n_lens"]]
    tasks = [(i, j) for i in range(len(lenses)) for j in range(len(srcs))]
    out.update(lens_bins=lenses, shape_bins=srcs, tasks=tasks, n_patch=cfg["n_patch"],
               n_boot=cfg["n_boot"])
    return out
