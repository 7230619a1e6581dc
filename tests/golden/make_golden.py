"""Generates the golden fixtures in tests/golden/ from the CPU oracle.

The reference (Fortran) cannot be compiled here and its own tests hold no
golden vectors for this path, so these fixtures pin the oracle itself: the FP64
canonical pair sums, the FP32 restatement of the reference loop, the
deterministic k-means and the block bootstrap, on small seeded inputs.  The
CPU tests recompute them and require bit-identical results; the GPU tests
compare the library against them.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def shear_inputs(seed, n_lens, n_src, box):
    rng = np.random.default_rng(seed)
    L = dict(x=f32(rng.uniform(0, box, n_lens)), y=f32(rng.uniform(0, box, n_lens)),
             z=f32(rng.uniform(-0.1, 0.6, n_lens)), val=f32(rng.normal(0, 0.02, n_lens)),
             w=f32(rng.uniform(0.5, 1.5, n_lens)))
    L["w"][::53] = 0.0
    S = dict(x=f32(rng.uniform(0, box, n_src)), y=f32(rng.uniform(0, box, n_src)),
             z=f32(rng.uniform(-0.1, 1.2, n_src)), e1=f32(rng.normal(0, 0.26, n_src)),
             e2=f32(rng.normal(0, 0.26, n_src)), w=f32(rng.uniform(0.5, 1.5, n_src)),
             m=f32(rng.normal(0, 0.02, n_src)))
    return L, S


def make_shear():
    L, S = shear_inputs(2001, 1500, 2000, 300.0)
    bins = (1.0, 100.0, 15)
    _, e2 = O.canonical_edges(*bins)
    can = O.canon_pairs(O.SHEAR, L, S, e2, num_threads=1)
    ref = O.ref_pairs(O.SHEAR, L, S, *bins, num_threads=1, marks=True)
    out = {f"L_{k}": v for k, v in L.items()}
    out.update({f"S_{k}": v for k, v in S.items()})
    out.update({f"canon_{k}": v for k, v in can.items()})
    out.update({f"ref_{k}": v for k, v in ref.items() if k != "xi_E_marks" or True})
    out["edges_sq"] = e2
    out["bins"] = np.array(bins)
    return out


def make_kappa():
    rng = np.random.default_rng(2002)
    n = 2500
    L = dict(x=f32(rng.uniform(0, 200, n)), y=f32(rng.uniform(0, 200, n)),
             val=f32(rng.normal(0, 0.02, n)), w=f32(rng.uniform(0.5, 1.5, n)))
    K = dict(x=f32(rng.uniform(0, 200, n)), y=f32(rng.uniform(0, 200, n)),
             kappa_E=f32(rng.normal(0, 0.02, n)), kappa_B=f32(rng.normal(0, 0.01, n)),
             w=f32(rng.uniform(0.5, 1.5, n)))
    bins = (0.5, 80.0, 30)
    _, e2 = O.canonical_edges(*bins)
    can = O.canon_pairs(O.KAPPA, L, K, e2, num_threads=1)
    ref = O.ref_pairs(O.KAPPA, L, K, *bins, num_threads=1)
    out = {f"L_{k}": v for k, v in L.items()}
    out.update({f"K_{k}": v for k, v in K.items()})
    out.update({f"canon_{k}": v for k, v in can.items()})
    out.update({f"ref_{k}": v for k, v in ref.items()})
    out["edges_sq"] = e2
    out["bins"] = np.array(bins)
    return out


def make_kmeans():
    rng = np.random.default_rng(2003)
    n = 4000
    x = f32(np.concatenate([rng.normal(50, 15, n // 2), rng.uniform(0, 200, n // 2)]))
    y = f32(np.concatenate([rng.normal(120, 20, n // 2), rng.uniform(0, 150, n // 2)]))
    w = f32(0.01 + rng.uniform(0.5, 1.5, n) / 1.5)
    lab_d, cen_d, it_d = O.kmeans_det(x, y, w, 12)
    lab_r, cen_r, it_r = O.kmeans_ref_f32(x, y, w, 12)
    return dict(x=x, y=y, w=w, k=np.array(12), det_labels=lab_d, det_centroids=cen_d,
                det_iters=np.array(it_d), ref_labels=lab_r, ref_centroids=cen_r, ref_iters=np.array(it_r))


def make_bootstrap():
    rng = np.random.default_rng(2004)
    n_patch, n_bin, n_boot = 17, 9, 64
    St = rng.normal(0, 1, (n_patch, n_bin))
    Sx = rng.normal(0, 1, (n_patch, n_bin))
    SK = rng.uniform(1, 5, (n_patch, n_bin))
    SK[3, 4] = 0.0
    Sw = rng.uniform(1, 5, n_patch)
    mult = O.bootstrap_multiplicity(12345, n_boot, n_patch, n_patch)
    gt, gx, W = O.block_bootstrap(mult, St, Sx, SK, Sw)
    cov = O.covariance(gt)
    return dict(St=St, Sx=Sx, SK=SK, Sw=Sw, seed=np.array(12345, np.uint64), mult=mult, gt=gt, gx=gx,
                W=W, cov_gt=cov)


def main():
    for name, fn in (("shear_small", make_shear), ("kappa_small", make_kappa),
                     ("kmeans_small", make_kmeans), ("bootstrap_small", make_bootstrap)):
        data = fn()
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
        print(name, sum(v.nbytes for v in data.values()), "bytes")


if __name__ == "__main__":
    main()
