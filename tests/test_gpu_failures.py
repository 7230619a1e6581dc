"""Failure paths, made to happen without a GPU fault or hang
(tpcf_debug_inject; the reference stops the program instead,
src/kdtree.f90:119-122, :265-267):

- a device workspace allocation that fails at one of several points of a
  call returns TPCF_ERR_OOM with its message, and the same context then
  computes the correct result;
- a source tile of the pair kernel whose bulk copy is never issued makes the
  bounded mbarrier waits on it run out: the call returns TPCF_ERR_TIMEOUT
  (every copy that was issued has landed before the blocks exit), and the
  same context then computes the correct result;
- the same for the first tile of the marks kernel (xi from marks and the
  marks bootstrap).
Invalid arguments and a missing device are covered on the CPU (test_abi)."""
import ctypes as C
import time

import numpy as np
import pytest

from conftest import uniform_shear
from parity import check_sums

pytestmark = pytest.mark.gpu


def shear(tpcf, ctx, L, S, bins):
    return tpcf.tangential_shear_tpcf(L["x"], L["y"], L["z"], L["val"], L["w"], S["x"], S["y"], S["z"],
                                      S["e1"], S["e2"], S["w"], S["m"], bins, calculate_marks=False, ctx=ctx)


def inject(tpcf, ctx, fail_alloc=-1, skip_tile=-1, wait_polls=0):
    st = tpcf._lib.lib().tpcf_debug_inject(ctx.handle, int(fail_alloc), int(skip_tile), C.c_uint32(wait_polls))
    assert st == tpcf._lib.TPCF_OK


@pytest.mark.parametrize("k", [0, 4, 12, 30])
def test_injected_allocation_failure_then_recovery(tpcf, oracle, k):
    ctx = tpcf.Context(0)
    L, S = uniform_shear(2000, 3000, 200.0, 80 + k)
    bins = tpcf.create_bins(1.0, 40.0, 10)
    can = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq)
    if k == 30:
        shear(tpcf, ctx, L, S, bins)   # a warm context: the failing allocation is a regrowth
        S = {q: np.concatenate([v, v]) for q, v in S.items()}
        can = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq)
    inject(tpcf, ctx, fail_alloc=k if k < 30 else 0)
    with pytest.raises(tpcf.TPCFError) as e:
        shear(tpcf, ctx, L, S, bins)
    assert e.value.status == tpcf._lib.TPCF_ERR_OOM
    assert "allocation" in str(e.value)
    check_sums(f"call after an injected allocation failure at workspace allocation {k}", shear(tpcf, ctx, L, S, bins),
               can)
    ctx.close()


def test_bounded_wait_runs_out_then_recovery(tpcf, oracle):
    ctx = tpcf.Context(0)
    L, S = uniform_shear(3000, 20000, 300.0, 90)
    bins = tpcf.create_bins(1.0, 60.0, 12)
    can = oracle.canon_pairs(oracle.SHEAR, L, S, bins.bin_edges_sq)
    for tile, polls in ((0, 1 << 12), (5, 1 << 16)):
        inject(tpcf, ctx, skip_tile=tile, wait_polls=polls)
        t0 = time.time()
        with pytest.raises(tpcf.TPCFError) as e:
            shear(tpcf, ctx, L, S, bins)
        dt = time.time() - t0
        assert e.value.status == tpcf._lib.TPCF_ERR_TIMEOUT, str(e.value)
        print(f"tile {tile} never issued, {polls} polls per wait: TIMEOUT after {dt:.3f} s")
    inject(tpcf, ctx)
    check_sums("call after a bounded wait ran out", shear(tpcf, ctx, L, S, bins), can)
    ctx.close()


def test_marks_bounded_wait_runs_out_then_recovery(tpcf, oracle):
    ctx = tpcf.Context(0)
    rng = np.random.default_rng(92)
    n, nb, n_map = 8192, 20, 3
    raw = {"x": rng.normal(size=n).astype(np.float32), "y": rng.normal(size=n).astype(np.float32),
           "w": rng.uniform(0.1, 2, n).astype(np.float32),
           "xi_E": rng.normal(size=(n, nb)).astype(np.float32), "xi_B": rng.normal(size=(n, nb)).astype(np.float32),
           "K": rng.uniform(0.5, 1.5, (n, nb)).astype(np.float32)}
    marks = [tpcf.MarksField(**raw)]
    val = rng.normal(0, 0.02, (n_map, n)).astype(np.float32)
    w = rng.uniform(0.5, 1.5, (n_map, n)).astype(np.float32)
    inject(tpcf, ctx, skip_tile=0, wait_polls=1 << 12)
    for call in (lambda: tpcf.calculate_tpcf_from_marks(marks, [val], [w], ctx=ctx),
                 lambda: tpcf.marks_bootstrap(marks, 20, seed=3, covariance=False, ctx=ctx)):
        with pytest.raises(tpcf.TPCFError) as e:
            call()
        assert e.value.status == tpcf._lib.TPCF_ERR_TIMEOUT, str(e.value)
    inject(tpcf, ctx)
    out = tpcf.calculate_tpcf_from_marks(marks, [val], [w], ctx=ctx)
    for m in range(n_map):
        per, _ = oracle.xi_from_marks([raw], [val[m]], [w[m]])
        np.testing.assert_allclose(out["g_t"][m, 0], per[0]["g_t"], rtol=1e-9)
        np.testing.assert_allclose(out["weights"][m, 0], per[0]["weights"], rtol=1e-12)
    ctx.close()
