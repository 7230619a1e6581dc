"""CPU checks of the C-ABI library: it loads, exports every entry point that
include/tpcf_b200.h declares, and its host-only functions (edges, bin centres,
argument validation) agree with the oracle.  No compute call needs a GPU here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(tpcf_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol(tpcf):
    L = tpcf._lib.lib()
    decl = declared_functions()
    assert len(decl) >= 10
    for name in sorted(decl):
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
        assert name in tpcf._lib.EXPORTED, f"{name} has no ctypes signature in _lib.py"


def test_canonical_edges_equal_oracle(tpcf, oracle):
    for args in ((1.0, 100.0, 15, "log"), (0.5, 250.0, 30, "log"), (1.0, 300.0, 20, "log"),
                 (0.0, 10.0, 10, "lin"), (0.5, 50.0, 17, "sqrt"), (0.5, 50.0, 17, "ihs")):
        lo, hi, nb, sp = args
        b = tpcf.create_bins(lo, hi, nb, spacing=sp, p=0.3)
        e, e2 = oracle.canonical_edges(lo, hi, nb, tpcf._SPACING[sp], 0.3)
        np.testing.assert_array_equal(b.bin_edges, e)
        np.testing.assert_array_equal(b.bin_edges_sq, e2)


def test_bin_centers_equal_reference_fp32(tpcf, oracle):
    for lo, hi, nb, sp in ((1.0, 100.0, 15, 1), (0.5, 250.0, 30, 1), (0.0, 10.0, 10, 0), (0.5, 50.0, 17, 3)):
        b = tpcf.create_bins(lo, hi, nb, spacing=sp)
        _, centers, _ = oracle.create_bins_f32(lo, hi, nb, sp)
        np.testing.assert_array_equal(b.bin_centers, centers)


@pytest.mark.parametrize("bad", [(1.0, 100.0, 0, 1), (0.0, 100.0, 10, 1), (10.0, 1.0, 5, 1), (1.0, 100.0, 129, 1),
                                 (1.0, 100.0, 5, 7), (-1.0, 4.0, 5, 3)])
def test_invalid_bins_rejected(tpcf, bad):
    lo, hi, nb, sp = bad
    with pytest.raises(tpcf.TPCFError) as e:
        tpcf.create_bins(lo, hi, nb, spacing=sp)
    assert e.value.status == 1  # TPCF_ERR_INVALID_ARG, never an abort


def test_no_gpu_means_no_context(tpcf):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(tpcf.TPCFError) as e:
        tpcf.Context(0)
    assert e.value.status == 7  # TPCF_ERR_NO_DEVICE: there is no CPU fallback


def test_null_arguments_rejected(tpcf):
    L = tpcf._lib.lib()
    assert L.tpcf_create(None, 0, None) == 1
    assert L.tpcf_canonical_edges(None, None, None) == 1
    assert L.tpcf_shear_scalar(None, *([None] * 5), 0, *([None] * 7), 0, None, None, 0, None) == 1
    assert L.tpcf_abi_version() == 1
