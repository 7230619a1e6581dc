"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def tpcf():
    return importlib.import_module("2pcf_b200")


@pytest.fixture(scope="session")
def synth():
    return importlib.import_module("2pcf_b200.synth")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def ctx(tpcf):
    c = tpcf.Context(0)
    yield c
    c.close()


def uniform_shear(n_lens, n_src, box, seed, w="ones"):
    rng = np.random.default_rng(seed)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    L = dict(x=f(rng.uniform(0, box, n_lens)), y=f(rng.uniform(0, box, n_lens)),
             z=np.zeros(n_lens, np.float32), val=f(rng.normal(0, 0.02, n_lens)),
             w=f(np.ones(n_lens) if w == "ones" else rng.uniform(0.5, 1.5, n_lens)))
    S = dict(x=f(rng.uniform(0, box, n_src)), y=f(rng.uniform(0, box, n_src)),
             z=np.ones(n_src, np.float32), e1=f(rng.normal(0, 0.26, n_src)),
             e2=f(rng.normal(0, 0.26, n_src)),
             w=f(np.ones(n_src) if w == "ones" else rng.uniform(0.5, 1.5, n_src)),
             m=np.zeros(n_src, np.float32))
    return L, S
