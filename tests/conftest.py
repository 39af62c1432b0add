"""Shared test set-up: the gpu marker, the repo root on sys.path, and helpers
that load the golden fixtures. GPU tests call the product through the C ABI
(photon_tracer_b200 -> libphoton_cuda.so) and check it against the oracle."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs the CUDA library)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="session")
def built():
    """Builds (if stale) the product library and the oracle; returns the product module."""
    from photon_tracer_b200 import build as pbuild
    from oracle import build as obuild
    pbuild.build()
    obuild.build_oracle()
    obuild.build_ref()
    obuild.build_shim_check()
    import photon_tracer_b200
    return photon_tracer_b200
