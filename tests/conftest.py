"""Test configuration: the `gpu` marker and the shared fixtures.

CPU tests (`-m "not gpu"`) cover the oracle against the reference's golden
vectors, the host logic and the C-ABI library's exports. GPU tests are the
parity tests proper and call the CUDA path through the C ABI.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "_ref", "liborq_oracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "all"], check=True,
                       capture_output=True)
    return lib


@pytest.fixture(scope="session")
def oracle_lib():
    return _ensure_oracle()


@pytest.fixture(scope="session")
def golden():
    z = np.load(os.path.join(GOLDEN, "ref_golden.npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def digests():
    with open(os.path.join(GOLDEN, "ref_digests.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def aes_kat():
    with open(os.path.join(GOLDEN, "aes_gcm_kat.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def cuda_lib():
    """Build (if stale) and load liborq_cuda.so for GPU tests."""
    from orq_b200 import build as b

    b.build()
    import orq_b200

    return orq_b200.load_library()
