"""Shared test setup: paths, the `gpu` marker, oracle build, seeded inputs."""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "cuda-cholesky_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

# The reference's source tree, when a test run should (re)build its CPU library
# into oracle/_ref (normally __graft_entry__.build() has built it already).
REFERENCE_TREE = os.environ.get("CUCHOLESKY_REFERENCE", "")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: larger sizes")
    # the oracle is test infrastructure: build it on first use if it is missing
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile")], check=True)
    if (not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref.so"))
            and REFERENCE_TREE and os.path.isdir(REFERENCE_TREE)):
        subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile"), "ref",
                        f"REF={REFERENCE_TREE}"], check=False)


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "reference_small.npz"))


@pytest.fixture(scope="session")
def handle():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cucholesky
    h = cucholesky.Handle()
    yield h
    h.close()
