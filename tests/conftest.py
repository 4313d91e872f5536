"""Shared fixtures.  Tests marked `gpu` need a CUDA device; everything else runs on CPU.

The CPU oracles under oracle/ are test infrastructure: the restatement (oracle/_build) is rebuilt
here when missing; the reference build (oracle/_ref) is produced by __graft_entry__.build() and
the tests that need it skip with a message when it is absent."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu)")


def _ensure_oracle():
    so = os.path.join(ROOT, "oracle", "_build", "libptoracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "_build/libptoracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return so


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("reference build oracle/_ref/libptref.so is absent (built by __graft_entry__.build())")
    return Reference()


@pytest.fixture(scope="session")
def libc():
    return ctypes.CDLL(None)


def srand_all(libc, seed=1):
    """The build draws its populate order from the C library rand(), like the reference."""
    libc.srand(seed)


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    torch.cuda.init()
    return torch.device("cuda:0")
