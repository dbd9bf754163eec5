"""Test configuration: import paths, the `gpu` marker, shared fixtures.

CPU tests (``-m "not gpu"``) cover the oracle against the reference's golden
vectors, mesh generation, host-side logic and the C ABI library's exports.
GPU tests (``-m gpu``) are the parity tests proper: they call the CUDA library
through its C ABI and compare with the oracle.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "a-lls-matrix-parallel-assembly_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the CUDA library")
    config.addinivalue_line("markers", "slow: long CPU test")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    if not os.path.exists(os.path.join(ORACLE, "liboracle.so")):
        subprocess.run(["make", "-s", "-C", ORACLE, "oracle"], check=True)
    return oracle


@pytest.fixture(scope="session")
def fem():
    import build
    build.build()
    import fem_alls
    return fem_alls


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    return torch.device("cuda:0")


def diag_scale(row_ptr: np.ndarray, col_idx: np.ndarray, values: np.ndarray) -> np.ndarray:
    """sqrt(|K_ii K_jj|) for every stored entry (i, j) of a CSR matrix."""
    n = row_ptr.shape[0] - 1
    rows = np.repeat(np.arange(n), np.diff(row_ptr))
    d = np.zeros(n)
    on = rows == col_idx
    d[rows[on]] = np.abs(values[on])
    return np.sqrt(d[rows] * d[col_idx])


def value_errors(row_ptr, col_idx, ref, test):
    """(max per-entry relative error, max row-scaled error |d|/sqrt(|K_ii K_jj|))."""
    diff = np.abs(test - ref)
    nz = ref != 0
    rel = float(np.max(diff[nz] / np.abs(ref[nz]))) if nz.any() else 0.0
    sc = diag_scale(row_ptr, col_idx, ref)
    scaled = float(np.max(diff / np.where(sc > 0, sc, 1.0))) if diff.size else 0.0
    return rel, scaled
