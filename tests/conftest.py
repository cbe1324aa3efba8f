"""Shared fixtures: build the product library and the oracle once per session."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 GPU")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU visible")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import build as ob
    ob.build()
    from oracle import oracle as o
    return o


@pytest.fixture(scope="session")
def lib():
    from zynum_b200 import build as zb
    zb.build()
    from zynum_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def blas(lib):
    from zynum_b200 import blas as b
    return b


# --------------------------------------------------------------- fill helpers

def sample_value(row: int, col: int, salt: int) -> float:
    """fortran_compat_test.zig:12-16 sampleValue: ((row+1)(salt+3)+(col+1)(salt+7)) mod 29 - 14) / 9."""
    return (((row + 1) * (salt + 3) + (col + 1) * (salt + 7)) % 29 - 14.0) / 9.0


def padded(rows, cols, ld, salt, dtype, sentinel):
    """fortran_compat_test.zig:196-203 fillPaddedMatrix: sampleValue body, sentinel padding."""
    a = np.full((ld, max(cols, 1)), sentinel, dtype=dtype, order="F")
    r = np.arange(rows)[:, None]
    c = np.arange(cols)[None, :]
    a[:rows, :cols] = ((((r + 1) * (salt + 3) + (c + 1) * (salt + 7)) % 29) - 14.0) / 9.0
    return a


def uniform(rng, ld, cols, dtype=np.float64, rows=None):
    a = np.asfortranarray(rng.uniform(-1.0, 1.0, size=(ld, max(cols, 1))).astype(dtype))
    return a


def gemm_bound(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c0, u, cfac=4.0):
    """Componentwise bound c*k*u*(|alpha| |op(A)| |op(B)| + |beta| |C0|) (+ a few ulps of the result)."""
    A = np.abs(a[:m, :k] if ta == "N" else a[:k, :m].T).astype(np.float64)
    B = np.abs(b[:k, :n] if tb == "N" else b[:n, :k].T).astype(np.float64)
    ab = A @ B
    return cfac * max(k, 1) * u * (abs(alpha) * ab + abs(beta) * np.abs(c0[:m, :n])) + 1e-300
