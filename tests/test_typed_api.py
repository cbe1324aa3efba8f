"""C++ typed API mirror of Zynum's matrixMultiply (include/zynum/matrix_multiply.hpp)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def typed_api_binary(lib, tmp_path_factory):
    out = tmp_path_factory.mktemp("typed") / "typed_api_test"
    libdir = ROOT / "zynum_b200" / "lib"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "typed_api_test.cpp"),
                    f"-L{libdir}", "-lzynum_blas_gpu", f"-Wl,-rpath,{libdir}", "-o", str(out)], check=True)
    return out


def test_typed_api_errors(typed_api_binary):
    r = subprocess.run([str(typed_api_binary), "checks"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_typed_api_products(typed_api_binary):
    r = subprocess.run([str(typed_api_binary), "compute"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr + r.stdout
