"""C-ABI surface checks that need no GPU: the library loads, exports every
symbol the public header declares, and rejects illegal arguments exactly like
the reference's gemmError / CBLAS wrappers (before any GPU work)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared_symbols():
    names = []
    for h in (ROOT / "include").glob("*.h"):
        for m in re.finditer(r"^ZYNUM_BLAS_GPU_API\s+[\w\s\*]*?\b(\w+)\s*\(", h.read_text(), re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared_symbols()
    for required in ("dgemm_", "sgemm_", "cblas_dgemm", "cblas_sgemm", "xerbla_", "zynum_blas_gpu_dgemm_device"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    so = ROOT / "zynum_b200" / "lib" / "libzynum_blas_gpu.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in _declared_symbols() if s not in exported]
    assert not missing, missing
    for s in _declared_symbols():
        assert hasattr(lib, s)


def test_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "h.c"
    src.write_text('#include "zynum_blas_gpu.h"\nint main(void){return 0;}\n')
    for cc in (["gcc", "-std=c99"], ["g++", "-x", "c++", "-std=c++17"]):
        subprocess.run([*cc, "-fsyntax-only", f"-I{ROOT / 'include'}", str(src)], check=True)


def _dgemm_err(blas, ta, tb, m, n, k, lda, ldb, ldc):
    """Run dgemm_ with an illegal argument in a subprocess and capture xerbla's stderr."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from zynum_b200 import blas\n"
        "a=np.zeros((64,64),order='F'); c=np.full((64,64),7.0,order='F')\n"
        "blas.dgemm(%r,%r,%d,%d,%d,1.0,a,%d,a,%d,0.0,c,%d)\n"
        "assert (c==7.0).all()\n" % (str(ROOT), ta, tb, m, n, k, lda, ldb, ldc)
    )
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return r.stderr


@pytest.mark.parametrize(
    "args,param",
    [
        (("X", "N", 2, 2, 2, 2, 2, 2), 1),
        (("N", "Q", 2, 2, 2, 2, 2, 2), 2),
        (("N", "N", -1, 2, 2, 2, 2, 2), 3),
        (("N", "N", 2, -1, 2, 2, 2, 2), 4),
        (("N", "N", 2, 2, -1, 2, 2, 2), 5),
        (("N", "N", 4, 2, 2, 3, 2, 4), 8),
        (("T", "N", 4, 2, 5, 4, 5, 4), 8),
        (("N", "N", 2, 2, 5, 2, 4, 2), 10),
        (("N", "T", 2, 6, 5, 2, 5, 2), 10),
        (("N", "N", 5, 2, 2, 5, 2, 4), 13),
    ],
)
def test_dgemm_argument_errors_report_xerbla(lib, blas, args, param):
    err = _dgemm_err(blas, *args)
    assert f" ** On entry to DGEMM parameter number {param} had an illegal value" in err


def test_device_entry_returns_parameter_index(lib, blas):
    L = lib
    assert L.zynum_blas_gpu_dgemm_device(b"N", b"N", -1, 2, 2, 1.0, None, 2, None, 2, 0.0, None, 2, None) == 3
    assert L.zynum_blas_gpu_dgemm_device(b"Z", b"N", 2, 2, 2, 1.0, None, 2, None, 2, 0.0, None, 2, None) == 1
    assert L.zynum_blas_gpu_sgemm_device(b"N", b"N", 2, 2, 2, 1.0, None, 1, None, 2, 0.0, None, 2, None) == 8
    # m == 0 / n == 0: nothing to do, success without touching the GPU
    assert L.zynum_blas_gpu_dgemm_device(b"N", b"N", 0, 2, 2, 1.0, None, 1, None, 2, 0.0, None, 1, None) == 0


def test_cblas_invalid_enums_return_silently(lib, blas):
    c = np.full((2, 2), 5.0, order="F")
    a = np.ones((2, 2), order="F")
    blas.cblas_dgemm(99, blas.CblasNoTrans, blas.CblasNoTrans, 2, 2, 2, 1.0, a, 2, a, 2, 0.0, c, 2)
    blas.cblas_dgemm(blas.CblasColMajor, 7, blas.CblasNoTrans, 2, 2, 2, 1.0, a, 2, a, 2, 0.0, c, 2)
    blas.cblas_dgemm(blas.CblasColMajor, blas.CblasNoTrans, 0, 2, 2, 2, 1.0, a, 2, a, 2, 0.0, c, 2)
    assert (c == 5.0).all()


def test_lsame_and_xerbla_trim(lib):
    assert lib.lsame_(b"n", b"N") == 1 and lib.lsame_(b"T", b"N") == 0
    code = ("import sys; sys.path.insert(0,%r)\nimport ctypes as C\nfrom zynum_b200 import _lib\n"
            "L=_lib.load(); L.xerbla_(b'DGEMM ', C.byref(C.c_int32(3)))\n" % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=60)
    assert " ** On entry to DGEMM parameter number 3 had an illegal value" in r.stderr


def test_abi_manifest_is_current_and_matches_reference():
    """include/abi_manifest.json is what include/make_abi_manifest.py writes for the current
    header, and every reference Level-3 export the library provides (tests/golden/
    reference_abi_subset.json, from the reference's own manifest) has the same return type and
    argument types in the same order."""
    sys.path.insert(0, str(ROOT / "include"))
    try:
        import make_abi_manifest as mk
    finally:
        sys.path.pop(0)
    import json
    man = mk.build_manifest()
    committed = json.loads((ROOT / "include" / "abi_manifest.json").read_text())
    assert man == committed, "include/abi_manifest.json is stale: rerun include/make_abi_manifest.py"
    ref = json.loads((ROOT / "tests" / "golden" / "reference_abi_subset.json").read_text())
    report = mk.diff(man, ref)
    for part in ("fortran", "cblas"):
        assert report[part]["differ"] == [], report[part]["differ"]
        provided = set(report[part]["same"])
        # every Level-3 export of the reference is provided: nothing reference-only
        assert report[part]["reference_only"] == [], report[part]["reference_only"]
        for fam in ("gemm", "trsm", "syrk", "symm", "trmm", "syr2k"):
            for p in "sdcz":
                name = f"cblas_{p}{fam}" if part == "cblas" else f"{p}{fam}_"
                assert name in provided, name
        for fam in ("hemm", "herk", "her2k"):
            for p in "cz":
                name = f"cblas_{p}{fam}" if part == "cblas" else f"{p}{fam}_"
                assert name in provided, name
    assert {"xerbla_", "lsame_", "zynum_blas_shutdown"} <= set(report["fortran"]["same"])
