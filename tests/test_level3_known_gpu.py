"""The reference's own Level-3 known answers (2 x 2 problems of
test/abi/fortran_compat_test.zig:1676-1800) through this library's Fortran
ABI: DSYMM, ZHEMM, DSYRK, ZHERK, DSYR2K, ZHER2K, DTRMM, DTRSM, within the
reference's 1e-12 and with the untouched triangle keeping its sentinel."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())["level3_known_answers"]


def _lv(vals):
    if isinstance(vals[0], list):
        return np.asfortranarray(np.array([complex(r, i) for r, i in vals], np.complex128).reshape(2, 2).T)
    return np.asfortranarray(np.array(vals, np.float64).reshape(2, 2).T)


def _close(got, want):
    assert np.abs(got - want).max() <= 1e-12, (got, want)


def test_level3_known_answers_fortran_abi(blas):
    g = GOLDEN
    c = np.zeros((2, 2), order="F")
    blas.symm("L", "U", 2, 2, 1.0, _lv(g["dsymm"]["a"]), 2, _lv(g["dsymm"]["b"]), 2, 0.0, c, 2)
    _close(c, _lv(g["dsymm"]["c"]))
    c = np.zeros((2, 2), np.complex128, order="F")
    blas.symm("L", "U", 2, 2, 1.0, _lv(g["zhemm"]["a"]), 2, _lv(g["zhemm"]["b"]), 2, 0.0, c, 2, herm=True)
    _close(c, _lv(g["zhemm"]["c"]))
    c = _lv(g["dsyrk"]["c0"])
    blas.syrk("U", "N", 2, 2, 1.0, _lv(g["dsyrk"]["a"]), 2, 0.0, c, 2)
    _close(c, _lv(g["dsyrk"]["c"]))
    c = _lv(g["zherk"]["c0"])
    blas.herk("U", "N", 2, 2, 1.0, _lv(g["zherk"]["a"]), 2, 0.0, c, 2)
    _close(c, _lv(g["zherk"]["c"]))
    c = _lv(g["dsyr2k"]["c0"])
    blas.syr2k("U", "N", 2, 2, 1.0, _lv(g["dsyr2k"]["a"]), 2, _lv(g["dsyr2k"]["b"]), 2, 0.0, c, 2)
    _close(c, _lv(g["dsyr2k"]["c"]))
    c = _lv(g["zher2k"]["c0"])
    blas.syr2k("U", "N", 2, 2, 1.0, _lv(g["zher2k"]["a"]), 2, _lv(g["zher2k"]["b"]), 2, 0.0, c, 2, herm=True)
    _close(c, _lv(g["zher2k"]["c"]))
    b = _lv(g["dtrmm"]["b"])
    blas.trmm("L", "U", "N", "N", 2, 2, 1.0, _lv(g["dtrmm"]["a"]), 2, b, 2)
    _close(b, _lv(g["dtrmm"]["b_out"]))
    b = _lv(g["dtrsm"]["b"])
    blas.trsm("L", "U", "N", "N", 2, 2, 1.0, _lv(g["dtrsm"]["a"]), 2, b, 2)
    _close(b, _lv(g["dtrsm"]["b_out"]))


def _rm(vals):
    """Row-major 2 x 2 buffer (C-contiguous) from the reference's flat list."""
    if isinstance(vals[0], list):
        return np.ascontiguousarray(np.array([complex(r, i) for r, i in vals], np.complex128).reshape(2, 2))
    return np.ascontiguousarray(np.array(vals, np.float64).reshape(2, 2))


def test_cblas_row_major_level3_known_answers(blas):
    """cblas_dtrmm / cblas_dtrsm / cblas_dsyr2k / cblas_zher2k in row-major layout reproduce the
    reference's answers (test/abi/cblas_compat_test.zig:596-658), the untouched triangle included."""
    g = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())["cblas_level3_row_major"]
    R, L, U, N, NU = blas.CblasRowMajor, blas.CblasLeft, blas.CblasUpper, blas.CblasNoTrans, blas.CblasNonUnit
    b = _rm(g["dtrmm"]["b"])
    blas.cblas_trmm(R, L, U, N, NU, 2, 2, 1.0, _rm(g["dtrmm"]["a"]), 2, b, 2)
    _close(b, _rm(g["dtrmm"]["b_out"]))
    b = _rm(g["dtrsm"]["b"])
    blas.cblas_dtrsm(R, L, U, N, NU, 2, 2, 1.0, _rm(g["dtrsm"]["a"]), 2, b, 2)
    _close(b, _rm(g["dtrsm"]["b_out"]))
    c = _rm(g["dsyr2k"]["c0"])
    blas.cblas_syr2k(R, U, N, 2, 2, 1.0, _rm(g["dsyr2k"]["a"]), 2, _rm(g["dsyr2k"]["b"]), 2, 0.0, c, 2)
    _close(c, _rm(g["dsyr2k"]["c"]))
    c = _rm(g["zher2k"]["c0"])
    blas.cblas_syr2k_c(R, U, N, 2, 2, 1.0, _rm(g["zher2k"]["a"]), 2, _rm(g["zher2k"]["b"]), 2, 0.0, c, 2, herm=True)
    _close(c, _rm(g["zher2k"]["c"]))
