"""Writes tests/golden/known_answers.json.

The reference (Zig 0.16) cannot be built or run in this image, so its golden
vectors are its literal known-answer tests, transcribed here with the file
and line each comes from (paths inside the Zynum project).  Matrices are
listed column-major, as the reference's arrays are.

Run: python tests/golden/make_golden.py
"""
import json
from pathlib import Path

KNOWN = {
    # test/abi/fortran_compat_test.zig:537-560 "dgemm column major no transpose"
    "dgemm_column_major_nn": {
        "source": "test/abi/fortran_compat_test.zig:537-560",
        "a": [1, 2, 3, 4, 5, 6],          # 2 x 3, lda 2
        "b": [7, 8, 9, 10, 11, 12],       # 3 x 2, ldb 3
        "c": [76, 100, 103, 136],         # 2 x 2
    },
    # test/abi/cblas_compat_test.zig:405-421 "cblas row-major dgemm wrapper"
    "cblas_dgemm_row_major": {
        "source": "test/abi/cblas_compat_test.zig:405-421",
        "a_row_major": [1, 3, 5, 2, 4, 6],      # 2 x 3, lda 3
        "b_row_major": [7, 10, 8, 11, 9, 12],   # 3 x 2, ldb 2
        "c_row_major": [76, 103, 100, 136],     # 2 x 2, ldc 2
    },
    # test/abi/fortran_compat_test.zig:1012-1046 "gemm beta zero and alpha zero isolate inactive NaNs"
    "gemm_nan_isolation": {
        "source": "test/abi/fortran_compat_test.zig:1012-1046",
        "a": [1, 2, 3, 4],
        "b": [5, 6, 7, 8],
        "c_beta0": [23, 34, 31, 46],
        "c_alpha0": [2, 4, 6, 8],
    },
    # test/abi/fortran_compat_test.zig:1048-1074 "complex gemm beta zero and alpha zero isolate inactive NaNs"
    "zgemm_nan_isolation": {
        "source": "test/abi/fortran_compat_test.zig:1048-1074",
        "a": [2, 1],
        "b": [3, -1],
        "c_beta0": [7, 1],
        "c_alpha0": [11, 2],
    },
    # test/api/zynum_test.zig:28-41 matrixMultiply 2x3 * 3x2
    "matrix_multiply_typed": {
        "source": "test/api/zynum_test.zig:28-41",
        "c": [76, 100, 103, 136],
    },
    # test/abi/fortran_compat_test.zig:1676-1800 "level3 symmetric hermitian rank-k and triangular
    # fallbacks": 2 x 2 problems, ld 2, side L, uplo U, trans N, alpha 1, beta 0 (complex values as
    # [re, im]; C entries outside the updated triangle keep their sentinel)
    "level3_known_answers": {
        "source": "test/abi/fortran_compat_test.zig:1676-1800",
        "dsymm": {"a": [1, 777, 2, 3], "b": [4, 6, 5, 7], "c": [16, 26, 19, 31]},
        "zhemm": {"a": [[1, 99], [777, 777], [2, 1], [3, -7]], "b": [[1, 0], [0, 0], [0, 0], [1, 0]],
                  "c": [[1, 0], [2, -1], [2, 1], [3, 0]]},
        "dsyrk": {"a": [1, 3, 2, 4], "c0": [0, 777, 0, 0], "c": [5, 777, 11, 25]},
        "zherk": {"a": [[1, 1], [3, 0], [2, 0], [-1, 1]], "c0": [[0, 0], [777, 777], [0, 0], [0, 0]],
                  "c": [[6, 0], [777, 777], [1, 1], [11, 0]]},
        "dsyr2k": {"a": [1, 3, 2, 4], "b": [5, 7, 6, 8], "c0": [0, 777, 0, 0], "c": [34, 777, 62, 106]},
        "zher2k": {"a": [[1, 0], [3, 0], [2, 0], [4, 0]], "b": [[5, 0], [7, 0], [6, 0], [8, 0]],
                   "c0": [[0, 0], [777, 777], [0, 0], [0, 0]], "c": [[34, 0], [777, 777], [62, 0], [106, 0]]},
        "dtrmm": {"a": [1, 777, 2, 3], "b": [4, 6, 5, 7], "b_out": [16, 18, 19, 21]},
        "dtrsm": {"a": [1, 777, 2, 3], "b": [16, 18, 19, 21], "b_out": [4, 6, 5, 7]},
    },
    # test/abi/cblas_compat_test.zig:596-658 "cblas row-major level3 triangular and rank2k wrappers":
    # row-major 2 x 2 buffers (ld 2), side L, uplo U, trans N, alpha 1, beta 0
    "cblas_level3_row_major": {
        "source": "test/abi/cblas_compat_test.zig:596-658",
        "dtrmm": {"a": [1, 2, 777, 3], "b": [4, 5, 6, 7], "b_out": [16, 19, 18, 21]},
        "dtrsm": {"a": [1, 2, 777, 3], "b": [16, 19, 18, 21], "b_out": [4, 5, 6, 7]},
        "dsyr2k": {"a": [1, 2, 3, 4], "b": [5, 6, 7, 8], "c0": [0, 0, 777, 0], "c": [34, 62, 777, 106]},
        "zher2k": {"a": [[1, 0], [2, 0], [3, 0], [4, 0]], "b": [[5, 0], [6, 0], [7, 0], [8, 0]],
                   "c0": [[0, 0], [0, 0], [777, 7], [0, 0]], "c": [[34, 0], [62, 0], [777, 7], [106, 0]]},
    },
    # tolerances the reference's tests use (gemm_registry_test.zig:198-202,
    # fortran_compat_test.zig:371/406, gemm_sweep.zig:247-258)
    "tolerances": {
        "f64_abs": 1e-10, "f32_abs": 1e-3,
        "registry_f64": [2e-12, 2e-12], "registry_f32": [4e-4, 4e-4],
        "bench_f64_per_k": 1e-9, "bench_f32_per_k": 1e-3,
        "sentinel_f64": -999.0, "sentinel_f32": -777.0,
    },
}

if __name__ == "__main__":
    out = Path(__file__).with_name("known_answers.json")
    out.write_text(json.dumps(KNOWN, indent=1) + "\n")
    print(out)
