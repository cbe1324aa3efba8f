"""Writes tests/golden/reference_abi_subset.json: the reference's ABI manifest
entries (include/zynum/blas/abi_manifest.json, written by the reference's
tools/generate_compat_headers.zig) for the Level-3 families and the error /
shutdown helpers, i.e. the exports a GPU Level-3 library can stand in for.
The names, argument names and Zig argument types are copied as interface data.

Run in a checkout that holds the reference (path as the first argument):
    python tests/golden/make_abi_subset.py /path/to/zynum
"""
import json
import re
import sys
from pathlib import Path

FAMILIES = re.compile(r"^(cblas_)?[sdcz](gemm|symm|hemm|syrk|herk|syr2k|her2k|trmm|trsm)_?$")
HELPERS = {"xerbla_", "lsame_", "zynum_blas_shutdown", "zynum_blas_shutdown_"}


def main(root: str) -> None:
    src = Path(root) / "include" / "zynum" / "blas" / "abi_manifest.json"
    d = json.loads(src.read_text())
    out = {"source": "include/zynum/blas/abi_manifest.json", "schema": d["schema"],
           "generator": d["generator"], "blas_integer_abi": d["blas_integer_abi"],
           "blas_integer_bits": d["blas_integer_bits"]}
    for part in ("fortran", "cblas"):
        keep = [e for e in d[part]["exports"] if FAMILIES.match(e["name"]) or e["name"] in HELPERS]
        out[part] = {"reference_export_count": d[part]["export_count"], "exports": keep}
    dst = Path(__file__).with_name("reference_abi_subset.json")
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(dst, sum(len(out[p]["exports"]) for p in ("fortran", "cblas")))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else ".")
