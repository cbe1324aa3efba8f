"""Writes include/abi_manifest.json from include/zynum_blas_gpu.h, in the
reference library's manifest format (schema 1: per export its name, Fortran
procedure name, return type and argument names / Zig types), so the two ABIs
can be compared entry by entry.  Exports are grouped as the reference groups
them: "fortran" (trailing-underscore routines and the xerbla / lsame /
shutdown helpers), "cblas", and "gpu" (the zynum_blas_gpu_* entry points this
library adds, with C types only).

With --reference FILE (a manifest subset, e.g. tests/golden/reference_abi_subset.json)
it also writes include/abi_manifest_diff.md: which reference exports this
library provides with the same argument list, which differ, which it does
not provide, and which it adds.

Run: python include/make_abi_manifest.py [--reference tests/golden/reference_abi_subset.json]
"""
from __future__ import annotations

import argparse
import json
import re
from pathlib import Path

HERE = Path(__file__).resolve().parent
HEADER = HERE / "zynum_blas_gpu.h"
SCALAR_NAMES = {"alpha", "beta"}
BASE = {"double": "f64", "float": "f32", "char": "u8", "int": "c_int", "zynum_blas_int": "BlasInt",
        "int64_t": "i64", "int32_t": "i32", "size_t": "usize"}
HELPERS = {"xerbla_", "lsame_", "zynum_blas_shutdown", "zynum_blas_shutdown_"}


def declarations(text: str):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    for m in re.finditer(r"ZYNUM_BLAS_GPU_API\s+([^;{]*?)\b(\w+)\s*\(([^)]*)\)\s*;", text, flags=re.S):
        ret, name, args = " ".join(m.group(1).split()), m.group(2), " ".join(m.group(3).split())
        params = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        yield ret, name, params


def split_param(p: str):
    m = re.match(r"^(.*?)(\w+)$", p)
    ctype, pname = " ".join(m.group(1).replace("*", " * ").split()), m.group(2)
    return ctype.replace(" *", "*").replace("* ", "*").replace("*const", "* const"), pname


def complex_type(routine: str):
    base = routine[len("cblas_"):] if routine.startswith("cblas_") else routine
    return {"z": "ComplexF64", "c": "ComplexF32"}.get(base[:1])


def zig_type(ctype: str, pname: str, routine: str):
    """The Zig type the reference's manifest would give this C parameter (None if unmappable)."""
    t = ctype.replace(" ", "")
    const = t.startswith("const")
    core = t[5:] if const else t
    stars = core.count("*")
    core = core.replace("*", "").replace("const", "")
    if stars == 0:
        return BASE.get(core)
    if stars != 1:
        return None
    if core == "void":
        elt = complex_type(routine)
        if elt is None:
            return "?*anyopaque"
    elif core == "char":
        return "[*]const u8" if const else "[*]u8"
    else:
        elt = BASE.get(core)
        if elt is None:
            return None
    if core == "zynum_blas_int" or pname in SCALAR_NAMES:
        return ("*const " if const else "*") + elt
    return ("[*]const " if const else "[*]") + elt


def entry(ret: str, name: str, params):
    args = []
    for p in params:
        ctype, pname = split_param(p)
        args.append({"name": pname, "zig_type": zig_type(ctype, pname, name), "c_type": ctype})
    e = {"name": name}
    if name.endswith("_") and not name.startswith("zynum_blas_gpu_"):
        e["procedure_name"] = name[:-1]
    e["return_zig"] = {"void": "void", "int": "c_int"}.get(ret, None)
    e["return_c"] = ret
    e["args"] = args
    return e


def build_manifest():
    parts = {"fortran": [], "cblas": [], "gpu": []}
    for ret, name, params in declarations(HEADER.read_text()):
        e = entry(ret, name, params)
        if name.startswith("cblas_"):
            parts["cblas"].append(e)
        elif name.startswith("zynum_blas_gpu_"):
            parts["gpu"].append(e)
        elif name.endswith("_") or name in HELPERS:
            parts["fortran"].append(e)
        else:
            parts["gpu"].append(e)
    out = {"schema": 1, "generator": "include/make_abi_manifest.py", "blas_integer_abi": "LP64",
           "blas_integer_bits": 32}
    for k, v in parts.items():
        out[k] = {"source": ["include/zynum_blas_gpu.h"], "export_count": len(v), "exports": v}
    return out


def diff(ours, ref):
    """Per section: same argument types, different, reference-only, ours-only."""
    report = {}
    for part in ("fortran", "cblas"):
        mine = {e["name"]: e for e in ours[part]["exports"]}
        theirs = {e["name"]: e for e in ref[part]["exports"]}
        same, differ, renamed = [], [], []
        for name in sorted(set(mine) & set(theirs)):
            a, b = mine[name]["args"], theirs[name]["args"]
            ta = [x["zig_type"] for x in a]
            tb = [x["zig_type"] for x in b]
            if ta == tb and mine[name]["return_zig"] == theirs[name]["return_zig"]:
                same.append(name)
                names_a, names_b = [x["name"] for x in a], [x["name"] for x in b]
                if names_a != names_b:
                    renamed.append((name, [(x, y) for x, y in zip(names_a, names_b) if x != y]))
            else:
                differ.append((name, ta, tb))
        report[part] = {"same": same, "differ": differ, "renamed": renamed,
                        "reference_only": sorted(set(theirs) - set(mine)),
                        "ours_only": sorted(set(mine) - set(theirs))}
    return report


def write_diff_md(report, ours, path: Path):
    lines = ["# ABI manifest diff: libzynum_blas_gpu against the reference's Level-3 exports", "",
             "Generated by `python include/make_abi_manifest.py --reference "
             "tests/golden/reference_abi_subset.json`; the subset holds the reference manifest's "
             "entries for the Level-3 families (gemm, symm, hemm, syrk, herk, syr2k, her2k, trmm, trsm) "
             "and the xerbla / lsame / shutdown helpers. Argument lists are compared by Zig type and "
             "order; argument names are informational.", ""]
    for part in ("fortran", "cblas"):
        r = report[part]
        lines += [f"## {part}", "",
                  f"- same argument types and order ({len(r['same'])}): " + ", ".join(f"`{n}`" for n in r["same"]),
                  f"- different ({len(r['differ'])}): " + (", ".join(f"`{n}`" for n, _, _ in r["differ"]) or "none"),
                  f"- reference only, not provided by the GPU library ({len(r['reference_only'])}): "
                  + (", ".join(f"`{n}`" for n in r["reference_only"]) or "none"),
                  f"- GPU library only ({len(r['ours_only'])}): " + (", ".join(f"`{n}`" for n in r["ours_only"]) or "none"),
                  ""]
        if r["renamed"]:
            lines.append("Argument names that differ (same types):")
            lines.append("")
            for n, pairs in r["renamed"]:
                lines.append(f"- `{n}`: " + ", ".join(f"{a} (reference: {b})" for a, b in pairs))
            lines.append("")
    lines += ["## gpu", "",
              f"{ours['gpu']['export_count']} `zynum_blas_gpu_*` entry points (device pointers + stream, "
              "method switches, batching, profiling); no counterpart in the reference.", ""]
    path.write_text("\n".join(lines))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", help="reference manifest (or subset) to diff against")
    args = ap.parse_args(argv)
    man = build_manifest()
    (HERE / "abi_manifest.json").write_text(json.dumps(man, indent=1) + "\n")
    if args.reference:
        ref = json.loads(Path(args.reference).read_text())
        write_diff_md(diff(man, ref), man, HERE / "abi_manifest_diff.md")


if __name__ == "__main__":
    main()
