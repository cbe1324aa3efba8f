"""Build the CPU oracle (test infrastructure only) into oracle/lib/.

  liboracle.so         plain-C restatement of the reference's scalar GEMM /
                       TRSM / SYRK semantics plus a double-double GEMM
                       (zynum_oracle.c), compiled with -ffp-contract=off.
  libzynum_cpu.so      C++ restatement of the reference's x86-64 packed-SIMD
                       GEMM path and its CPU thread planner
                       (zynum_cpu_restated.cpp): the timed CPU baseline.

The reference itself is Zig 0.16 and cannot be compiled in this image (no
`zig` toolchain), so there is no oracle/_ref build.

Usage: python oracle/build.py [--force]
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib"

TARGETS = [
    (HERE / "zynum_oracle.c", LIB / "liboracle.so",
     ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared"], ["-lm"]),
    (HERE / "zynum_cpu_restated.cpp", LIB / "libzynum_cpu.so",
     ["g++", "-O3", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-pthread"], []),
]


def build(force: bool = False) -> list[Path]:
    LIB.mkdir(parents=True, exist_ok=True)
    out = []
    for src, lib, flags, libs in TARGETS:
        if not src.exists():
            continue
        if force or not lib.exists() or lib.stat().st_mtime < src.stat().st_mtime:
            cmd = [*flags, str(src), "-o", str(lib), *libs]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"oracle build failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        out.append(lib)
    return out


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv):
        print(p)
