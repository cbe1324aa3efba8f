"""CPU oracle for the Zynum GEMM path (test infrastructure; never imported by zynum_b200)."""
