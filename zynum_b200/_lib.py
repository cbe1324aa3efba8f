"""ctypes loader for libzynum_blas_gpu.so (the C ABI of the GPU backend).

The product path has no fallback: if the shared library is missing or does
not load, every call raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libzynum_blas_gpu.so"
_lib = None


class ZynumGpuError(RuntimeError):
    """A GPU entry point returned a non-zero status."""


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m zynum_b200.build` "
            "(the GPU backend has no CPU fallback)")
    L = C.CDLL(str(LIB_PATH))
    _declare(L)
    _lib = L
    return L


P = C.c_void_p
I32P = C.POINTER(C.c_int32)


def _declare(L: C.CDLL) -> None:
    ch, i, d, f = C.c_char, C.c_int, C.c_double, C.c_float
    cp = C.c_char_p
    L.xerbla_.argtypes = [cp, I32P]
    L.lsame_.argtypes = [cp, cp]
    L.lsame_.restype = i
    L.zynum_blas_shutdown.argtypes = []
    # Fortran GEMM: everything by pointer
    for name in ("sgemm_", "dgemm_"):
        getattr(L, name).argtypes = [cp, cp, I32P, I32P, I32P, P, P, I32P, P, I32P, P, P, I32P]
        getattr(L, name).restype = None
    L.cblas_dgemm.argtypes = [i, i, i, i, i, i, d, P, i, P, i, d, P, i]
    L.cblas_sgemm.argtypes = [i, i, i, i, i, i, f, P, i, P, i, f, P, i]
    for name in ("cgemm_", "zgemm_"):
        getattr(L, name).argtypes = [cp, cp, I32P, I32P, I32P, P, P, I32P, P, I32P, P, P, I32P]
        getattr(L, name).restype = None
    for name in ("cblas_cgemm", "cblas_zgemm"):
        getattr(L, name).argtypes = [i, i, i, i, i, i, P, P, i, P, i, P, P, i]
        getattr(L, name).restype = None
    for name in ("zynum_blas_gpu_zgemm_device", "zynum_blas_gpu_cgemm_device"):
        getattr(L, name).argtypes = [ch, ch, i, i, i, P, P, i, P, i, P, P, i, P]
        getattr(L, name).restype = i
    for name, T in (("dtrsm_", d), ("strsm_", f)):
        getattr(L, name).argtypes = [cp, cp, cp, cp, I32P, I32P, P, P, I32P, P, I32P]
        getattr(L, name).restype = None
    for name in ("dsyrk_", "ssyrk_"):
        getattr(L, name).argtypes = [cp, cp, I32P, I32P, P, P, I32P, P, P, I32P]
        getattr(L, name).restype = None
    L.cblas_dtrsm.argtypes = [i, i, i, i, i, i, i, d, P, i, P, i]
    L.cblas_strsm.argtypes = [i, i, i, i, i, i, i, f, P, i, P, i]
    L.cblas_dsyrk.argtypes = [i, i, i, i, i, d, P, i, d, P, i]
    L.cblas_ssyrk.argtypes = [i, i, i, i, i, f, P, i, f, P, i]
    L.zynum_blas_gpu_dtrsm_device.argtypes = [ch, ch, ch, ch, i, i, d, P, i, P, i, P]
    L.zynum_blas_gpu_strsm_device.argtypes = [ch, ch, ch, ch, i, i, f, P, i, P, i, P]
    L.zynum_blas_gpu_dsyrk_device.argtypes = [ch, ch, i, i, d, P, i, d, P, i, P]
    L.zynum_blas_gpu_ssyrk_device.argtypes = [ch, ch, i, i, f, P, i, f, P, i, P]
    L.zynum_blas_gpu_dtrsm_inverse_bytes.argtypes = [i]
    L.zynum_blas_gpu_dtrsm_inverse_bytes.restype = C.c_size_t
    L.zynum_blas_gpu_dtrsm_inverse_device.argtypes = [ch, ch, i, P, i, P, P]
    L.zynum_blas_gpu_dtrsm_with_inverse_device.argtypes = [ch, ch, ch, ch, i, i, d, P, i, P, i, P, P]
    for name in ("zynum_blas_gpu_dtrsm_device", "zynum_blas_gpu_strsm_device", "zynum_blas_gpu_dsyrk_device",
                 "zynum_blas_gpu_ssyrk_device", "zynum_blas_gpu_dtrsm_inverse_device",
                 "zynum_blas_gpu_dtrsm_with_inverse_device"):
        getattr(L, name).restype = i
    for name in ("ztrsm_", "ctrsm_"):
        getattr(L, name).argtypes = [cp, cp, cp, cp, I32P, I32P, P, P, I32P, P, I32P]
        getattr(L, name).restype = None
    for name in ("zsyrk_", "csyrk_"):
        getattr(L, name).argtypes = [cp, cp, I32P, I32P, P, P, I32P, P, P, I32P]
        getattr(L, name).restype = None
    for name in ("cblas_ztrsm", "cblas_ctrsm"):
        getattr(L, name).argtypes = [i, i, i, i, i, i, i, P, P, i, P, i]
        getattr(L, name).restype = None
    for name in ("cblas_zsyrk", "cblas_csyrk"):
        getattr(L, name).argtypes = [i, i, i, i, i, P, P, i, P, P, i]
        getattr(L, name).restype = None
    for name in ("zynum_blas_gpu_ztrsm_device", "zynum_blas_gpu_ctrsm_device"):
        getattr(L, name).argtypes = [ch, ch, ch, ch, i, i, P, P, i, P, i, P]
        getattr(L, name).restype = i
    for name in ("zynum_blas_gpu_zsyrk_device", "zynum_blas_gpu_csyrk_device"):
        getattr(L, name).argtypes = [ch, ch, i, i, P, P, i, P, P, i, P]
        getattr(L, name).restype = i
    for name in ("zynum_blas_gpu_zsymm_device", "zynum_blas_gpu_csymm_device", "zynum_blas_gpu_zhemm_device",
                 "zynum_blas_gpu_chemm_device"):
        getattr(L, name).argtypes = [ch, ch, i, i, P, P, i, P, i, P, P, i, P]
        getattr(L, name).restype = i
    for name in ("zynum_blas_gpu_ztrmm_device", "zynum_blas_gpu_ctrmm_device"):
        getattr(L, name).argtypes = [ch, ch, ch, ch, i, i, P, P, i, P, i, P]
        getattr(L, name).restype = i
    for name in ("zynum_blas_gpu_zsyr2k_device", "zynum_blas_gpu_csyr2k_device"):
        getattr(L, name).argtypes = [ch, ch, i, i, P, P, i, P, i, P, P, i, P]
        getattr(L, name).restype = i
    L.zynum_blas_gpu_zher2k_device.argtypes = [ch, ch, i, i, P, P, i, P, i, d, P, i, P]
    L.zynum_blas_gpu_cher2k_device.argtypes = [ch, ch, i, i, P, P, i, P, i, f, P, i, P]
    L.zynum_blas_gpu_zherk_device.argtypes = [ch, ch, i, i, d, P, i, d, P, i, P]
    L.zynum_blas_gpu_cherk_device.argtypes = [ch, ch, i, i, f, P, i, f, P, i, P]
    for name in ("zynum_blas_gpu_zher2k_device", "zynum_blas_gpu_cher2k_device", "zynum_blas_gpu_zherk_device",
                 "zynum_blas_gpu_cherk_device"):
        getattr(L, name).restype = i
    for name in ("dsymm_", "ssymm_", "zsymm_", "csymm_", "zhemm_", "chemm_"):
        getattr(L, name).argtypes = [cp, cp, I32P, I32P, P, P, I32P, P, I32P, P, P, I32P]
        getattr(L, name).restype = None
    for name in ("ztrmm_", "ctrmm_"):
        getattr(L, name).argtypes = [cp, cp, cp, cp, I32P, I32P, P, P, I32P, P, I32P]
        getattr(L, name).restype = None
    for name in ("zsyr2k_", "csyr2k_", "zher2k_", "cher2k_"):
        getattr(L, name).argtypes = [cp, cp, I32P, I32P, P, P, I32P, P, I32P, P, P, I32P]
        getattr(L, name).restype = None
    for name in ("zherk_", "cherk_"):
        getattr(L, name).argtypes = [cp, cp, I32P, I32P, P, P, I32P, P, P, I32P]
        getattr(L, name).restype = None
    for name in ("cblas_zsymm", "cblas_csymm", "cblas_zhemm", "cblas_chemm"):
        getattr(L, name).argtypes = [i, i, i, i, i, P, P, i, P, i, P, P, i]
        getattr(L, name).restype = None
    for name in ("cblas_ztrmm", "cblas_ctrmm"):
        getattr(L, name).argtypes = [i, i, i, i, i, i, i, P, P, i, P, i]
        getattr(L, name).restype = None
    for name in ("cblas_zsyr2k", "cblas_csyr2k"):
        getattr(L, name).argtypes = [i, i, i, i, i, P, P, i, P, i, P, P, i]
        getattr(L, name).restype = None
    L.cblas_zher2k.argtypes = [i, i, i, i, i, P, P, i, P, i, d, P, i]
    L.cblas_cher2k.argtypes = [i, i, i, i, i, P, P, i, P, i, f, P, i]
    L.cblas_zherk.argtypes = [i, i, i, i, i, d, P, i, d, P, i]
    L.cblas_cherk.argtypes = [i, i, i, i, i, f, P, i, f, P, i]
    for name in ("cblas_zher2k", "cblas_cher2k", "cblas_zherk", "cblas_cherk"):
        getattr(L, name).restype = None
    for name in ("dtrmm_", "strmm_"):
        getattr(L, name).argtypes = [cp, cp, cp, cp, I32P, I32P, P, P, I32P, P, I32P]
        getattr(L, name).restype = None
    for name in ("dsyr2k_", "ssyr2k_"):
        getattr(L, name).argtypes = [cp, cp, I32P, I32P, P, P, I32P, P, I32P, P, P, I32P]
        getattr(L, name).restype = None
    L.cblas_dsymm.argtypes = [i, i, i, i, i, d, P, i, P, i, d, P, i]
    L.cblas_ssymm.argtypes = [i, i, i, i, i, f, P, i, P, i, f, P, i]
    L.cblas_dtrmm.argtypes = [i, i, i, i, i, i, i, d, P, i, P, i]
    L.cblas_strmm.argtypes = [i, i, i, i, i, i, i, f, P, i, P, i]
    L.cblas_dsyr2k.argtypes = [i, i, i, i, i, d, P, i, P, i, d, P, i]
    L.cblas_ssyr2k.argtypes = [i, i, i, i, i, f, P, i, P, i, f, P, i]
    for name in ("cblas_dsymm", "cblas_ssymm", "cblas_dtrmm", "cblas_strmm", "cblas_dsyr2k", "cblas_ssyr2k"):
        getattr(L, name).restype = None
    L.zynum_blas_gpu_dsymm_device.argtypes = [ch, ch, i, i, d, P, i, P, i, d, P, i, P]
    L.zynum_blas_gpu_ssymm_device.argtypes = [ch, ch, i, i, f, P, i, P, i, f, P, i, P]
    L.zynum_blas_gpu_dtrmm_device.argtypes = [ch, ch, ch, ch, i, i, d, P, i, P, i, P]
    L.zynum_blas_gpu_strmm_device.argtypes = [ch, ch, ch, ch, i, i, f, P, i, P, i, P]
    L.zynum_blas_gpu_dsyr2k_device.argtypes = [ch, ch, i, i, d, P, i, P, i, d, P, i, P]
    L.zynum_blas_gpu_ssyr2k_device.argtypes = [ch, ch, i, i, f, P, i, P, i, f, P, i, P]
    for name in ("zynum_blas_gpu_dsymm_device", "zynum_blas_gpu_ssymm_device", "zynum_blas_gpu_dtrmm_device",
                 "zynum_blas_gpu_strmm_device", "zynum_blas_gpu_dsyr2k_device", "zynum_blas_gpu_ssyr2k_device"):
        getattr(L, name).restype = i
    L.zynum_blas_gpu_dgemmt_device.argtypes = [ch, ch, ch, i, i, d, P, i, P, i, d, P, i, P]
    L.zynum_blas_gpu_dgemmt_device.restype = i
    L.zynum_blas_gpu_dsymmetrize_device.argtypes = [ch, i, P, i, P]
    L.zynum_blas_gpu_dsymmetrize_device.restype = i
    IP = C.POINTER(C.c_int)
    L.zynum_blas_gpu_gemm_batch_create.argtypes = [C.POINTER(P), i, ch, ch, i, P, P, P, i]
    L.zynum_blas_gpu_gemm_batch_create.restype = i
    L.zynum_blas_gpu_trsm_batch_create.argtypes = [C.POINTER(P), i, ch, ch, ch, ch, i, P, P]
    L.zynum_blas_gpu_trsm_batch_create.restype = i
    L.zynum_blas_gpu_batch_destroy.argtypes = [P]
    L.zynum_blas_gpu_batch_destroy.restype = None
    L.zynum_blas_gpu_batch_info.argtypes = [P, IP, IP, P]
    L.zynum_blas_gpu_batch_info.restype = i
    L.zynum_blas_gpu_dgemm_batch_run.argtypes = [P, d, P, P, P, P, d, P, P, P, i]
    L.zynum_blas_gpu_sgemm_batch_run.argtypes = [P, f, P, P, P, P, f, P, P, P, i]
    L.zynum_blas_gpu_dtrsm_batch_run.argtypes = [P, d, P, P, P, P, P, i]
    L.zynum_blas_gpu_strsm_batch_run.argtypes = [P, f, P, P, P, P, P, i]
    for name in ("zynum_blas_gpu_dgemm_batch_run", "zynum_blas_gpu_sgemm_batch_run",
                 "zynum_blas_gpu_dtrsm_batch_run", "zynum_blas_gpu_strsm_batch_run"):
        getattr(L, name).restype = i
    L.zynum_blas_gpu_set_complex_method.argtypes = [i]
    L.zynum_blas_gpu_set_complex_method.restype = i
    L.zynum_blas_gpu_dgemm_device.argtypes = [ch, ch, i, i, i, d, P, i, P, i, d, P, i, P]
    L.zynum_blas_gpu_dgemm_device.restype = i
    L.zynum_blas_gpu_sgemm_device.argtypes = [ch, ch, i, i, i, f, P, i, P, i, f, P, i, P]
    L.zynum_blas_gpu_sgemm_device.restype = i
    L.zynum_blas_gpu_dgemm_noalloc_device.argtypes = [ch, ch, i, i, i, d, P, i, P, i, d, P, i, i, P]
    L.zynum_blas_gpu_dgemm_noalloc_device.restype = i
    for name in ("zynum_blas_gpu_set_dgemm_method", "zynum_blas_gpu_set_sgemm_method",
                 "zynum_blas_gpu_set_ozaki_slices", "zynum_blas_gpu_set_ozaki_scheme",
                 "zynum_blas_gpu_set_ozaki_moduli"):
        getattr(L, name).argtypes = [i]
        getattr(L, name).restype = i
    L.zynum_blas_gpu_ozaki_plan.argtypes = [i, i, i, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.zynum_blas_gpu_ozaki_plan.restype = i
    L.zynum_blas_gpu_ozaki_plan_ex.argtypes = [i, i, i, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.zynum_blas_gpu_ozaki_plan_ex.restype = i
    L.zynum_blas_gpu_last_error.argtypes = []
    L.zynum_blas_gpu_last_error.restype = cp
    L.zynum_blas_gpu_inject_fault.argtypes = [i, i]
    L.zynum_blas_gpu_inject_fault.restype = None
    L.zynum_blas_gpu_device_status.argtypes = [P]
    L.zynum_blas_gpu_device_status.restype = i
    L.zynum_blas_gpu_measure_pipe_rate.argtypes = [i, C.POINTER(C.c_double), P]
    L.zynum_blas_gpu_measure_pipe_rate.restype = i
    L.zynum_blas_gpu_profile.argtypes = [i]
    L.zynum_blas_gpu_profile.restype = i
    L.zynum_blas_gpu_profile_read.argtypes = [P, i]
    L.zynum_blas_gpu_profile_read.restype = i
    L.zynum_blas_gpu_launch_count.argtypes = []
    L.zynum_blas_gpu_launch_count.restype = C.c_longlong


def check(status: int, what: str) -> None:
    if status != 0:
        msg = load().zynum_blas_gpu_last_error().decode(errors="replace")
        if status > 0:
            raise ValueError(f"{what}: parameter number {status} had an illegal value")
        raise ZynumGpuError(f"{what} failed with status {status}: {msg}")
