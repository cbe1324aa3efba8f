"""Benchmark of the Zynum B200 GEMM backend.

Headline workload: DGEMM C = A B, M = N = K = 8192, column-major FP64,
entries u * 10^e, u ~ U[-1, 1], e ~ U[-phi, phi] with phi = 0 (seeded,
synthetic), alpha = 1, beta = 0.  Metric: effective DGEMM TFLOP/s
(2 * 8192^3 flop per call) of the Ozaki-emulated DGEMM, with the native FP64
DGEMM measured in the same run on the same inputs and both errors stated
against a double-double oracle on sampled entries.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` times the device entry point with inputs resident in HBM (3 x 512 MiB,
larger than the 126 MB L2, so no flush is needed).  `e2e` times the Fortran
`dgemm_` entry point on pinned host buffers: host->device copies of A and B,
the GEMM, and the device->host copy of C are inside the timed region.
With --gpus N > 1 every rank runs an independent replica (GEMM does not shard
without an exchange step; the product is single-GPU).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
FP64_NOMINAL_TFLOPS = 148 * 128 * 1.965e9 / 1e12  # 64 DFMA/clk/SM at the 1965 MHz max clock
FP32_NOMINAL_TFLOPS = 148 * 256 * 1.965e9 / 1e12  # 128 FFMA/clk/SM at the 1965 MHz max clock
METRIC = "DGEMM TFLOP/s @8192^3: Ozaki-emulated vs native FP64 at equal error; batch GFLOP/s"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the dominant kernel on the
# 8192^3 headline workload, one launch each in one-pass ncu captures (profiles/ozaki_crt_umma_gemm_dram_8192.md):
# CRT modular-product GEMM 5.38 GB + 1.06 GB; native TMA DGEMM 15.82 GB + 0.53 GB.
TRAFFIC_8192 = {"crt": 5.38e9 + 1.06e9, "native": 15.82e9 + 0.53e9}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        d["_source"] = "measured"
        return d
    d = dict(PEAKS_FALLBACK)
    d["_source"] = "fallback"
    return d


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"zb_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, window=None):
        """Median SM clock under load and the throttle reasons seen; `window` = (t0, t1) wall-clock
        seconds (time.time()) restricts the samples to a timed region."""
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        import datetime
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                clk = float(parts[2])
                mx = float(parts[3])
                pw = float(parts[4])
            except ValueError:
                continue
            if window is not None and not (window[0] <= ts <= window[1]):
                continue
            sm.append(clk)
            power.append(pw)
            for nm, v in zip(names, parts[6:10]):
                if v.lower() == "active":
                    reasons.add(nm)
        load = [x for x in sm if mx and x > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "power_w": statistics.median(power) if power else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ inputs
def make_inputs(torch, n, phi, seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(seed)

    def one():
        u = torch.rand((n, n), generator=g, device=device, dtype=torch.float64) * 2 - 1
        if phi:
            e = torch.rand((n, n), generator=g, device=device, dtype=torch.float64) * 2 * phi - phi
            u = u * torch.pow(10.0, e)
        return u

    return one(), one()


def sampled_error(oracle, a_h, b_h, c_h, n, count=2048, seed=1):
    """Max / median relative error of c against a double-double oracle at sampled (i, j)."""
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, n, count)
    cols = rng.integers(0, n, count)
    hi, lo, ab = oracle.ddgemm_sampled("N", "N", n, a_h, n, b_h, n, rows, cols)
    exact = hi + lo
    got = c_h[rows, cols]
    rel = np.abs(got - exact) / np.maximum(np.abs(exact), 1e-300)
    rel_ab = np.abs(got - exact) / np.maximum(ab, 1e-300)
    return {"max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
            "max_err_over_abs_ab": float(rel_ab.max()), "samples": int(count)}


# ------------------------------------------------------------- CPU baseline
def cpu_gemm_lib():
    import ctypes as C
    from oracle import build as ob
    ob.build()
    L = C.CDLL(str(ROOT / "oracle" / "lib" / "libzynum_cpu.so"))
    L.zynum_cpu_dgemm.argtypes = [C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int,
                                  C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int]
    L.zynum_cpu_threads.argtypes = [C.c_int, C.c_int, C.c_int]
    L.zynum_cpu_threads.restype = C.c_int
    return L


def cpu_baseline(n, slab, min_seconds=10.0, max_reps=20):
    """Restated Zynum CPU DGEMM on an n x slab x n slab of the headline problem."""
    L = cpu_gemm_lib()
    rng = np.random.default_rng(5)
    a = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    b = np.asfortranarray(rng.uniform(-1, 1, (n, slab)))
    c = np.zeros((n, slab), order="F")
    times = []
    t_end = time.perf_counter() + min_seconds
    while len(times) < max_reps and (len(times) < 2 or time.perf_counter() < t_end):
        t0 = time.perf_counter()
        L.zynum_cpu_dgemm(b"N", b"N", n, slab, n, 1.0, a.ctypes.data, n, b.ctypes.data, n, 0.0, c.ctypes.data, n)
        times.append(time.perf_counter() - t0)
    best = min(times)
    return {"value": 2.0 * n * slab * n / best / 1e12, "unit": "TFLOP/s",
            "cores": int(L.zynum_cpu_threads(n, slab, n)), "kind": "port",
            "sample": f"DGEMM {n}x{slab}x{n} column slab of the {n}^3 problem, best of {len(times)}; "
                      f"restated Zynum x86-64 packed-SIMD path (AVX-512 8x2x8 tile, planner column split)"}


# --------------------------------------------------------------- reference
def run_reference(args, rank, world):
    metric, unit = METRIC, "TFLOP/s"
    if rank != 0:
        return 0
    n = args.size
    slab = max(256, n // 4)
    L = cpu_gemm_lib()
    rng = np.random.default_rng(5)
    a = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    b = np.asfortranarray(rng.uniform(-1, 1, (n, slab)))
    c = np.zeros((n, slab), order="F")

    def step():
        L.zynum_cpu_dgemm(b"N", b"N", n, slab, n, 1.0, a.ctypes.data, n, b.ctypes.data, n, 0.0, c.ctypes.data, n)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    value = 2.0 * n * slab * n / dt / 1e12
    cores = int(L.zynum_cpu_threads(n, slab, n))
    line = {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic U[-1,1], seeded",
            "config": {"workload": f"DGEMM M=N=K={n} NN column-major FP64 alpha=1 beta=0",
                       "step_sample": f"{n}x{slab}x{n} column slab of the {n}^3 problem per step"},
            "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port",
                             "sample": f"{n}x{slab}x{n} slab per step; restated Zynum x86-64 packed-SIMD path "
                                       "(reference is Zig 0.16, no zig toolchain in the image)"},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ batches
def bench_batched(torch, blas, steps, warmup, seed=7, count=20000, tcount=5000, which=("dgemm", "sgemm", "dtrsm")):
    """20,000 variable-size DGEMM and SGEMM problems (M, N, K log-uniform on [8, 512], alpha 1, beta 0)
    and 5,000 left-lower TRSMs (n log-uniform on [16, 1024], 1..64 right-hand sides, L = tril(N(0,1))
    with diagonal 2 + |N(0,1)|), each batch one persistent launch replayed from a CUDA graph.
    count / tcount / which select a smaller sample of the same distributions (profiling)."""
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda")
    out = {}

    def lu(lo, hi, size):
        return np.exp(rng.uniform(np.log(lo), np.log(hi), size)).astype(np.int64)

    def carve(sizes, dtype, fill):
        """One flat buffer holding every problem's matrix; returns (buffer, pointer tensor)."""
        esz = 8 if dtype == torch.float64 else 4
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        buf = torch.empty(int(sizes.sum()) + 1, dtype=dtype, device=dev)
        fill(buf)
        ptrs = torch.from_numpy(offs * esz + buf.data_ptr()).to(dev)
        return buf, ptrs

    m, n, k = lu(8, 512, count), lu(8, 512, count), lu(8, 512, count)
    flops = float(np.sum(2.0 * m * n * k))
    for name, tdt in (("dgemm", torch.float64), ("sgemm", torch.float32)):
        if name not in which:
            continue
        g = torch.Generator(device=dev).manual_seed(seed)
        ufill = lambda b: b.uniform_(-1, 1, generator=g)  # noqa: E731
        A, pa = carve(m * k, tdt, ufill)
        B, pb = carve(k * n, tdt, ufill)
        Cb, pc = carve(m * n, tdt, lambda b: b.zero_())
        la = torch.from_numpy(m.astype(np.int32)).to(dev)
        lb = torch.from_numpy(k.astype(np.int32)).to(dev)
        t0 = time.perf_counter()
        batch = blas.GemmBatch(m, n, k, dtype="f64" if tdt == torch.float64 else "f32", tune=True)
        plan_s = time.perf_counter() - t0
        run = lambda: batch.run(1.0, pa, la, pb, lb, 0.0, pc, la, use_graph=True)  # noqa: E731
        ms = time_device(torch, run, steps, warmup, torch.cuda.current_stream())
        gf = flops / (ms * 1e-3) / 1e9
        # both batches run on the FP64 DMMA pipe (FP32 operands widened to FP64 in the tiles)
        peak = FP64_NOMINAL_TFLOPS
        roof = {"bound": "tensor", "achieved": gf / 1e3, "peak": peak, "unit": "TFLOP/s", "frac": gf / 1e3 / peak,
                "peak_source": "nominal FP64 DMMA pipe, 148 SMs x 128 flop/clk x 1.965 GHz"}
        if name == "sgemm":
            roof["frac_of_fp32_ffma"] = gf / 1e3 / FP32_NOMINAL_TFLOPS
        out[name] = {"problems": count, "gflop": flops / 1e9, "ms": ms, "gflops": gf,
                     "plan_and_tune_s": plan_s, **batch.info(), "roofline": roof}
        batch.close()
        del A, B, Cb
    if "dtrsm" not in which:
        return out
    tn = lu(16, 1024, tcount)
    tr = rng.integers(1, 65, tcount).astype(np.int64)
    tflops = float(np.sum(tn.astype(np.float64) ** 2 * tr))

    def lfill(buf):
        buf.normal_(0, 1)

    A, pa = carve(tn * tn, torch.float64, lfill)
    # make every A_q lower triangular with diagonal 2 + |N(0,1)| (upper part is never read)
    offs = np.concatenate([[0], np.cumsum(tn * tn)[:-1]])
    for q in range(tcount):
        a = A[offs[q]: offs[q] + tn[q] * tn[q]].view(int(tn[q]), int(tn[q]))
        a.diagonal().abs_().add_(2.0)
    B, pb = carve(tn * tr, torch.float64, lfill)
    la = torch.from_numpy(tn.astype(np.int32)).to(dev)
    batch = blas.TrsmBatch(tn, tr, dtype="f64", uplo="L")
    run = lambda: batch.run(1.0, pa, la, pb, la, use_graph=True)  # noqa: E731
    ms = time_device(torch, run, steps, warmup, torch.cuda.current_stream())
    gf = tflops / (ms * 1e-3) / 1e9
    out["dtrsm"] = {"problems": tcount, "gflop": tflops / 1e9, "ms": ms, "gflops": gf,
                    "note": "GFLOP = sum n^2 * nrhs", **batch.info(),
                    "roofline": {"bound": "tensor", "achieved": gf / 1e3, "peak": FP64_NOMINAL_TFLOPS,
                                 "unit": "TFLOP/s", "frac": gf / 1e3 / FP64_NOMINAL_TFLOPS,
                                 "peak_source": "nominal FP64 DMMA pipe (substitution steps are latency-bound)"}}
    batch.close()
    return out


# ----------------------------------------------------------- differentiation
def bench_differentiation(torch, steps, warmup, n=4096, r=512, seed=11):
    """X = TRSM(L, B), C = SYRK(X^T) = X^T X, loss = sum(sin(C)); forward + backward with X recomputed.
    L: n x n lower, off-diagonals N(0, 1/n), diagonal 1 + |N(0,1)|; B: n x r N(0,1)."""
    from zynum_b200 import autograd as ag
    from zynum_b200 import blas
    old = blas.set_dgemm_method(blas.METHOD_NATIVE)  # the adjoint workload runs native FP64
    g = torch.Generator(device="cuda").manual_seed(seed)
    L = torch.tril(torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64) / np.sqrt(n), -1)
    L += torch.diag(1 + torch.randn(n, generator=g, device="cuda", dtype=torch.float64).abs())
    B = torch.randn(n, r, generator=g, device="cuda", dtype=torch.float64)
    L.requires_grad_(True)
    B.requires_grad_(True)

    def step():
        loss = ag.chain_loss(L, B, recompute=True)
        torch.autograd.grad(loss, (L, B))

    ms = time_device(torch, step, steps, warmup, torch.cuda.current_stream())
    blas.set_dgemm_method(old)
    # nominal flops: forward TRSM n^2 r + SYRK r(r+1)n; backward TRSM (dB) n^2 r + recompute n^2 r
    # + dL = -tril(dB X^T) n^2 r + dX = X (G + G^T) 4 n r^2
    gflop = (3 * n * n * r + n * n * r + r * (r + 1) * n + 4 * n * r * r) / 1e9
    gf = gflop / (ms * 1e-3)
    return {"n": n, "nrhs": r, "ms_fwd_bwd": ms, "gflop_nominal": gflop, "gflops": gf,
            "recompute": True, "dgemm_method": "native FP64",
            "roofline": {"bound": "tensor", "achieved": gf / 1e3, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                         "frac": gf / 1e3 / FP64_NOMINAL_TFLOPS,
                         "peak_source": "nominal FP64 DMMA pipe; the chain's TRSM steps are latency-bound"}}


# ---------------------------------------------------------------- our arm
def time_device(torch, fn, steps, warmup, stream):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        fn()
    ev1.record(stream)
    ev1.synchronize()
    return ev0.elapsed_time(ev1) / steps


def precision_methods(torch, blas, orc, n, steps, warmup, stream, seed):
    """The rest of the precision configuration on the headline size: DGEMM with
    entries u * 10^e, e ~ U[-phi, phi], for phi = 4 and 8, Ozaki and native on the
    same inputs; SGEMM as a 3xBF16 split product, as INT8 CRT residue products (exact, one rounding) and
    native FP32 on U[-1, 1] data.
    Each: time per call (CUDA events, inputs resident) and max / median relative
    error against the double-double oracle on 2048 sampled entries."""
    dev = torch.device("cuda")
    flop = 2.0 * n ** 3
    out = {}
    for phi in (4.0, 8.0):
        A, B = make_inputs(torch, n, phi, seed, dev)
        C = torch.zeros((n, n), dtype=torch.float64, device=dev)
        a_h = np.asfortranarray(A.cpu().numpy().T)
        b_h = np.asfortranarray(B.cpu().numpy().T)
        for name, mid in (("ozaki", blas.METHOD_OZAKI), ("native", blas.METHOD_NATIVE)):
            blas.set_dgemm_method(mid)
            fn = lambda: blas.dgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n)  # noqa: E731
            ms = time_device(torch, fn, steps, warmup, stream)
            fn()
            torch.cuda.synchronize()
            err = sampled_error(orc, a_h, b_h, np.asfortranarray(C.cpu().numpy().T), n)
            out[f"{name}_phi{int(phi)}"] = {"phi": phi, "ms": ms, "tflops": flop / (ms * 1e-3) / 1e12,
                                            "error": err}
        del A, B, C
    blas.set_dgemm_method(blas.METHOD_NATIVE)
    g = torch.Generator(device=dev).manual_seed(seed + 99)
    A = torch.rand((n, n), generator=g, device=dev, dtype=torch.float32) * 2 - 1
    B = torch.rand((n, n), generator=g, device=dev, dtype=torch.float32) * 2 - 1
    C = torch.zeros((n, n), dtype=torch.float32, device=dev)
    a_h = np.asfortranarray(A.cpu().numpy().T.astype(np.float64))
    b_h = np.asfortranarray(B.cpu().numpy().T.astype(np.float64))
    for name, mid in (("sgemm_bf16x3", blas.SMETHOD_BF16X3), ("sgemm_ozaki", blas.SMETHOD_OZAKI),
                      ("sgemm_native", blas.SMETHOD_NATIVE)):
        blas.set_sgemm_method(mid)
        fn = lambda: blas.sgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n)  # noqa: E731
        ms = time_device(torch, fn, steps, warmup, stream)
        fn()
        torch.cuda.synchronize()
        err = sampled_error(orc, a_h, b_h, np.asfortranarray(C.cpu().numpy().T.astype(np.float64)), n)
        out[name] = {"ms": ms, "tflops": flop / (ms * 1e-3) / 1e12, "error": err,
                     "data": "U[-1,1] float32"}
    blas.set_sgemm_method(blas.SMETHOD_NATIVE)
    del A, B, C
    return out


def sweep_subset(torch, blas, stream, peaks, steps, warmup):
    """The shape-sweep rows the default line carries (each a few ms of work):
    tall-skinny 131072 x 64 x 64 FP64 / FP32 at beta 0 and 1 with achieved HBM GB/s
    against the measured copy bandwidth and the compute bound of the pipe it uses;
    K-dominant 256 x 256 x 262144 FP64 (split K); ZGEMM / CGEMM 4096^3 (4M and 3M)."""
    rows = []
    hbm = peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    for dt, tdt, fn, pipe in (("f64", torch.float64, blas.dgemm_device, FP64_NOMINAL_TFLOPS),
                              ("f32", torch.float32, blas.sgemm_device, FP32_NOMINAL_TFLOPS)):
        m, n, k = 131072, 64, 64
        g = torch.Generator(device="cuda").manual_seed(7)
        A = torch.rand((k, m), generator=g, device="cuda", dtype=tdt) * 2 - 1
        B = torch.rand((n, k), generator=g, device="cuda", dtype=tdt) * 2 - 1
        C = torch.rand((n, m), generator=g, device="cuda", dtype=tdt) * 2 - 1
        esz = 8 if dt == "f64" else 4
        for beta in (0.0, 1.0):
            f = lambda: fn("N", "N", m, n, k, 1.0, A, m, B, k, beta, C, m)  # noqa: E731
            ms = time_device(torch, f, max(20, steps), max(5, warmup), stream)
            byts = esz * (m * k + k * n + m * n * (2 if beta else 1))
            t_hbm = byts / (hbm * 1e9) * 1e3
            t_pipe = 2.0 * m * n * k / (pipe * 1e12) * 1e3
            rows.append({"shape": "tall-skinny", "dtype": dt, "m": m, "n": n, "k": k, "beta": beta, "ms": ms,
                         "gbs": byts / (ms * 1e-3) / 1e9, "frac_of_measured_hbm": byts / (ms * 1e-3) / 1e9 / hbm,
                         "tflops": 2.0 * m * n * k / (ms * 1e-3) / 1e12,
                         "bound": "hbm" if t_hbm >= t_pipe else ("fp64 dmma" if dt == "f64" else "fp32 ffma"),
                         "frac_of_bound": max(t_hbm, t_pipe) / ms})
        del A, B, C
    m, n, k = 256, 256, 262144
    g = torch.Generator(device="cuda").manual_seed(8)
    A = torch.rand((k, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    B = torch.rand((n, k), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    C = torch.zeros((n, m), device="cuda", dtype=torch.float64)
    f = lambda: blas.dgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m)  # noqa: E731
    ms = time_device(torch, f, max(5, steps // 2), max(3, warmup), stream)
    tf = 2.0 * m * n * k / (ms * 1e-3) / 1e12
    rows.append({"shape": "K-dominant", "dtype": "f64", "m": m, "n": n, "k": k, "beta": 0.0, "ms": ms, "tflops": tf,
                 "bound": "fp64 dmma", "frac_of_bound": tf / FP64_NOMINAL_TFLOPS})
    del A, B, C
    for dt, tdt, fn, real in (("z", torch.complex128, blas.zgemm_device, torch.float64),
                              ("c", torch.complex64, blas.cgemm_device, torch.float32)):
        nn = 4096
        g = torch.Generator(device="cuda").manual_seed(5)
        A = torch.complex(torch.rand((nn, nn), generator=g, device="cuda", dtype=real) * 2 - 1,
                          torch.rand((nn, nn), generator=g, device="cuda", dtype=real) * 2 - 1)
        B = torch.complex(torch.rand((nn, nn), generator=g, device="cuda", dtype=real) * 2 - 1,
                          torch.rand((nn, nn), generator=g, device="cuda", dtype=real) * 2 - 1)
        C = torch.zeros((nn, nn), device="cuda", dtype=tdt)
        for cm, cname in ((blas.COMPLEX_4M, "4M"), (blas.COMPLEX_3M, "3M")):
            old = blas.set_complex_method(cm)
            f = lambda: fn("N", "N", nn, nn, nn, 1.0, A, nn, B, nn, 0.0, C, nn)  # noqa: E731
            ms = time_device(torch, f, max(3, steps // 4), max(3, warmup), stream)
            blas.set_complex_method(old)
            rows.append({"shape": "square", "dtype": dt, "method": cname, "m": nn, "n": nn, "k": nn, "ms": ms,
                         "tflops": 8.0 * nn ** 3 / (ms * 1e-3) / 1e12, "note": "8mnk flops"})
        del A, B, C
    return rows


def _ozaki_desc(n):
    from zynum_b200 import ozaki_info
    info = ozaki_info(n, n, n)
    if info["scheme"] == "crt":
        return f"scheme II (CRT): {info['moduli']} int8 moduli, {info['products']} modular products"
    return f"scheme I: {info['slices']} int8 slices, {info['products']} slice products"


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from zynum_b200 import blas
    from zynum_b200._lib import load

    L = load()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.size
    flop = 2.0 * n ** 3
    peaks = _peaks()
    A, B = make_inputs(torch, n, args.phi, 1234 + rank, dev)  # column-major view: storage of A^T row-major
    C = torch.zeros((n, n), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    def call(method):
        blas.set_dgemm_method(method)
        return lambda: blas.dgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n)

    methods = []
    if args.method in ("ozaki", "both"):
        methods.append(("ozaki", blas.METHOD_OZAKI))
    if args.method in ("native", "both"):
        methods.append(("native", blas.METHOD_NATIVE))

    results = {}
    with ClockSampler(local_rank) as clocks:
        for name, mid in methods:
            fn = call(mid)
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            launches0 = L.zynum_blas_gpu_launch_count()
            L.zynum_blas_gpu_profile(1)
            t_begin = time.time()
            ms = time_device(torch, fn, args.steps, args.warmup, stream)
            t_end = time.time()
            # one event pair per call around the dominant kernel: keep the timed steps' records
            buf = np.zeros(4096)
            cnt = L.zynum_blas_gpu_profile_read(buf.ctypes.data, 4096)
            L.zynum_blas_gpu_profile(0)
            launches = (L.zynum_blas_gpu_launch_count() - launches0) // (args.steps + args.warmup)
            kern_ms = float(np.mean(buf[cnt - args.steps:cnt])) if cnt >= args.steps else None
            if world > 1:
                t = torch.tensor([ms], device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                ms = float(t.item())
            results[name] = {"phi": args.phi, "ms": ms, "tflops": flop / (ms * 1e-3) / 1e12,
                             "launches_per_step": int(launches), "kernel_ms": kern_ms, "window": (t_begin, t_end)}
        time.sleep(0.1)  # the sampler's last lines cover the end of the timed region
    clk = clocks.summary(results[methods[0][0]]["window"])
    for name in results:
        results[name]["clocks"] = clocks.summary(results[name].pop("window"))

    # errors of both methods vs the double-double oracle (rank 0, sampled entries)
    err = {}
    if rank == 0 and not args.no_error:
        from oracle import oracle as orc
        a_h = np.asfortranarray(A.cpu().numpy().T)
        b_h = np.asfortranarray(B.cpu().numpy().T)
        for name, mid in methods:
            call(mid)()
            torch.cuda.synchronize()
            c_h = np.asfortranarray(C.cpu().numpy().T)
            err[name] = sampled_error(orc, a_h, b_h, c_h, n)

    # end-to-end through the Fortran ABI with pinned host buffers
    head = methods[0]
    blas.set_dgemm_method(head[1])
    a_p = torch.empty((n, n), dtype=torch.float64).pin_memory()
    b_p = torch.empty((n, n), dtype=torch.float64).pin_memory()
    c_p = torch.zeros((n, n), dtype=torch.float64).pin_memory()
    a_p.copy_(A)
    b_p.copy_(B)
    e2e_steps = max(2, min(args.steps, 5))

    def host_call():
        blas.dgemm("N", "N", n, n, n, 1.0, a_p, n, b_p, n, 0.0, c_p, n)

    host_call()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_call()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    if rank != 0:
        return 0
    # measured raw issue rates of the two tensor pipes (denominators beside the nominal ones)
    import ctypes as C
    raw = {}
    for pipe, key in ((0, "fp64_dmma_tflops"), (1, "int8_tcgen05_tops")):
        r = C.c_double(0.0)
        if L.zynum_blas_gpu_measure_pipe_rate(pipe, C.byref(r), stream.cuda_stream) == 0:
            raw[key] = r.value
    hr = results[head[0]]
    value = world * hr["tflops"]
    # roofline of the dominant kernel
    if head[0] == "ozaki":
        from zynum_b200 import ozaki_info
        info = ozaki_info(n, n, n)
        ops = info["slice_products"] * flop
        int8_peak = 2.0 * peaks.get("bf16_tflops", PEAKS_FALLBACK["bf16_tflops"])
        achieved = ops / (hr["kernel_ms"] * 1e-3) / 1e12 if hr["kernel_ms"] else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOP/s (int8)",
                "frac": (achieved / int8_peak) if achieved else None,
                "peak_raw_issue": raw.get("int8_tcgen05_tops"),
                "frac_of_raw_issue": (achieved / raw["int8_tcgen05_tops"])
                if achieved and raw.get("int8_tcgen05_tops") else None,
                "traffic": TRAFFIC_8192["crt"] if (n == 8192 and info["scheme"] == "crt") else None,
                "kernel": ("ozaki int8 modular-product GEMM (CRT residues, tcgen05 kind::i8)" if info["scheme"] == "crt"
                           else "ozaki int8 slice-product GEMM (tcgen05 kind::i8)"),
                "peak_source": f"2 x bf16_tflops of {peaks['_source']} peaks (int8 dense rate is 2x bf16 on sm_100)",
                "work_per_launch": f"{info['products']} {'modular' if info['scheme'] == 'crt' else 'slice'} products"
                                   f" x 2*{n}^3 int8 ops"}
    else:
        achieved = flop / (hr["kernel_ms"] * 1e-3) / 1e12 if hr["kernel_ms"] else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                "frac": (achieved / FP64_NOMINAL_TFLOPS) if achieved else None,
                "peak_raw_issue": raw.get("fp64_dmma_tflops"),
                "frac_of_raw_issue": (achieved / raw["fp64_dmma_tflops"])
                if achieved and raw.get("fp64_dmma_tflops") else None,
                "traffic": TRAFFIC_8192["native"] if n == 8192 else None,
                "kernel": "native DGEMM (DMMA m16n8k8 f64)",
                "peak_source": "nominal FP64 pipe: 148 SMs x 128 flop/clk x 1.965 GHz (no measured FP64 peak)"}
    line = {
        "metric": METRIC,
        "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": hr["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": f"synthetic u*10^e, u~U[-1,1], e~U[-{args.phi},{args.phi}], seeded",
        "config": {"workload": f"DGEMM M=N=K={n} NN column-major FP64 alpha=1 beta=0",
                   "method": head[0], "l2": "inputs 3 x 512 MiB > 126 MB L2 (no flush needed)",
                   **({"ozaki": _ozaki_desc(n)} if head[0] == "ozaki" else {}),
                   "parallelism": "replicas" if world > 1 else "single-GPU"},
        "methods": {k: {**v, **({"error": err[k]} if k in err else {})} for k, v in results.items()},
        "roofline": roof,
        "raw_pipe_rates": {**raw, "how": "zynum_blas_gpu_measure_pipe_rate: register-only DMMA loop on every SM; "
                                          "tcgen05 cta_group::2 i8 M256 N256 K32 chain on shared-memory operands"},
        "clocks": clk,
        "gpu_launches": int(hr["launches_per_step"] * args.steps),
        "e2e": {"value": world * flop / e2e_s / 1e12, "unit": "TFLOP/s", "ms_per_step": e2e_s * 1e3,
                "h2d_bytes_per_step": 2 * n * n * 8, "d2h_bytes_per_step": n * n * 8,
                "path": "dgemm_ Fortran ABI, pinned host buffers"},
    }
    if "native" in results and results["native"].get("kernel_ms") and raw.get("fp64_dmma_tflops"):
        nat = flop / (results["native"]["kernel_ms"] * 1e-3) / 1e12
        line["methods"]["native"]["roofline"] = {
            "bound": "tensor", "achieved": nat, "unit": "TFLOP/s", "peak": FP64_NOMINAL_TFLOPS,
            "frac": nat / FP64_NOMINAL_TFLOPS, "peak_raw_issue": raw["fp64_dmma_tflops"],
            "frac_of_raw_issue": nat / raw["fp64_dmma_tflops"], "kernel": "native DGEMM (TMA-fed DMMA tiles)"}
    if not args.no_precision and not args.no_error and head[0] == "ozaki" and len(methods) == 2:
        from oracle import oracle as orc
        extra = precision_methods(torch, blas, orc, n, max(3, min(args.steps, 10)), max(3, args.warmup), stream,
                                  1234 + rank)
        line["methods"].update(extra)
        line["config"]["precision"] = ("methods: ozaki / native at phi = 0 (headline), 4, 8 on the same inputs per "
                                       "phi; sgemm_bf16x3 / sgemm_native on U[-1,1]; errors vs double-double")
    if not args.no_sweep:
        line["sweep"] = sweep_subset(torch, blas, stream, peaks, args.steps, args.warmup)
    if not args.no_batched:
        line["batched"] = bench_batched(torch, blas, max(3, args.steps), args.warmup)
        line["differentiation"] = bench_differentiation(torch, max(3, args.steps), args.warmup)
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(n if n <= 8192 else 8192, 256)
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ suites
def suite_precision(args):
    """DGEMM 8192^3 native vs Ozaki for phi in {0, 4, 8} and SGEMM 8192^3 3xBF16 vs native FP32:
    TFLOP/s and max / median relative error against the double-double oracle on sampled entries."""
    import torch
    from oracle import oracle as orc
    from zynum_b200 import blas
    n = args.size
    flop = 2.0 * n ** 3
    stream = torch.cuda.current_stream()
    out = {"suite": "precision", "n": n, "dgemm": {}, "sgemm": {}}
    for phi in (0.0, 4.0, 8.0):
        A, B = make_inputs(torch, n, phi, 1234, torch.device("cuda"))
        C = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        a_h = np.asfortranarray(A.cpu().numpy().T)
        b_h = np.asfortranarray(B.cpu().numpy().T)
        row = {}
        for name, mid in (("native", blas.METHOD_NATIVE), ("ozaki", blas.METHOD_OZAKI)):
            blas.set_dgemm_method(mid)
            fn = lambda: blas.dgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n)  # noqa: E731
            ms = time_device(torch, fn, args.steps, args.warmup, stream)
            fn()
            torch.cuda.synchronize()
            err = sampled_error(orc, a_h, b_h, np.asfortranarray(C.cpu().numpy().T), n)
            row[name] = {"tflops": flop / (ms * 1e-3) / 1e12, "ms": ms, **err}
            if name == "ozaki":
                from zynum_b200 import ozaki_info
                row[name]["slices"] = ozaki_info(n, n, n)["slices"]
        blas.set_dgemm_method(blas.METHOD_NATIVE)
        out["dgemm"][f"phi={phi:g}"] = row
        del A, B, C
    g = torch.Generator(device="cuda").manual_seed(99)
    A = torch.rand((n, n), generator=g, device="cuda", dtype=torch.float32) * 2 - 1
    B = torch.rand((n, n), generator=g, device="cuda", dtype=torch.float32) * 2 - 1
    C = torch.zeros((n, n), dtype=torch.float32, device="cuda")
    a_h = np.asfortranarray(A.cpu().numpy().T)
    b_h = np.asfortranarray(B.cpu().numpy().T)
    for name, mid in (("native_fp32", blas.SMETHOD_NATIVE), ("bf16x3", blas.SMETHOD_BF16X3),
                      ("ozaki_int8", blas.SMETHOD_OZAKI)):
        blas.set_sgemm_method(mid)
        fn = lambda: blas.sgemm_device("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n)  # noqa: E731
        ms = time_device(torch, fn, args.steps, args.warmup, stream)
        fn()
        torch.cuda.synchronize()
        err = sampled_error(orc, a_h, b_h, np.asfortranarray(C.cpu().numpy().T.astype(np.float32)), n)
        out["sgemm"][name] = {"tflops": flop / (ms * 1e-3) / 1e12, "ms": ms, **err}
    blas.set_sgemm_method(blas.SMETHOD_NATIVE)
    print(json.dumps(out), flush=True)
    return 0


def suite_sweep(args):
    """Native GEMM shape sweep (FP64 and FP32): square n^3, tall-skinny 131072 x 64 x 64,
    K-dominant 256 x 256 x 262144, beta in {0, 1}; ZGEMM / CGEMM 4096^3."""
    import torch
    from zynum_b200 import blas
    stream = torch.cuda.current_stream()
    rows = []
    shapes = [(n, n, n) for n in (256, 1024, 4096, 8192, 16384)] + [(131072, 64, 64), (256, 256, 262144)]
    for dt, tdt, fn in (("f64", torch.float64, blas.dgemm_device), ("f32", torch.float32, blas.sgemm_device)):
        for (m, n, k) in shapes:
            if dt == "f64" and m == 16384:
                pass
            g = torch.Generator(device="cuda").manual_seed(m + n + k)
            A = torch.rand((k, m), generator=g, device="cuda", dtype=tdt) * 2 - 1   # column-major m x k
            B = torch.rand((n, k), generator=g, device="cuda", dtype=tdt) * 2 - 1   # column-major k x n
            C = torch.rand((n, m), generator=g, device="cuda", dtype=tdt) * 2 - 1
            for beta in (0.0, 1.0):
                f = lambda: fn("N", "N", m, n, k, 1.0, A, m, B, k, beta, C, m)  # noqa: E731
                steps = max(2, min(args.steps, int(2e12 / (2.0 * m * n * k)) + 2))
                ms = time_device(torch, f, steps, max(1, args.warmup), stream)
                esz = 8 if dt == "f64" else 4
                byts = esz * (m * k + k * n + m * n * (2 if beta else 1))
                rows.append({"dtype": dt, "m": m, "n": n, "k": k, "beta": beta, "ms": ms,
                             "tflops": 2.0 * m * n * k / (ms * 1e-3) / 1e12, "gbs": byts / (ms * 1e-3) / 1e9})
            del A, B, C
    for dt, tdt, fn in (("z", torch.complex128, blas.zgemm_device), ("c", torch.complex64, blas.cgemm_device)):
        n = 4096
        g = torch.Generator(device="cuda").manual_seed(5)
        real = torch.float64 if dt == "z" else torch.float32
        A = torch.complex(torch.rand((n, n), generator=g, device="cuda", dtype=real) * 2 - 1,
                          torch.rand((n, n), generator=g, device="cuda", dtype=real) * 2 - 1)
        B = torch.complex(torch.rand((n, n), generator=g, device="cuda", dtype=real) * 2 - 1,
                          torch.rand((n, n), generator=g, device="cuda", dtype=real) * 2 - 1)
        C = torch.zeros((n, n), device="cuda", dtype=tdt)
        for cm, cname in ((blas.COMPLEX_4M, "4M"), (blas.COMPLEX_3M, "3M")):
            blas.set_complex_method(cm)
            f = lambda: fn("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n)  # noqa: E731
            ms = time_device(torch, f, max(2, args.steps), max(1, args.warmup), stream)
            rows.append({"dtype": dt, "m": n, "n": n, "k": n, "beta": 0.0, "method": cname, "ms": ms,
                         "tflops": 8.0 * n ** 3 / (ms * 1e-3) / 1e12})
        blas.set_complex_method(blas.COMPLEX_4M)
        del A, B, C
    print(json.dumps({"suite": "sweep", "rows": rows}), flush=True)
    return 0


def suite_vector(args):
    """Vector-edge GEMM (n == 1 / m == 1, the matrix-vector kernels): HBM GB/s of the
    matrix read against the measured copy bandwidth, every transpose pair, a long-K
    case that takes the K-split partials, a short-K tall case; torch.mv (cuBLAS GEMV)
    on the same NN data as a library reference.  Every matrix is larger than L2."""
    import torch
    from zynum_b200 import blas
    stream = torch.cuda.current_stream()
    peak = _peaks()["hbm_gbs"]
    rows = []
    cases = [(16384, 1, 16384), (1, 16384, 16384), (2048, 1, 262144), (4194304, 1, 64), (1, 4194304, 64)]
    for dt, tdt, fn in (("f64", torch.float64, blas.dgemm_device), ("f32", torch.float32, blas.sgemm_device)):
        esz = 8 if dt == "f64" else 4
        for (m, n, k) in cases:
            rm, rk = (m, k) if n == 1 else (n, k)          # the matrix is rm x rk or rk x rm
            g = torch.Generator(device="cuda").manual_seed(rm + rk)
            M = torch.rand((rm * rk,), generator=g, device="cuda", dtype=tdt) * 2 - 1
            x = torch.rand((k,), generator=g, device="cuda", dtype=tdt) * 2 - 1
            y = torch.zeros((max(m, n),), device="cuda", dtype=tdt)
            for t in ("N", "T"):
                if n == 1:      # op(A) = A (m x k, ld m) or A^T (A k x m, ld k); x = B (k x 1)
                    lda = m if t == "N" else k
                    f = lambda: fn(t, "N", m, 1, k, 1.0, M, lda, x, k, 0.0, y, m)  # noqa: E731
                else:           # op(B) = B (k x n, ld k) or B^T (B n x k, ld n); x = A (1 x k, ld 1)
                    ldb = k if t == "N" else n
                    f = lambda: fn("N", t, 1, n, k, 1.0, x, 1, M, ldb, 0.0, y, 1)  # noqa: E731
                ms = time_device(torch, f, max(5, args.steps), max(3, args.warmup), stream)
                byts = esz * (rm * rk + k + max(m, n))
                gbs = byts / (ms * 1e-3) / 1e9
                rows.append({"dtype": dt, "m": m, "n": n, "k": k, "trans": t, "ms": ms, "gbs": gbs,
                             "frac_of_measured_hbm": gbs / peak})
            if n == 1:  # cuBLAS GEMV through torch on the NN layout (row-major view of A^T)
                Mv = M.view(k, m).t()
                f = lambda: torch.mv(Mv, x, out=y)  # noqa: E731
                ms = time_device(torch, f, max(5, args.steps), max(3, args.warmup), stream)
                gbs = esz * (rm * rk + k + m) / (ms * 1e-3) / 1e9
                rows.append({"dtype": dt, "m": m, "n": 1, "k": k, "trans": "N", "impl": "torch.mv", "ms": ms,
                             "gbs": gbs, "frac_of_measured_hbm": gbs / peak})
            del M, x, y
        # narrow n / narrow m (2..16 vectors): one matrix read serves every vector
        for nv in (2, 4, 8, 16):
            for side in ("n", "m"):
                m, n, k = (16384, nv, 16384) if side == "n" else (nv, 16384, 16384)
                g = torch.Generator(device="cuda").manual_seed(nv)
                A = torch.rand((m * k,), generator=g, device="cuda", dtype=tdt) * 2 - 1
                B = torch.rand((k * n,), generator=g, device="cuda", dtype=tdt) * 2 - 1
                C = torch.zeros((m * n,), device="cuda", dtype=tdt)
                f = lambda: fn("N", "N", m, n, k, 1.0, A, m, B, k, 0.0, C, m)  # noqa: E731
                ms = time_device(torch, f, max(5, args.steps), max(3, args.warmup), stream)
                gbs = esz * (m * k + k * n + m * n) / (ms * 1e-3) / 1e9
                rows.append({"dtype": dt, "m": m, "n": n, "k": k, "trans": "NN", "ms": ms, "gbs": gbs,
                             "frac_of_measured_hbm": gbs / peak, "tflops": 2.0 * m * n * k / (ms * 1e-3) / 1e12})
                del A, B, C
    print(json.dumps({"suite": "vector", "hbm_peak_gbs": peak, "rows": rows}), flush=True)
    return 0


def suite_level3(args):
    """Triangular / symmetric Level-3 routines on device pointers, n = 8192 (TRSM and
    TRMM with 8192 right-hand sides, SYRK / SYR2K with k = 8192), FP64 under the native
    and the automatic (Ozaki-capable) method and FP32 native.  TFLOP/s counts the
    useful flops: TRSM / TRMM m^2 n, SYMM 2 m^2 n, SYRK n^2 k, SYR2K 2 n^2 k."""
    import torch
    from zynum_b200 import blas
    stream = torch.cuda.current_stream()
    n = args.size
    rows = []
    for dt, tdt in (("f64", torch.float64), ("f32", torch.float32)):
        g = torch.Generator(device="cuda").manual_seed(3)
        A = torch.rand((n, n), generator=g, device="cuda", dtype=tdt) * 2 - 1
        A += n * torch.eye(n, device="cuda", dtype=tdt)   # well-conditioned triangles for TRSM
        B = torch.rand((n, n), generator=g, device="cuda", dtype=tdt) * 2 - 1
        C = torch.zeros((n, n), device="cuda", dtype=tdt)
        X = B.clone()
        ops = {
            "trsm": (lambda: (X.copy_(B), blas.dtrsm_device("L", "L", "N", "N", n, n, 1.0, A, n, X, n)),
                     float(n) ** 3),
            "trmm": (lambda: (X.copy_(B), blas.trmm_device("L", "L", "N", "N", n, n, 1.0, A, n, X, n)),
                     float(n) ** 3),
            "symm": (lambda: blas.symm_device("L", "U", n, n, 1.0, A, n, B, n, 0.0, C, n), 2.0 * float(n) ** 3),
            "syr2k": (lambda: blas.syr2k_device("L", "N", n, n, 1.0, A, n, B, n, 0.0, C, n), 2.0 * float(n) ** 3),
        }
        if dt == "f64":
            ops["syrk"] = (lambda: blas.dsyrk_device("L", "N", n, n, 1.0, A, n, 0.0, C, n), float(n) ** 3)
        else:
            ops.pop("trsm")
        methods = (("native", blas.METHOD_NATIVE), ("auto", blas.METHOD_AUTO)) if dt == "f64" else (("native", None),)
        for mname, mval in methods:
            old = blas.set_dgemm_method(mval) if mval is not None else None
            for name, (fn, flops) in ops.items():
                ms = time_device(torch, fn, max(3, min(args.steps, 5)), max(3, args.warmup), stream)
                if name in ("trsm", "trmm"):  # the timed call includes an n x n device copy of B
                    ms_copy = time_device(torch, lambda: X.copy_(B), 5, 2, stream)
                    ms -= ms_copy
                rows.append({"op": name, "dtype": dt, "method": mname, "n": n, "ms": ms,
                             "tflops": flops / (ms * 1e-3) / 1e12})
            if old is not None:
                blas.set_dgemm_method(old)
        del A, B, C, X
    # the differentiation chain's shapes: TRSM L 4096 x 4096 with 512 right-hand sides, SYRK 512 x 4096
    for mname, mval in (("native", blas.METHOD_NATIVE), ("auto", blas.METHOD_AUTO)):
        old = blas.set_dgemm_method(mval)
        g = torch.Generator(device="cuda").manual_seed(11)
        nn, r = 4096, 512
        L = torch.tril(torch.randn((nn, nn), generator=g, device="cuda", dtype=torch.float64) / nn ** 0.5, -1)
        L += torch.diag(1 + torch.randn(nn, generator=g, device="cuda", dtype=torch.float64).abs())
        Lc = L.t().contiguous()  # column-major storage of L
        B = torch.randn((r, nn), generator=g, device="cuda", dtype=torch.float64)  # column-major 4096 x 512
        X = B.clone()
        C = torch.zeros((r, r), device="cuda", dtype=torch.float64)
        fn = lambda: (X.copy_(B), blas.dtrsm_device("L", "L", "N", "N", nn, r, 1.0, Lc, nn, X, nn))  # noqa: E731
        ms = time_device(torch, fn, 10, 3, stream) - time_device(torch, lambda: X.copy_(B), 10, 3, stream)
        rows.append({"op": "trsm_4096x512", "dtype": "f64", "method": mname, "ms": ms,
                     "tflops": float(nn) ** 2 * r / (ms * 1e-3) / 1e12})
        fn = lambda: blas.dsyrk_device("L", "T", r, nn, 1.0, X, nn, 0.0, C, r)  # noqa: E731
        ms = time_device(torch, fn, 10, 3, stream)
        rows.append({"op": "syrk_512x4096", "dtype": "f64", "method": mname, "ms": ms,
                     "tflops": float(r) * r * nn / (ms * 1e-3) / 1e12})
        blas.set_dgemm_method(old)
        del L, Lc, B, X, C
    # complex rank-k / rank-2k updates, n = k = 4096: ZHERK / ZSYRK form one triangle of the
    # product (useful flops 4 n^2 k), ZHER2K / ZSYR2K the full n x n product W (8 n^2 k)
    nc = 4096
    g = torch.Generator(device="cuda").manual_seed(13)
    A = torch.complex(torch.rand((nc, nc), generator=g, device="cuda", dtype=torch.float64) * 2 - 1,
                      torch.rand((nc, nc), generator=g, device="cuda", dtype=torch.float64) * 2 - 1)
    B = A.flip(0).contiguous()
    C = torch.zeros((nc, nc), device="cuda", dtype=torch.complex128)
    for cname, cm in (("4M", blas.COMPLEX_4M), ("3M", blas.COMPLEX_3M)):
        old = blas.set_complex_method(cm)
        ops = {
            "zherk": (lambda: blas.herk_device("L", "N", nc, nc, 1.0, A, nc, 0.0, C, nc), 4.0 * nc ** 3),
            "zsyrk": (lambda: blas.syrk_device_c("L", "N", nc, nc, 1.0, A, nc, 0.0, C, nc), 4.0 * nc ** 3),
            "zher2k": (lambda: blas.syr2k_device_c("L", "N", nc, nc, 1.0, A, nc, B, nc, 0.0, C, nc, herm=True),
                       8.0 * nc ** 3),
        }
        for name, (fn, flops) in ops.items():
            ms = time_device(torch, fn, max(3, min(args.steps, 5)), max(3, args.warmup), stream)
            rows.append({"op": name, "dtype": "z", "method": cname, "n": nc, "k": nc, "ms": ms,
                         "tflops": flops / (ms * 1e-3) / 1e12})
        blas.set_complex_method(old)
    del A, B, C
    print(json.dumps({"suite": "level3", "rows": rows}), flush=True)
    return 0


def suite_batched(args):
    """The batched workloads alone (optionally a smaller sample of the same distributions)."""
    import torch
    from zynum_b200 import blas
    out = bench_batched(torch, blas, args.steps, args.warmup, count=args.batch_count,
                        tcount=max(1, args.batch_count // 4), which=tuple(args.batch_only.split(",")))
    print(json.dumps({"suite": "batched", "count": args.batch_count, "rows": out}), flush=True)
    return 0


def suite_chain(args):
    """The differentiation workload's pieces alone, for launch lists: the solve
    X = L^-1 B (L 4096 x 4096 lower, off-diagonals N(0, 1/4096), diagonal
    1 + |N(0,1)|; B 4096 x 512 N(0,1); FP64, native method) `--warmup` untimed
    and `--steps` timed calls, then the forward + backward chain likewise."""
    import torch
    from zynum_b200 import blas
    n, r = 4096, 512
    old = blas.set_dgemm_method(blas.METHOD_NATIVE)
    g = torch.Generator(device="cuda").manual_seed(11)
    L = torch.tril(torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64) / n ** 0.5, -1)
    L += torch.diag(1 + torch.randn(n, generator=g, device="cuda", dtype=torch.float64).abs())
    Lc = L.t().contiguous()  # column-major storage of L
    B = torch.randn((r, n), generator=g, device="cuda", dtype=torch.float64)  # column-major 4096 x 512
    X = B.clone()
    fn = lambda: blas.dtrsm_device("L", "L", "N", "N", n, r, 1.0, Lc, n, X, n)  # noqa: E731
    ms = time_device(torch, fn, args.steps, args.warmup, torch.cuda.current_stream())
    blas.set_dgemm_method(old)
    diff = bench_differentiation(torch, args.steps, args.warmup)
    print(json.dumps({"suite": "chain", "trsm_4096x512_ms": ms, "trsm_tflops": float(n) ** 2 * r / (ms * 1e-3) / 1e12,
                      "differentiation": diff}), flush=True)
    return 0


def suite_one(args):
    """One GEMM shape, for profiling a single kernel: --dtype f64|f32|z|c, --m/--n/--k,
    --method (native or ozaki for f64; ozaki means 3xBF16 for f32), --beta, NN,
    column-major U[-1,1] inputs; `--warmup` untimed calls, then `--steps` timed ones."""
    import torch
    from zynum_b200 import blas
    m, n, k = args.m, args.n, args.k
    dt = args.dtype
    tdt = {"f64": torch.float64, "f32": torch.float32, "z": torch.complex128, "c": torch.complex64}[dt]
    g = torch.Generator(device="cuda").manual_seed(1)
    real = torch.float64 if dt in ("f64", "z") else torch.float32

    def rnd(rows, cols):
        x = torch.rand((cols, rows), generator=g, device="cuda", dtype=real) * 2 - 1
        if dt in ("z", "c"):
            x = torch.complex(x, torch.rand((cols, rows), generator=g, device="cuda", dtype=real) * 2 - 1)
        return x

    A, B = rnd(m, k), rnd(k, n)
    C = torch.zeros((n, m), device="cuda", dtype=tdt)
    if dt == "f64":
        blas.set_dgemm_method(blas.METHOD_OZAKI if args.method == "ozaki" else blas.METHOD_NATIVE)
        fn = lambda: blas.dgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, args.beta, C, m)  # noqa: E731
    elif dt == "f32":
        blas.set_sgemm_method(blas.SMETHOD_BF16X3 if args.method == "ozaki" else blas.SMETHOD_NATIVE)
        fn = lambda: blas.sgemm_device("N", "N", m, n, k, 1.0, A, m, B, k, args.beta, C, m)  # noqa: E731
    else:
        f = blas.zgemm_device if dt == "z" else blas.cgemm_device
        fn = lambda: f("N", "N", m, n, k, 1.0, A, m, B, k, args.beta, C, m)  # noqa: E731
    ms = time_device(torch, fn, args.steps, args.warmup, torch.cuda.current_stream())
    flop = (8.0 if dt in ("z", "c") else 2.0) * m * n * k
    esz = C.element_size()
    byts = esz * (m * k + k * n + m * n * (2 if args.beta else 1))
    print(json.dumps({"suite": "one", "dtype": dt, "m": m, "n": n, "k": k, "beta": args.beta, "method": args.method,
                      "ms": ms,
                      "tflops": flop / (ms * 1e-3) / 1e12, "gbs": byts / (ms * 1e-3) / 1e9}), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--method", choices=["ozaki", "native", "both"], default="both")
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--phi", type=float, default=0.0)
    ap.add_argument("--no-error", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-precision", action="store_true", help="skip the phi = 4 / 8 and SGEMM methods")
    ap.add_argument("--no-sweep", action="store_true", help="skip the tall-skinny / K-dominant / complex rows")
    ap.add_argument("--dtype", choices=["f64", "f32", "z", "c"], default="f64", help="suite one: element type")
    ap.add_argument("--m", type=int, default=4096, help="suite one: rows of C")
    ap.add_argument("--n", type=int, default=4096, help="suite one: columns of C")
    ap.add_argument("--k", type=int, default=4096, help="suite one: inner dimension")
    ap.add_argument("--beta", type=float, default=0.0, help="suite one: beta")
    ap.add_argument("--suite", choices=["headline", "precision", "sweep", "vector", "level3", "batched", "one", "chain"],
                    default="headline", help="secondary measurement suites (one JSON line each)")
    ap.add_argument("--batch-count", type=int, default=20000,
                    help="batched suite: GEMM problems per batch (TRSM problems: a quarter)")
    ap.add_argument("--batch-only", default="dgemm,sgemm,dtrsm", help="batched suite: which batches")
    args = ap.parse_args(argv)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if args.impl == "ours":
            torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            return run_reference(args, rank, world)
        if args.suite == "precision":
            return suite_precision(args)
        if args.suite == "sweep":
            return suite_sweep(args)
        if args.suite == "vector":
            return suite_vector(args)
        if args.suite == "level3":
            return suite_level3(args)
        if args.suite == "batched":
            return suite_batched(args)
        if args.suite == "one":
            return suite_one(args)
        if args.suite == "chain":
            return suite_chain(args)
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
