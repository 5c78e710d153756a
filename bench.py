"""Benchmark of the B200 Cholesky path: FP64-accurate pposv TFLOP/s at n=32768.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 32768] [--nrhs 8] [--kappa 1e6] [--no-cpu] [--no-plain]
                    [--no-batched] [--no-gp] [--no-gp-large] [--batched-count 4096] [--gp-batch 256]
                    [--only mixed-B|mixed-T|plain|batched|gp]

Workload: solve A X = B to FP64 accuracy for a double n x n SPD matrix
A = U diag(s) U^T (U = product of 4 Householder reflectors with N(0,1)
vectors, s geometric from 1 to 1/kappa) and nrhs N(0,1) right-hand sides,
uplo 'L'.  One step = one solve.  Two paths are timed:
  mixed+IR : ddla_d_pposv_mixed (tensor-core BF16 or TF32 factor, FP64
             refinement / GMRES-IR, ?sposv stopping test) -- the headline value
             is the faster of the two precisions;
  plain    : ddla_d_pposv (FP64 factor on the FP64 tensor cores + fused solve).
TFLOP/s use the FP64 factor+solve count n^3/3 + 2 n^2 nrhs for both paths.
The 8.6 GB matrix is larger than the 126 MB L2, so no L2 flush is needed.

Two secondary figures ride on the same JSON line: "batched" (4096 uneven SPD
matrices, n_i in [16, 512], factor + solve + log-determinant in one persistent
graph-replayed launch, matrices/s, against a per-matrix loop of the plain
path) and "gp" (256 Gaussian-process likelihoods of order 1024 with their
hyperparameter gradients through the adjoint kernels, evaluations/s, against
a per-matrix torch.linalg loop and torch's batched path).

Device timing: CUDA events on the library handle's stream around each call,
summed over the K steps; the plain path restores A from a pristine copy
outside the events (it overwrites A with its factor; the mixed path leaves A
unchanged).  The timed loop is bracketed by a barrier and a device
synchronize on both sides; the max over ranks is taken.  With --gpus N > 1
every rank solves its own system (replicas: one pposv on a 1x1 grid does not
shard), so scaling is weak.

e2e: the headline path through the public C ABI with host buffers -- the H2D
copy of A's lower triangle (the part uplo 'L' references) and of B from pinned
memory, the solve and the D2H copy of X, inside the events.  The reference arm
(--impl reference) times the reference's own CPU implementation of the path
(LAPACK dpotrf + two dtrsm, the calls its CPU handle makes) on the host cores,
every timed step one full solve of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "pposv TFLOP/s n=32768 at FP64 accuracy (plain vs mixed+IR)"
UNIT = "TFLOP/s"
KIND = {"potrf_diag": 0, "trsm_panel": 1, "syrk_update": 2, "potrs_fused": 3, "logdet": 4, "mixed_update": 5,
        "mixed_other": 6, "symm_residual": 7, "batched_posv": 8, "adjoint_contract": 9, "trtri_batched": 10}


def flops_pposv(n: int, nrhs: int) -> float:
    return n ** 3 / 3.0 + 2.0 * n * n * nrhs


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


def traffic_summary() -> dict:
    """Per-launch DRAM traffic of the dominant kernels from the committed ncu summary (profiles/)."""
    p = ROOT / "profiles" / "dram_traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons of one GPU, sampled while the timed region runs.

    NVML is read in-process every 20 ms from a thread (reads only; no setting of the
    GPU is touched), so a timed region of a few hundred milliseconds still gets a
    dozen samples.  Where NVML cannot be opened, ``nvidia-smi -lms 200`` is read
    instead.  The torch device is matched to its NVML handle by UUID, so the index
    is right under CUDA_VISIBLE_DEVICES too.
    """
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))
    PERIOD_S = 0.02

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.samples = []  # (sm MHz, reason bitmask) from NVML
        self.max_mhz = None
        self._nvml = None
        self._stop = threading.Event()
        self._t = None

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        self._nvml = pynvml
        try:
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _poll_nvml(self, h):
        nv = self._nvml
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(get_reasons(h))))
            except Exception:
                break
            self._stop.wait(self.PERIOD_S)

    def __enter__(self):
        try:
            h = self._nvml_handle()
            self.max_mhz = float(self._nvml.nvmlDeviceGetMaxClockInfo(h, self._nvml.NVML_CLOCK_SM))
            self._t = threading.Thread(target=self._poll_nvml, args=(h,), daemon=True)
            self._t.start()
            return self
        except Exception:
            self._nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self._nvml is not None:
            self._stop.set()
            self._t.join(timeout=5)
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], self.max_mhz, set()
        for mhz, bits in self.samples:
            sm.append(mhz)
            for name, bit in self.REASON_BITS:
                if bits & bit:
                    reasons.add(name)
        names = [name for name, _ in self.REASON_BITS]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


# ---------------------------------------------------------------------------
# CPU side: the reference's CPU arm on a bounded sample
# ---------------------------------------------------------------------------
def cpu_sample(budget_s: float = 12.0, nrhs: int = 8, kappa: float = 1e6, max_n: int = 12288):
    """Time LAPACK dpotrf + 2 dtrsm (the reference CPU handle's calls) on the bench's matrix family,
    growing n until one solve takes a few seconds; returns (TFLOP/s, sample description, info)."""
    from libddla_b200.workloads import householder_spd_host
    from oracle import lapack_arm

    info = lapack_arm.blas_info()
    n = 2048
    best = None
    spent = 0.0
    while True:
        A = householder_spd_host(n, kappa, 0xDD1A0003)
        B = np.random.default_rng(7).standard_normal((n, nrhs))
        Af = np.asfortranarray(A)
        t0 = time.perf_counter()
        lapack_arm.pposv(Af, B, "L", overwrite=True)
        dt = time.perf_counter() - t0
        spent += dt
        best = (flops_pposv(n, nrhs) / dt / 1e12, n, dt)
        if dt > budget_s / 4 or n >= max_n or spent > budget_s:
            break
        n = min(max_n, int(n * 1.5) // 256 * 256)
    tf, n, dt = best
    sample = (f"LAPACK dpotrf('L')+2x dtrsm via {info.get('library')} {info.get('version')} "
              f"({info.get('core')}), n={n} nrhs={nrhs} kappa={kappa:g}, {dt:.2f} s per solve")
    return tf, sample, info


def run_reference(args, rank: int):
    """The reference's CPU arm on the headline workload itself: every timed step is one full
    LAPACK dpotrf('L') + 2 dtrsm solve at n = args.n (the reference CPU handle's calls at a
    1x1 grid), on all host threads; the warm-up steps are solves at n = 4096 (thread pool and
    page warm-up), and A is restored from a pristine copy outside the timed region."""
    if rank != 0:
        return
    from libddla_b200.workloads import householder_spd_host_lower
    from oracle import lapack_arm

    info = lapack_arm.blas_info()
    n, nrhs = args.n, args.nrhs
    nw = min(4096, n)
    Aw = householder_spd_host_lower(nw, args.kappa, 0xDD1A0003)
    Bw = np.random.default_rng(7).standard_normal((nw, nrhs))
    for _ in range(args.warmup):
        lapack_arm.pposv(np.array(Aw, order="F"), np.array(Bw, order="F"), "L", overwrite=True)
    t0 = time.perf_counter()
    A0 = householder_spd_host_lower(n, args.kappa, 0xDD1A0003)
    gen_s = time.perf_counter() - t0
    B0 = np.asfortranarray(np.random.default_rng(7).standard_normal((n, nrhs)))
    A = np.empty_like(A0, order="F")
    B = np.empty_like(B0, order="F")
    times = []
    for _ in range(args.steps):
        np.copyto(A, A0)
        np.copyto(B, B0)
        t0 = time.perf_counter()
        _, X, cinfo = lapack_arm.pposv(A, B, "L", overwrite=True)
        times.append(time.perf_counter() - t0)
        assert cinfo == 0, cinfo
    total = sum(times)
    v = flops_pposv(n, nrhs) * args.steps / total / 1e12
    cores = int(info.get("threads") or os.cpu_count() or 1)
    sample = (f"LAPACK dpotrf('L') + 2x dtrsm via {info.get('library')} {info.get('version')} ({info.get('core')}), "
              f"{args.steps} full solves at n={n} nrhs={nrhs} kappa={args.kappa:g}, "
              f"median {statistics.median(times):.2f} s per solve (warm-up {args.warmup} solves at n={nw}; "
              f"matrix generated on the host in {gen_s:.1f} s)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"pposv d uplo=L n={n} nrhs={nrhs} A=U diag(s) U^T kappa={args.kappa:g}",
                       "path": "reference CPU handle at a 1x1 grid: LAPACK dpotrf + 2 dtrsm (OpenBLAS)",
                       "sample": sample},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def fp64_peak_tflops(torch, device) -> float:
    """cuBLAS DGEMM 8192^3 best of 5 (the FP64 tensor-core reference peak, measured here)."""
    n = 8192
    a = torch.randn(n, n, device=device, dtype=torch.float64)
    b = torch.randn(n, n, device=device, dtype=torch.float64)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def read_kernels(C):
    out = {}
    for name, kind in KIND.items():
        ms, cnt, fl, by = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
        C.ddla_c_profile_read(kind, ctypes.byref(ms), ctypes.byref(cnt), ctypes.byref(fl), ctypes.byref(by), 1)
        if cnt.value:
            out[name] = {"ms": ms.value, "launches": cnt.value, "flops": fl.value, "bytes": by.value}
    return out


# ---------------------------------------------------------------------------
# secondary legs: batched uneven SPD (factor+solve+logdet) and the GP likelihood
# ---------------------------------------------------------------------------
def vendor_leg(args, torch, A0, B0, backward_error):
    """The reference's GPU arm at a 1x1 grid: one cusolverDn?potrf and two cublas?trsm
    (src/Cholesky/ppotrf.cpp:39-54 -> potrf.cpp:106-113; ppotrs.cpp:44-61 -> trsm.cpp:154-159).
    torch.linalg.cholesky_ex and torch.cholesky_solve call cuSOLVER's potrf and potrs on the
    bench's matrix and right-hand sides (FP64); CUDA events on torch's stream around each
    solve, the factor's allocation included as the reference allocates its lwork per call."""
    n, nrhs = args.n, args.nrhs
    B = B0.T  # the n x nrhs view of the column-major right-hand sides

    def step():
        L, info = torch.linalg.cholesky_ex(A0)
        return info, torch.cholesky_solve(B, L)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times, last = [], None
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        last = step()
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    info, X = last
    assert int(info.item()) == 0, int(info.item())
    total = sum(times)
    return {"metric": "pposv TFLOP/s through cuSOLVER (the reference's GPU arm)", "unit": "TFLOP/s",
            "value": flops_pposv(n, nrhs) * args.steps / (total * 1e-3) / 1e12, "ms_per_step": total / args.steps,
            "backward_error": backward_error(X.T),
            "config": {"workload": f"pposv d uplo=L n={n} nrhs={nrhs} kappa={args.kappa:g}",
                       "calls": "torch.linalg.cholesky_ex + torch.cholesky_solve (cuSOLVER potrf, potrs)"}}


def flops_pposv_cplx(n: int, nrhs: int) -> float:
    return 4.0 * n ** 3 / 3.0 + 8.0 * n * n * nrhs


def se_kernel_leg(args, torch, device, h, stream, C):
    """The SE-kernel configuration: pposv on A = K + 1e-2 I, K a squared-exponential kernel
    (lengthscale 0.2) on 16384 points uniform in [0,1]^3, nrhs = 64, for double and complex
    double (K times exp(i k.(x - y)), k ~ N(0, I3)).  Ours: ddla pposv (plain path) through the
    C ABI, device-timed on the handle's stream with A restored outside the events.  Beside it the
    reference's GPU arm (cuSOLVER potrf + potrs through torch) and its CPU arm (LAPACK ?potrf +
    2 ?trsm, one solve on the host cores), the solution's relative difference from the CPU arm,
    and the factor's scaled backward error ||A - L L^H||_F / (n eps ||A||_F)."""
    from libddla_b200 import ddla
    from libddla_b200.workloads import se_kernel
    from oracle import lapack_arm

    n, nrhs = args.se_n, 64
    out = {}
    for p, cplx in (("d", False), ("z", True)):
        A = se_kernel(n, 0xDD1A0002, complex_=cplx, device=device)  # Hermitian, row-major
        Acm = A.T.contiguous()  # column-major storage of A
        dt = A.dtype
        g = torch.Generator(device=device).manual_seed(0xDD1A0102)
        Bt = torch.randn(nrhs, n, generator=g, device=device, dtype=torch.float64)
        if cplx:
            Bt = torch.complex(Bt, torch.randn(nrhs, n, generator=g, device=device, dtype=torch.float64))
        Aw, Xw = torch.empty_like(Acm), torch.empty_like(Bt)
        # A, Acm and Bt were made on torch's current stream; restore() copies them on the
        # library's stream, so they must be complete first
        torch.cuda.synchronize()
        npdt = np.complex128 if cplx else np.float64
        dA = ddla.DistributedMatrix.wrap(h, Aw.data_ptr(), n, n, n, npdt, mb=256, nb=256)
        dX = ddla.DistributedMatrix.wrap(h, Xw.data_ptr(), n, nrhs, n, npdt, mb=256, nb=256)
        fl = flops_pposv_cplx(n, nrhs) if cplx else flops_pposv(n, nrhs)

        def restore():
            with torch.cuda.stream(stream):
                Aw.copy_(Acm)
                Xw.copy_(Bt)

        times = []
        for i in range(args.warmup + max(1, min(3, args.steps))):
            restore()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, info = ddla.pposv(dA, dX, "L")
            e1.record(stream)
            e1.synchronize()
            assert info == 0, (p, info)
            if i >= args.warmup:
                times.append(e0.elapsed_time(e1))
        ms = statistics.median(times)
        L = torch.tril(Aw.T)
        eps = float(np.finfo(np.float64).eps)
        R = L @ L.conj().T
        R -= A
        bwd = float(torch.linalg.norm(R) / (n * eps * torch.linalg.norm(A)))
        del R, L
        X = Xw.T  # n x nrhs
        # the reference's GPU arm on the same matrix
        vt = []
        for i in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            Lv, vinfo = torch.linalg.cholesky_ex(A)
            Xv = torch.cholesky_solve(Bt.T, Lv)
            e1.record()
            e1.synchronize()
            vt.append(e0.elapsed_time(e1))
            del Lv
        vms = min(vt)
        # the reference's CPU arm: one solve on the host cores, and the solution agreement
        Ah = np.asfortranarray(A.cpu().numpy())
        Bh = np.asfortranarray(Bt.T.cpu().numpy())
        t0 = time.perf_counter()
        _, Xref, cinfo = lapack_arm.pposv(Ah, Bh, "L", overwrite=True)
        cpu_s = time.perf_counter() - t0
        del Ah
        Xr = torch.from_numpy(np.ascontiguousarray(Xref)).to(device)
        rel = float((X - Xr).abs().max() / Xr.abs().max())
        rel_v = float((Xv - Xr).abs().max() / Xr.abs().max())
        info_b = lapack_arm.blas_info()
        out[p] = {"value": fl / (ms * 1e-3) / 1e12, "unit": "TFLOP/s", "ms_per_step": ms,
                  "factor_backward_error": bwd, "rel_diff_vs_cpu_arm": rel,
                  "vendor": {"value": fl / (vms * 1e-3) / 1e12, "ms": vms, "rel_diff_vs_cpu_arm": rel_v},
                  "cpu_arm": {"value": fl / cpu_s / 1e12, "s": cpu_s, "cores": info_b.get("threads"),
                              "info": int(cinfo)}}
        del A, Acm, Aw, Xw, Bt, Xv, Xr, X
        torch.cuda.empty_cache()
    return {"metric": "pposv TFLOP/s (plain path) on the SE-kernel matrices", "unit": "TFLOP/s",
            "config": {"workload": f"pposv d and z uplo=L n={n} nrhs={nrhs}, A = K + 1e-2 I, SE kernel l=0.2 on "
                                   "points U[0,1]^3 (z: K exp(i k.(x-y)), k ~ N(0, I3)), B ~ N(0,1)",
                       "flops": "d: n^3/3 + 2 n^2 nrhs; z: 4 n^3/3 + 8 n^2 nrhs"}, **out}


def kappa_leg(args, torch, device, h, stream, C, mixed_solve_fn):
    """The Householder family at every kappa of its configuration (1e2, 1e6, 1e10) for both
    tensor-core precisions: one device-timed mixed solve each, with the refinement report (sweeps,
    GMRES use, diagonal shift, FP64 fallback), the normwise backward error and the forward error
    against the exact solution U diag(1/s) U^T B."""
    from libddla_b200.workloads import householder_factors, householder_solve, householder_spd

    n, nrhs = args.n, args.nrhs
    out = {}
    g = torch.Generator(device=device).manual_seed(0xDD1A0103)
    B0 = torch.randn(nrhs, n, generator=g, device=device, dtype=torch.float64)
    for kappa in (1e2, 1e6, 1e10):
        A = householder_spd(n, kappa, 0xDD1A0003, device=device)
        s, vs = householder_factors(n, kappa, 0xDD1A0003, device=device)
        Xex = householder_solve(s, vs, B0.T)
        an = float(A.abs().sum(dim=0).max())
        for prec in ("B", "T"):
            ms, info, rep, X = mixed_solve_fn(A, B0, prec)
            R = B0.T - A @ X.T
            bwd = float((R.abs().max(dim=0).values / (an * X.T.abs().max(dim=0).values)).max())
            fwd = float(((X.T - Xex).abs().max(dim=0).values / Xex.abs().max(dim=0).values).max())
            out[f"{prec} kappa={kappa:g}"] = {
                "ms": ms, "tflops": flops_pposv(n, nrhs) / (ms * 1e-3) / 1e12, "info": info, "iter": rep["iter"],
                "gmres": rep["gmres"], "shift": rep["shift"], "fp64_fallback": rep["iter"] < 0,
                "backward_error": bwd, "forward_error_vs_exact": fwd}
            del R, X
        del A, Xex
        torch.cuda.empty_cache()
    return {"config": {"workload": f"pposv_mixed d n={n} nrhs={nrhs} A=U diag(s) U^T, s geometric 1..1/kappa",
                       "forward_error": "max over columns of ||x - x*||_inf / ||x*||_inf, x* = U diag(1/s) U^T b"},
            **out}


def gemm_vbatched_leg(args, torch, device, h, stream, C):
    """Variable-size batched GEMM (gemmVbatched): 2000 entries, m, n, k uniform in [32, 256],
    C_i = A_i B_i + 0.5 C_i, column-major with tight leading dimensions, for s/d/c/z.  Timed
    through the kernel layer (ddlak_gemm_vbatched, kernel only) and through the public C ABI
    (ddla_?_gemm_vbatched: the device validation pass and its read-back included); 8 entries
    are checked against a torch FP64 product."""
    lib = C.lib
    f = lib.ddlak_gemm_vbatched
    f.restype = ctypes.c_int
    f.argtypes = ([ctypes.c_char, ctypes.c_char, ctypes.c_char, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 11
                  + [ctypes.c_int, ctypes.c_void_p])
    out = {}
    nb, reps = 2000, 20
    rng = np.random.default_rng(0xDD1A0006)
    m, n, k = (rng.integers(32, 257, nb).astype(np.int32) for _ in range(3))
    mk, kn, mn = (a.astype(np.int64) * b for a, b in ((m, k), (k, n), (m, n)))
    offA, offB, offC = (np.concatenate([[0], np.cumsum(x)[:-1]]) for x in (mk, kn, mn))
    dm, dn, dk = (torch.from_numpy(x).to(device) for x in (m, n, k))
    for code, tdt, sdt in (("s", torch.float32, np.float32), ("d", torch.float64, np.float64),
                           ("c", torch.complex64, np.complex64), ("z", torch.complex128, np.complex128)):
        g = torch.Generator(device=device).manual_seed(0xDD1A0006)
        A = torch.randn(int(mk.sum()), dtype=tdt, device=device, generator=g)
        B = torch.randn(int(kn.sum()), dtype=tdt, device=device, generator=g)
        C0 = torch.randn(int(mn.sum()), dtype=tdt, device=device, generator=g)
        Cw = C0.clone()
        es = A.element_size()
        pa, pb, pc = (torch.from_numpy(t.data_ptr() + off * es).to(device) for t, off in ((A, offA), (B, offB),
                                                                                             (Cw, offC)))
        al, be = np.array([1.0], dtype=sdt), np.array([0.5], dtype=sdt)
        torch.cuda.synchronize()

        def kernel_call():
            rc = f(code.encode(), b"N", b"N", int(m.max()), int(n.max()), dm.data_ptr(), dn.data_ptr(), dk.data_ptr(),
                   al.ctypes.data, pa.data_ptr(), dm.data_ptr(), pb.data_ptr(), dk.data_ptr(), be.ctypes.data,
                   pc.data_ptr(), dm.data_ptr(), nb, stream.cuda_stream)
            assert rc == 0, rc

        def api_call():
            fn = getattr(C, f"ddla_{code}_gemm_vbatched")
            C.check_status(fn(h.ptr, b"N", b"N", dm.data_ptr(), dn.data_ptr(), dk.data_ptr(), al.ctypes.data,
                              pa.data_ptr(), dm.data_ptr(), pb.data_ptr(), dk.data_ptr(), be.ctypes.data,
                              pc.data_ptr(), dm.data_ptr(), nb), "gemm_vbatched")

        # parity: one call on a fresh C, 8 entries against torch in FP64
        kernel_call()
        torch.cuda.synchronize()
        hi = torch.complex128 if code in "cz" else torch.float64
        err = 0.0
        for i in rng.choice(nb, 8, replace=False):
            a = A[offA[i]:offA[i] + mk[i]].view(int(k[i]), int(m[i])).t().to(hi)
            b = B[offB[i]:offB[i] + kn[i]].view(int(n[i]), int(k[i])).t().to(hi)
            c0 = C0[offC[i]:offC[i] + mn[i]].view(int(n[i]), int(m[i])).t().to(hi)
            want = a @ b + 0.5 * c0
            got = Cw[offC[i]:offC[i] + mn[i]].view(int(n[i]), int(m[i])).t().to(hi)
            err = max(err, float((got - want).abs().max() / want.abs().max()))
        assert err < (1e-4 if code in "sc" else 1e-12), (code, err)
        flops = float((2.0 * m.astype(np.float64) * n * k).sum()) * (4 if code in "cz" else 1)
        res = {"max_rel_err_vs_torch_fp64": err}
        for name, fn in (("kernel", kernel_call), ("api", api_call)):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            res[name] = {"ms": ms, "tflops": flops / ms / 1e9}
        out[code] = res
    return {"metric": "batched GEMM TFLOP/s", "unit": "TFLOP/s",
            "config": {"workload": "2000 entries, m, n, k ~ U[32, 256], NN, alpha 1, beta 0.5, tight ld",
                       "launch": "one validation pass + one tiled launch per call"}, **out}


def batched_leg(args, torch, device, h, stream, C):
    """4096 matrices, n_i uniform in [16, 512], A_i = G_i G_i^T / n_i + 0.1 I, b_i ~ N(0, 1):
    one persistent launch replayed from a CUDA graph (VbatchedPlan) vs a per-matrix loop
    of the plain path (ddla.pposv + ddla.diag_logdet) on a sample of the same matrices."""
    from libddla_b200 import ddla
    from libddla_b200.ddla import batched

    out = {}
    count = args.batched_count
    g = torch.Generator(device=device).manual_seed(0xDD1A0004)
    orders = np.random.default_rng(0xDD1A0004).integers(16, 513, size=count)
    for tname, dt, code in (("f64", torch.float64, "d"), ("f32", torch.float32, "s")):
        es = 8 if dt == torch.float64 else 4
        sizes = (orders.astype(np.int64) ** 2 + 31) // 32 * 32
        aoff = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        voff = np.concatenate([[0], np.cumsum((orders.astype(np.int64) + 31) // 32 * 32)[:-1]])
        mats = torch.zeros(int(sizes.sum()), dtype=dt, device=device)
        rhs = torch.zeros(int(voff[-1] + 512), dtype=dt, device=device)
        for nv in np.unique(orders):
            idx = np.nonzero(orders == nv)[0]
            G = torch.randn(len(idx), nv, nv, generator=g, device=device, dtype=torch.float64)
            M = (G @ G.transpose(1, 2) / nv + 0.1 * torch.eye(nv, device=device, dtype=torch.float64)).to(dt)
            for k, i in enumerate(idx):
                mats[aoff[i]:aoff[i] + nv * nv] = M[k].reshape(-1)
                rhs[voff[i]:voff[i] + nv] = torch.randn(nv, generator=g, device=device, dtype=torch.float64).to(dt)
        pb = batched.PackedBatch(
            dtype=np.dtype(np.float64 if dt == torch.float64 else np.float32), orders=orders.astype(np.int32),
            a_offsets=aoff, b_offsets=voff, mats=mats, rhs=rhs,
            d_n=torch.from_numpy(orders.astype(np.int32)).to(device),
            d_lda=torch.from_numpy(orders.astype(np.int32)).to(device),
            d_A=torch.from_numpy((mats.data_ptr() + aoff * es).astype(np.int64)).to(device),
            d_B=torch.from_numpy((rhs.data_ptr() + voff * es).astype(np.int64)).to(device),
            logdet=torch.zeros(count, dtype=torch.float64, device=device),
            info=torch.zeros(count, dtype=torch.int32, device=device), max_n=512)
        A0, B0 = mats.clone(), rhs.clone()
        torch.cuda.synchronize()  # made on torch's stream, read on the library's
        batched.autotune(h, code, 512)
        plan = batched.VbatchedPlan(h, pb)
        flops = plan.info()["flops"]

        def restore():
            with torch.cuda.stream(stream):
                mats.copy_(A0)
                rhs.copy_(B0)

        for _ in range(args.warmup):
            restore()
            plan.run()
        torch.cuda.synchronize()
        times = []
        for _ in range(args.steps):
            restore()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.run()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = statistics.median(times)
        bad = int((pb.info != 0).sum())
        plan.close()
        # per-matrix loop of the plain path (device-resident inputs), on a sample
        rs = np.random.default_rng(5)
        sample = rs.choice(count, size=min(64, count), replace=False)
        dev = []
        for i in sample:
            nv = int(orders[i])
            Ai = A0[aoff[i]:aoff[i] + nv * nv].clone()
            bi = B0[voff[i]:voff[i] + nv].clone()
            dev.append((Ai, bi, ddla.DistributedMatrix.wrap(h, Ai.data_ptr(), nv, nv, nv, pb.dtype, mb=256, nb=256),
                        ddla.DistributedMatrix.wrap(h, bi.data_ptr(), nv, 1, nv, pb.dtype, mb=256, nb=256)))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _, _, dA, dB in dev:
            ddla.pposv(dA, dB)
            ddla.diag_logdet(dA)
        torch.cuda.synchronize()
        loop_rate = len(dev) / (time.perf_counter() - t0)
        rate = count / (ms * 1e-3)
        out[tname] = {"value": rate, "unit": "matrices/s", "ms_per_step": ms, "tflops": flops / (ms * 1e-3) / 1e12,
                      "failed": bad, "loop_value": loop_rate, "vs_loop": rate / loop_rate,
                      "tuning": batched.tuning(h, code, 512)["variant"]}
        del mats, rhs, A0, B0, pb, dev
    return {"metric": "batched factor+solve+logdet matrices/s", "unit": "matrices/s",
            "config": {"workload": f"{count} SPD matrices n_i ~ U[16,512], A_i = G_i G_i^T/n_i + 0.1 I, one rhs",
                       "launch": "one persistent kernel per step, replayed from a CUDA graph",
                       "loop": "per-matrix ddla.pposv + ddla.diag_logdet (plain path, device-resident), 64-matrix "
                               "sample", "l2": "3 GB of matrices > 126 MB L2"},
            **out}


def gp_leg(args, torch, device):
    """Batch of 256 GP likelihoods n=1024 (FP64), SE kernel on points in [0,1]^2, l=0.3,
    sigma^2=1e-2: loss and dloss/dtheta per step through libddla_b200.ddla.autograd; against a
    per-matrix torch.linalg (cuSOLVER) loop and torch's batched path.  Plus one n=16384 FP32."""
    from libddla_b200.ddla import autograd as ag

    g = torch.Generator(device=device).manual_seed(0xDD1A0005)
    B, n = args.gp_batch, 1024
    X = torch.rand(B, n, 2, generator=g, device=device, dtype=torch.float64)
    y = torch.randn(B, n, generator=g, device=device, dtype=torch.float64)
    th = torch.tensor([0.3, 1.0, 1e-2], dtype=torch.float64, device=device, requires_grad=True)

    dist = torch.distributed
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    red = torch.zeros(4, dtype=torch.float64, device=device)

    def ours():
        th.grad = None
        loss = ag.gp_nll(X, y, th).sum()
        loss.backward()
        if world > 1:
            # data-parallel fit: every rank holds its own problems; the summed likelihood and its
            # theta-gradient (4 doubles) are all-reduced once per step
            red[0] = loss.detach()
            red[1:] = th.grad
            dist.all_reduce(red)
        return loss

    def se(Xb, t):
        r2 = ((Xb[:, :, None, :] - Xb[:, None, :, :]) ** 2).sum(-1)
        return t[1] * torch.exp(-r2 / (2 * t[0] ** 2)) + t[2] * torch.eye(Xb.shape[1], dtype=Xb.dtype, device=device)

    def ref_one(b, t):
        L = torch.linalg.cholesky(se(X[b:b + 1], t)[0])
        a = torch.cholesky_solve(y[b].unsqueeze(-1), L).squeeze(-1)
        return 0.5 * ((y[b] * a).sum() + 2 * torch.log(torch.diagonal(L)).sum())

    def timed(fn, reps):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    ms = timed(ours, max(1, args.steps - 1))
    # one more step with per-kernel CUDA-event timing
    from libddla_b200.ddla import _c_api as C
    C.ddla_c_profile_read(-1, None, None, None, None, 1)
    C.ddla_c_profile_enable(1)
    ours()
    torch.cuda.synchronize()
    C.ddla_c_profile_enable(0)
    kern = read_kernels(C)
    grad = th.grad.clone()
    # torch reference gradient (FP64 autograd, batched) for the error line
    t2 = th.detach().clone().requires_grad_(True)
    K = se(X, t2)
    L = torch.linalg.cholesky(K)
    a = torch.cholesky_solve(y.unsqueeze(-1), L).squeeze(-1)
    (0.5 * ((y * a).sum(-1) + 2 * torch.log(torch.diagonal(L, dim1=-2, dim2=-1)).sum(-1))).sum().backward()
    rel = float(((grad - t2.grad).abs().max() / t2.grad.abs().max()).item())
    del K, L, a

    def torch_batched():
        t = th.detach().clone().requires_grad_(True)
        K = se(X, t)
        Lb = torch.linalg.cholesky(K)
        ab = torch.cholesky_solve(y.unsqueeze(-1), Lb).squeeze(-1)
        (0.5 * ((y * ab).sum(-1) + 2 * torch.log(torch.diagonal(Lb, dim1=-2, dim2=-1)).sum(-1))).sum().backward()

    tb = timed(torch_batched, 2)
    nloop = min(32, B)

    def torch_loop():
        t = th.detach().clone().requires_grad_(True)
        tot = sum(ref_one(b, t) for b in range(nloop))
        tot.backward()

    tl = timed(torch_loop, 2)
    rate = B / (ms * 1e-3)
    loop_rate = nloop / (tl * 1e-3)
    # one large float32 problem (blocked kernels)
    n2 = 16384
    X2 = torch.rand(1, n2, 2, generator=g, device=device, dtype=torch.float32)
    y2 = torch.randn(1, n2, generator=g, device=device, dtype=torch.float32)
    th2 = torch.tensor([0.3, 1.0, 1e-2], dtype=torch.float64, device=device, requires_grad=True)

    def big():
        th2.grad = None
        ag.gp_nll(X2, y2, th2).sum().backward()

    ms_big = timed(big, 1) if not args.no_gp_large else None
    big_err = None
    if not args.no_gp_large:
        big_err = gp_large_gradient_check(torch, device, X2, y2, th2.grad.detach().clone())
    return {"metric": "GP marginal likelihood logdet+grad evaluations/s", "value": rate * world, "unit": "1/s",
            "ms_per_step": ms, "dtype": "f64", "ranks": world,
            "exchange": "all-reduce (sum) of the likelihood and dloss/dtheta, 4 doubles per step" if world > 1
            else "none (one rank)",
            "config": {"workload": f"{B} x n={n} SE-kernel GPs, points U[0,1]^2, l=0.3 sigma_f^2=1 sigma^2=1e-2, "
                                   "loss = 1/2 (y^T A^-1 y + logdet A), dloss/dtheta by the adjoint kernels",
                       "loop": f"torch.linalg.cholesky/cholesky_solve + autograd one matrix at a time "
                               f"({nloop}-matrix sample)"},
            "kernels": kern,
            "loop_value": loop_rate, "vs_loop": rate / loop_rate, "torch_batched_value": B / (tb * 1e-3),
            "grad_rel_err_vs_torch_fp64": rel,
            "single_n16384_f32_ms": ms_big, "single_n16384_f32_grad_check": big_err}


def gp_large_gradient_check(torch, device, X, y, grad):
    """dloss/dtheta of the n=16384 FP32 problem against FP64 torch autograd on the same points, with
    torch's own FP32 autograd gradient beside it as the error a same-precision computation makes."""
    def torch_grad(dt):
        t = torch.tensor([0.3, 1.0, 1e-2], dtype=torch.float64, device=device, requires_grad=True)
        Xd = X[0].to(dt)
        r2 = torch.cdist(Xd, Xd).square_()
        K = t[1].to(dt) * torch.exp(-r2 / (2 * t[0].to(dt) ** 2))
        del r2
        K = K + t[2].to(dt) * torch.eye(Xd.shape[0], dtype=dt, device=device)
        L = torch.linalg.cholesky(K)
        del K
        yd = y[0].to(dt)
        a = torch.cholesky_solve(yd.unsqueeze(-1), L).squeeze(-1)
        (0.5 * ((yd * a).sum() + 2 * torch.log(torch.diagonal(L)).sum())).backward()
        return t.grad.detach().clone()

    g64 = torch_grad(torch.float64)
    torch.cuda.empty_cache()
    g32 = torch_grad(torch.float32)
    torch.cuda.empty_cache()
    rel = lambda g: float(((g - g64).abs() / g64.abs()).max())
    return {"ours_rel_err_vs_fp64": rel(grad), "torch_f32_rel_err_vs_fp64": rel(g32),
            "grad": grad.tolist(), "grad_fp64": g64.tolist()}


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch

    from libddla_b200 import ddla
    from libddla_b200.workloads import householder_spd

    C = ddla._c_api
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    n, nrhs = args.n, args.nrhs
    h = ddla.Handle(ddla.Backend.GPU)
    sp = ctypes.c_void_p()
    C.check_status(C.ddla_c_get_stream(h.ptr, ctypes.byref(sp)), "get_stream")
    stream = torch.cuda.ExternalStream(sp.value, device=device)

    A0 = householder_spd(n, args.kappa, 0xDD1A0003 + rank, device=device)  # symmetric: row-major == column-major
    Apristine = A0.clone()
    gB = torch.Generator(device=device).manual_seed(0xDD1A0103 + rank)
    B0 = torch.randn(nrhs, n, generator=gB, device=device, dtype=torch.float64)  # column-major n x nrhs
    X = torch.empty_like(B0)
    torch.cuda.synchronize()
    desc = lambda ptr, rows, cols: ddla.DistributedMatrix.wrap(h, ptr, rows, cols, n, np.float64, mb=256, nb=256)
    dA0 = desc(A0.data_ptr(), n, n)
    dB0 = desc(B0.data_ptr(), n, nrhs)
    dX = desc(X.data_ptr(), n, nrhs)
    rep_arr = (ctypes.c_double * 4)()

    def mixed_solve(prec):
        info = ctypes.c_int(0)
        C.check_status(C.ddla_d_pposv_mixed(h.ptr, b"L", prec.encode(), n, nrhs, dA0.data_ptr, dA0.desc.ctypes.data,
                                            dB0.data_ptr, dB0.desc.ctypes.data, dX.data_ptr, dX.desc.ctypes.data,
                                            ctypes.byref(info), rep_arr), "pposv_mixed")
        return info.value, {"iter": int(rep_arr[0]), "gmres": int(rep_arr[1]), "shift": rep_arr[2],
                            "backward_error": rep_arr[3]}

    def backward_error(Xt) -> float:
        R = B0.T - A0 @ Xt.T
        an = A0.abs().sum(dim=0).max()
        return float((R.abs().max(dim=0).values / (an * Xt.T.abs().max(dim=0).values)).max())

    def timed(fn, pre=None):
        """W warm-up + K device-timed calls; returns (total ms, per-step results, kernels, launches, clocks)."""
        for _ in range(args.warmup):
            if pre:
                pre()
            fn()
        torch.cuda.synchronize()
        launches0 = C.ddla_c_launch_count()
        C.ddla_c_profile_read(-1, None, None, None, None, 1)
        C.ddla_c_profile_enable(1)
        times, res = [], []
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        with ClockSampler(torch.cuda.current_device()) as clk:
            for _ in range(args.steps):
                if pre:
                    pre()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                res.append(fn())
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        C.ddla_c_profile_enable(0)
        launches = C.ddla_c_launch_count() - launches0
        total = torch.tensor([sum(times)], device=device, dtype=torch.float64)
        if world > 1:
            torch.distributed.all_reduce(total, op=torch.distributed.ReduceOp.MAX)
        return float(total.item()), res, read_kernels(C), launches, clk.summary()

    tf = lambda total_ms: world * flops_pposv(n, nrhs) * args.steps / (total_ms * 1e-3) / 1e12

    only = args.only
    if only in ("batched", "gp", "gemm-vbatched"):
        # one secondary leg alone (a profiling driver): its object is the line
        if only == "batched":
            leg = batched_leg(args, torch, device, h, stream, C)
        elif only == "gp":
            leg = gp_leg(args, torch, device)
        else:
            leg = gemm_vbatched_leg(args, torch, device, h, stream, C)
        if rank == 0:
            print(json.dumps({"only": only, only: leg}), flush=True)
        h.destroy()
        return

    def mixed_solve_on(A, Bt, prec):
        """One device-timed mixed solve of A X = B (A n x n symmetric, Bt nrhs x n) -> (ms, info, report, Xt)."""
        Xt = torch.empty_like(Bt)
        dA = desc(A.data_ptr(), n, n)
        dB = desc(Bt.data_ptr(), n, nrhs)
        dXo = desc(Xt.data_ptr(), n, nrhs)
        info = ctypes.c_int(0)
        rep = (ctypes.c_double * 4)()
        Asave = A.clone()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        C.check_status(C.ddla_d_pposv_mixed(h.ptr, b"L", prec.encode(), n, nrhs, dA.data_ptr, dA.desc.ctypes.data,
                                            dB.data_ptr, dB.desc.ctypes.data, dXo.data_ptr, dXo.desc.ctypes.data,
                                            ctypes.byref(info), rep), "pposv_mixed")
        e1.record(stream)
        e1.synchronize()
        A.copy_(Asave)  # the FP64 fallback leaves its factor in A
        del Asave
        return (e0.elapsed_time(e1), info.value,
                {"iter": int(rep[0]), "gmres": int(rep[1]), "shift": rep[2], "backward_error": rep[3]}, Xt)

    if only in ("vendor", "se-kernel", "kappa"):
        if only == "vendor":
            leg = vendor_leg(args, torch, A0, B0, backward_error)
        elif only == "se-kernel":
            del A0, Apristine
            torch.cuda.empty_cache()
            leg = se_kernel_leg(args, torch, device, h, stream, C)
        else:
            leg = kappa_leg(args, torch, device, h, stream, C, mixed_solve_on)
        if rank == 0:
            print(json.dumps({"only": only, only: leg}), flush=True)
        h.destroy()
        return

    # ---- mixed precision + refinement (headline) ----
    mixed = {}
    precs = ("B", "T") if only is None else ((only[-1],) if only.startswith("mixed-") else ())
    if only == "plain":
        precs = ()
    for prec in precs:
        fell_back = [False]

        def solve_and_note(prec=prec):
            r = mixed_solve(prec)
            fell_back[0] = r[1]["iter"] < 0  # the FP64 fallback overwrote A with its factor
            return r

        def restore_if_needed():
            if fell_back[0]:
                with torch.cuda.stream(stream):
                    A0.copy_(Apristine)
                fell_back[0] = False

        total, res, kern, launches, clocks = timed(solve_and_note, pre=restore_if_needed)
        restore_if_needed()
        info, rep = res[-1]
        assert info == 0, (prec, info)
        mixed[prec] = {"value": tf(total), "ms_per_step": total / args.steps, "report": rep,
                       "backward_error": backward_error(X), "kernels": kern, "launches": launches, "clocks": clocks}
    if only == "plain":
        mixed = {}
    best = max(mixed, key=lambda p: mixed[p]["value"] if mixed[p]["report"]["iter"] >= 0 else -1) if mixed else None
    head = mixed[best] if mixed else None

    # ---- plain FP64 ----
    plain = None
    if not args.no_plain and only in (None, "plain"):
        A = torch.empty_like(A0)
        dA = desc(A.data_ptr(), n, n)

        def restore():
            with torch.cuda.stream(stream):
                A.copy_(A0)
                X.copy_(B0)

        def plain_solve():
            _, info = ddla.pposv(dA, dX, "L")
            return info

        total, res, kern, launches, clocks = timed(plain_solve, pre=restore)
        assert all(r == 0 for r in res)
        plain = {"value": tf(total), "ms_per_step": total / args.steps, "backward_error": backward_error(X),
                 "kernels": kern, "launches": launches}
        del A

    if only is not None:
        # one leg alone (a profiling driver): no e2e, CPU or secondary figures
        if rank == 0:
            print(json.dumps({"only": only, "mixed": mixed, "plain": plain}), flush=True)
        h.destroy()
        return

    # ---- e2e through the public API with host buffers (headline path) ----
    # ddla_d_pposv_mixed_host takes A, B and X in (pinned) host memory: A's lower
    # triangle (the part uplo 'L' references, as LAPACK) streams to the device in
    # 512-column panels while the panels that have arrived are already factored,
    # so the host-to-device copy overlaps the factorization; X comes back to host
    # memory inside the call.
    E2E_PANEL = 128 * 4
    Ah = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    Ah.copy_(A0)  # symmetric: row-major storage == column-major A
    Bh = torch.empty((nrhs, n), dtype=torch.float64, pin_memory=True)
    Bh.copy_(B0)
    Xh = torch.empty((nrhs, n), dtype=torch.float64, pin_memory=True)
    h2d_a = 0
    for j0 in range(0, n, E2E_PANEL):
        h2d_a += (n - j0) * min(E2E_PANEL, n - j0) * 8

    def e2e_solve():
        info = ctypes.c_int(0)
        C.check_status(C.ddla_d_pposv_mixed_host(h.ptr, b"L", best.encode(), n, nrhs, Ah.data_ptr(), n,
                                                 Bh.data_ptr(), n, Xh.data_ptr(), n, ctypes.byref(info), rep_arr),
                       "pposv_mixed_host")
        return info.value

    e2e_solve()  # warm-up: the stream-ordered pool maps its workspace once
    e2e_ms = []
    for _ in range(max(1, min(3, args.steps))):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_info = e2e_solve()
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        assert e2e_info == 0 and int(rep_arr[0]) >= 0, (e2e_info, list(rep_arr))
    e2e_rep = {"iter": int(rep_arr[0]), "gmres": int(rep_arr[1]), "shift": rep_arr[2], "backward_error": rep_arr[3]}
    X.copy_(Xh.to(device))
    e2e_bwd = backward_error(X)
    assert e2e_bwd < 10 * n * 2.2e-16, e2e_bwd
    e2e_value = world * flops_pposv(n, nrhs) / (statistics.median(e2e_ms) * 1e-3) / 1e12

    peaks = measured_peaks()
    traffic = traffic_summary()
    dom = head["kernels"].get("mixed_update", {})
    gbs = dom["bytes"] / (dom["ms"] * 1e-3) / 1e9 if dom.get("ms") else None
    hbm = peaks.get("hbm_gbs") or 6650.0
    roof = {"bound": "hbm", "kernel": "k_mixed_update_cta2 / k_mixed_update_pair / k_mixed_update (tcgen05 trailing update, FP32 W read-modify-write)",
            "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm if gbs else None,
            # DRAM bytes per launch: the measured bytes per 128 x 128 tile times the tiles an average launch updates
            "traffic": (traffic["k_mixed_update"]["bytes_per_tile"] * (dom["bytes"] / dom["launches"]) /
                        traffic["k_mixed_update"]["algorithmic_bytes_per_tile"])
            if dom.get("launches") and "bytes_per_tile" in traffic.get("k_mixed_update", {}) else None,
            "traffic_source": "profiles/dram_traffic.json (one-launch capture at n=8192, per tile, scaled)",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks.get("hbm_gbs") else "fallback 6650 GB/s",
            "launches": dom.get("launches"), "avg_launch_ms": (dom["ms"] / dom["launches"]) if dom.get("launches") else None}
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"pposv d uplo=L n={n} nrhs={nrhs} A=U diag(s) U^T kappa={args.kappa:g}",
                   "path": f"mixed+IR precision {best} (tcgen05 {'BF16' if best == 'B' else 'TF32'} factor, "
                           f"FP64 refinement)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU 1x1 grid",
                   "l2": "inputs 8.6 GB > 126 MB L2, no flush", "report": head["report"],
                   "backward_error": head["backward_error"]},
        "roofline": roof,
        "mixed": {p: {k: v for k, v in d.items() if k != "kernels"} for p, d in mixed.items()},
        "plain": None if plain is None else dict(
            {k: v for k, v in plain.items() if k != "kernels"},
            kernels={name: dict(d, per_launch_ms=d["ms"] / d["launches"],
                                gbs=(d["bytes"] / (d["ms"] * 1e-3) / 1e9) if d["ms"] else None,
                                tflops=(d["flops"] / (d["ms"] * 1e-3) / 1e12) if d["ms"] else None)
                     for name, d in plain["kernels"].items()}),
        "kernels": head["kernels"],
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_a + Bh.numel() * 8,
                "d2h_bytes_per_step": Xh.numel() * 8, "ms_per_step": statistics.median(e2e_ms),
                "call": "ddla_d_pposv_mixed_host (A, B, X in pinned host memory)",
                "copies": f"A's lower triangle (the part uplo 'L' references) in {E2E_PANEL}-column panels, "
                          f"overlapped with the left-looking factorization of the panels already on the device; "
                          f"B in, X out",
                "report": e2e_rep, "backward_error": e2e_bwd},
        "gpu_launches": int(head["launches"]),
        "clocks": head["clocks"],
    }
    if plain is not None:
        dm = plain["kernels"].get("syrk_update", {})
        ach = dm["flops"] / (dm["ms"] * 1e-3) / 1e12 if dm.get("ms") else None
        fp64 = fp64_peak_tflops(torch, device)
        line["roofline_plain"] = {"bound": "tensor", "kernel": "k_syrk_dmma (FP64 DMMA trailing update)",
                                  "achieved": ach, "peak": fp64, "unit": "TFLOP/s", "frac": ach / fp64 if ach else None,
                                  "traffic": traffic.get("k_syrk_dmma", {}).get("bytes_per_launch_at_bench"),
                                  "peak_source": "cuBLAS DGEMM 8192^3 best-of-5 measured in this run"}
        line["speedup_mixed_over_plain"] = head["value"] / plain["value"]
    if not args.no_vendor:
        line["vendor"] = vendor_leg(args, torch, A0, B0, backward_error)
        line["vendor"]["plain_over_vendor"] = plain["value"] / line["vendor"]["value"] if plain else None
        line["vendor"]["mixed_over_vendor"] = head["value"] / line["vendor"]["value"]
    if not args.no_kappa:
        line["kappa"] = kappa_leg(args, torch, device, h, stream, C, mixed_solve_on)
    if not args.no_se:
        del Apristine
        torch.cuda.empty_cache()
        line["se_kernel"] = se_kernel_leg(args, torch, device, h, stream, C)
    if not args.no_batched:
        line["batched"] = batched_leg(args, torch, device, h, stream, C)
    if not args.no_gp:
        line["gp"] = gp_leg(args, torch, device)
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu_tf, sample, info = cpu_sample(budget_s=12.0, nrhs=nrhs, kappa=args.kappa)
        line["cpu_baseline"] = {"value": cpu_tf, "unit": UNIT,
                                "cores": int(info.get("threads") or os.cpu_count()), "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    h.destroy()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=32768)
    ap.add_argument("--nrhs", type=int, default=8)
    ap.add_argument("--kappa", type=float, default=1e6)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=8.0,
                    help="seconds of CPU work per step of the reference arm's bounded sample")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-vendor", action="store_true")
    ap.add_argument("--no-kappa", action="store_true")
    ap.add_argument("--no-se", action="store_true")
    ap.add_argument("--se-n", type=int, default=16384)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-gp", action="store_true")
    ap.add_argument("--no-gp-large", action="store_true")
    ap.add_argument("--batched-count", type=int, default=4096)
    ap.add_argument("--gp-batch", type=int, default=256)
    ap.add_argument("--only", choices=["mixed-B", "mixed-T", "plain", "batched", "gp", "gemm-vbatched", "vendor",
                                                 "se-kernel", "kappa"],
                    default=None,
                    help="run one leg alone (profiling driver); prints that leg's figures only")
    args = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return 0
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
