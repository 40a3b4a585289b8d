"""Time-to-solution benchmark for the mixed-precision Cholesky-preconditioned PCG.

Metric: time to a 1e-10 FP64-checked relative residual ||b - A x|| / ||b|| on
one B200, for the switching mixed-precision factor (E4M3 / FP16 / FP32 trailing
updates chosen per step) next to the plain FP32-factor PCG on the same GPU.

Workload (default): n = 8192 dense SPD A = Q diag(sigma) Q^T in FP32 storage,
Q from QR of a seeded N(0,1) matrix, sigma geometric 1 -> 1e-6 (kappa = 1e6),
block 256, one right-hand side b ~ N(0,1).  Synthetic seeded inputs stand in
for the reference's generated matrices.  One "step" = factor + PCG to 1e-10 of
that system.  A (256 MiB) is larger than the 126 MB L2, so every step streams
it from HBM; no separate L2 flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mpchol|reference]

Under torchrun with N > 1 every rank solves its own system (replicas, no
collective on the data path): value = max over ranks of the time to solution.
`--impl reference` times the reference's own CPU path (its micro_cholesky,
src/micro_chol.hpp, built from the reference sources into oracle/_ref, or the
oracle's restatement of it) on the host cores.
"""
from __future__ import annotations

import argparse
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
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "time to 1e-10 FP64 residual: FP8/MXFP8-chol PCG vs FP32-chol PCG, one B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mpchol", choices=["mpchol", "reference"])
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--kappa", type=float, default=1e6)
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--eps-prime", type=float, default=1e-5)
    ap.add_argument("--precision", default="switching",
                    help="policy of the mixed arm: switching, e4m3, e5m2, fp16, fp16x2")
    ap.add_argument("--ladder", default="e4m3,fp16,fp16x2",
                    help="switching ladder, lowest precision first (its last entry is the "
                         "fallback)")
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--max-it", type=int, default=400)
    ap.add_argument("--check-every", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="spd", choices=["spd", "rbf", "rbf-grad", "batch"],
                    help="spd: the dense SPD time-to-solution workload (default); rbf: Gaussian "
                         "RBF kernel matrix, n=16384 points in [0,1]^784, 8 rhs; rbf-grad: "
                         "forward + adjoint gradients of 1/2 y^T K^-1 y, n=8192, d=64; batch: "
                         "512 SPD systems of order U[64, 2048]")
    return ap.parse_args()


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and throttle-reason sampling during a region (NVML reads every
    10 ms from a thread; nvidia-smi -lms 200 if NVML is not importable)."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}
    FALLBACK_BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40,
                     "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, pci_bus_id: str | None = None):
        self.index = index
        self.pci = pci_bus_id
        self.proc = None
        self.nvml = None
        self.samples = []          # (sm_mhz, max_mhz, set of reasons)
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = None
            if isinstance(self.pci, str):
                try:
                    h = nv.nvmlDeviceGetHandleByPciBusId(self.pci.encode())
                except Exception:
                    h = None
            if h is None:
                h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.nvml, self.h = nv, h
            self.bits = {k: getattr(nv, v, self.FALLBACK_BITS[k]) for k, v in self.REASONS.items()}
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _poll(self):
        nv, h = self.nvml, self.h
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx),
                                     {k for k, bit in self.bits.items() if r & bit}))
            except Exception:
                return
            time.sleep(0.01)

    def _read(self):
        names = list(self.FALLBACK_BITS)
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.strip().split(",")]
            if len(parts) < 8:
                continue
            try:
                self.samples.append((float(parts[0]), float(parts[1]),
                                     {nm for nm, v in zip(names, parts[4:8])
                                      if v.lower() == "active"}))
            except ValueError:
                continue

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        elif self.nvml is not None:
            self.t.join(timeout=1.0)

    def summary(self):
        sm = [s[0] for s in self.samples]
        mx = self.samples[-1][1] if self.samples else None
        reasons = set().union(*[s[2] for s in self.samples]) if self.samples else set()
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def pci_bus_id(torch, index: int):
    """NVML-style PCI bus id string ("DDDDDDDD:BB:DD.0") of a CUDA device."""
    p = torch.cuda.get_device_properties(index)
    ids = [getattr(p, k, None) for k in ("pci_domain_id", "pci_bus_id", "pci_device_id")]
    if not all(isinstance(v, int) for v in ids):
        return None
    return "%08X:%02X:%02X.0" % tuple(ids)


# ---------------------------------------------------------------- peaks
def measured_peaks():
    """(HBM GB/s, dense bf16 TFLOP/s burst, kind): the driver-measured copy
    bandwidth and cuBLAS bf16 rate of this GPU type, else the pool fallback."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def profiled_traffic(kernel: str, n: int):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    recorded from an ncu capture in profiles/<kernel>_n<n>.txt as a line
    'traffic_bytes_per_launch: <int>', or None."""
    p = ROOT / "profiles" / f"{kernel}_n{n}.txt"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        if ln.startswith("traffic_bytes_per_launch:"):
            try:
                return int(ln.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------- GPU arm
def run_gpu(args, world, rank, local):
    import torch
    import cholesky_gpu_b200 as mp
    from cholesky_gpu_b200 import _lib, matgen

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist
    lib = _lib.load()
    n, b = args.n, args.block
    seed = 3 + rank
    A = matgen.spd_matrix(n, args.kappa, seed, device=dev)
    B = matgen.rhs(n, 1, 100 + rank, device=dev)
    A_host = A.cpu().pin_memory()
    B_host = B.cpu().pin_memory()
    stream = torch.cuda.current_stream(dev)

    def solve_once(precision, Ad, Bd):
        f = mp.Factor(n, block_size=b, precision=precision, eps_prime=args.eps_prime)
        f.compute(Ad)
        X, rep = f.pcg(Ad, Bd, rel_tol=args.tol, max_it=args.max_it, check_every=args.check_every)
        return f, X, rep

    # factor objects are created outside the timed region (allocation is setup)
    # "switching" is the mixed-precision arm (its policy from --precision /
    # --ladder), "fp32" the plain FP32-factor comparator
    ladder = [x.strip() for x in args.ladder.split(",") if x.strip()]
    fobj = {"switching": mp.Factor(n, block_size=b, precision=args.precision,
                                   eps_prime=args.eps_prime, ladder=ladder),
            "fp32": mp.Factor(n, block_size=b, precision="fp32")}

    def step(precision):
        f = fobj[precision]
        f.compute(A)
        X, rep = f.pcg(A, B, rel_tol=args.tol, max_it=args.max_it, check_every=args.check_every)
        return X, rep

    def timed(precision, k):
        times, reps = [], []
        for _ in range(k):
            if pg:
                pg.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            X, rep = step(precision)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            reps.append(rep)
        return times, reps

    for _ in range(args.warmup):
        step("switching")
        step("fp32")
    launches0 = lib.mpchol_kernel_launches()
    with ClockSampler(local, pci_bus_id(torch, local)) as clk:
        t_sw, r_sw = timed("switching", args.steps)
        launches_sw = lib.mpchol_kernel_launches() - launches0
        t_32, r_32 = timed("fp32", args.steps)
    info_sw = fobj["switching"].info()

    def mx(v):
        if pg:
            t = torch.tensor([v], dtype=torch.float64, device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            return t.item()
        return v

    ms_sw = mx(statistics.median(t_sw))
    ms_32 = mx(statistics.median(t_32))

    # end-to-end through the public API with host buffers: Factor.solve_host
    # (mpchol_solve_host) copies A's lower triangle (block columns from the
    # diagonal down) and b to the device, factors, runs PCG and copies x back
    e2e_times = []
    for i in range(max(2, min(args.steps, 3)) + 1):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        xh, rep = fobj["switching"].solve_host(A_host, B_host, rel_tol=args.tol,
                                               max_it=args.max_it, check_every=args.check_every)
        e1.record(stream)
        torch.cuda.synchronize()
        if i > 0:
            e2e_times.append(e0.elapsed_time(e1))
    e2e_h2d = sum((n - c) * min(b, n - c) for c in range(0, n, b)) * 4 + B_host.numel() * 8
    e2e_ms = mx(statistics.median(e2e_times))

    # per-phase breakdown of one profiled step (events inside the library)
    lib.mpchol_profile_enable(1)
    prof0 = _lib.Profile()
    lib.mpchol_profile_read(prof0, 1)
    _, rep_p = step("switching")
    torch.cuda.synchronize()
    prof = _lib.Profile()
    lib.mpchol_profile_read(prof, 1)
    lib.mpchol_profile_enable(0)
    phases = {nm: round(prof.ms[i], 4) for i, nm in enumerate(_lib.PHASE_NAMES) if prof.calls[i]}
    calls = {nm: int(prof.calls[i]) for i, nm in enumerate(_lib.PHASE_NAMES) if prof.calls[i]}

    # rooflines of the bandwidth- and tensor-bound phases of the profiled step;
    # the headline one is the phase with the largest device time
    hbm, bf16, peak_kind = measured_peaks()
    info_p = fobj["switching"].info()
    tc_flops, tc_bytes, tc_exec, tc_fmts = 0.0, 0.0, 0, {}
    panel_bytes = {_lib.PREC_FP16: 2, _lib.PREC_E4M3: 1, _lib.PREC_E5M2: 1, _lib.PREC_MXFP8: 1,
                   _lib.PREC_FP16X2: 4}
    for k, pr in enumerate(info_p.step_prec):
        s0 = k * b
        bs = min(b, n - s0)
        m = n - s0 - bs
        if m <= 0:
            break
        if pr != _lib.PREC_FP32:
            tc_flops += float(m) * (m + 1) * bs       # lower triangle, algorithmic
            # C lower triangle read + written in FP32, the quantized panel read once
            tc_bytes += float(m) * (m + 1) / 2 * 8 + float(m) * bs * panel_bytes.get(pr, 1)
            tc_exec += 1
            tc_fmts[pr] = tc_fmts.get(pr, 0) + 1
    by_phase = {}

    def add(name, bound, unit, peak, work, launches, note):
        if name not in phases or launches <= 0:
            return
        sec = phases[name] * 1e-3
        scale = 1e9 if unit == "GB/s" else 1e12
        achieved = work * launches / sec / scale
        by_phase[name] = {"bound": bound, "unit": unit, "achieved": round(achieved, 1),
                          "peak": peak, "frac": round(achieved / peak, 4),
                          "work_per_launch": work, "launches": launches,
                          "ms": phases[name], "note": note}

    tri = n * (n + 1) / 2 * 4 + 3 * n * 8
    add("trsv", "hbm", "GB/s", hbm, tri, calls.get("trsv", 0),
        "one triangular solve: lower triangle of L in FP32 + FP64 vectors")
    add("symv", "hbm", "GB/s", hbm, n * (n + 1) / 2 * 4 + 2 * n * 8, calls.get("symv", 0),
        "A x from the lower triangle of A in FP32, FP64 vectors")
    if tc_exec:
        # At b = 256 the trailing update moves 8 bytes of C per 2b (x3 for FP16X2)
        # flops: below the B200 ridge point, so HBM is the binding roof; the
        # tensor rate is reported beside it.
        fp8 = sum(v for k_, v in tc_fmts.items() if k_ in (_lib.PREC_E4M3, _lib.PREC_E5M2,
                                                             _lib.PREC_MXFP8))
        tpeak = 2 * bf16 if fp8 * 2 > tc_exec else bf16
        add("syrk_tc", "hbm", "GB/s", hbm, tc_bytes / tc_exec, tc_exec,
            "trailing update: C lower triangle read+write (FP32) + quantized panel per "
            "executing launch; tensor_tflops = m(m+1)b useful flops / time (FP16X2 issues 3x)")
        if "syrk_tc" in by_phase:
            tt = tc_flops / (phases["syrk_tc"] * 1e-3) / 1e12
            by_phase["syrk_tc"]["tensor_tflops"] = round(tt, 1)
            by_phase["syrk_tc"]["tensor_frac"] = round(tt / tpeak, 4)
            by_phase["syrk_tc"]["tensor_peak"] = tpeak
    dom = max(by_phase, key=lambda k_: by_phase[k_]["ms"]) if by_phase else None
    if dom:
        r = by_phase[dom]
        roof = {"kernel": dom, "bound": r["bound"], "achieved": r["achieved"], "peak": r["peak"],
                "peak_kind": peak_kind, "unit": r["unit"], "frac": r["frac"],
                "algorithmic_per_launch": r["work_per_launch"],
                "traffic": profiled_traffic(dom, n), "by_phase": by_phase}
    else:
        roof = {"kernel": None, "bound": "hbm", "achieved": None, "peak": hbm,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": None, "traffic": None}

    result = {
        "metric": METRIC,
        "value": round(ms_sw, 3),
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_sw, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "%s factor, fp64 pcg" % "/".join(
            nm for i, nm in ((2, "e4m3"), (3, "e5m2"), (1, "fp16"), (6, "fp16x2"), (0, "fp32"))
            if info_sw.steps_by_prec[i]),
        "data": "synthetic (seeded Q diag(sigma) Q^T, geometric spectrum)",
        "config": {"workload": (f"spd n={n} kappa={args.kappa:g} block={b} {args.precision}"
                                f" ladder={args.ladder} eps'={args.eps_prime}"),
                   "n": n, "kappa": args.kappa, "block": b, "rhs": 1, "tol": args.tol,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (A = %d MiB)" % (n * n * 4 // (1 << 20))},
        "comparator_fp32_factor_ms": round(ms_32, 3),
        "speedup_vs_fp32_factor": round(ms_32 / ms_sw, 3),
        "iterations": {"switching": r_sw[-1].iterations, "fp32": r_32[-1].iterations},
        "rel_residual": {"switching": r_sw[-1].rel_residual, "fp32": r_32[-1].rel_residual},
        "backward_error": {"switching": r_sw[-1].backward_error, "fp32": r_32[-1].backward_error},
        "step_precisions": {nm: info_sw.steps_by_prec[i]
                            for i, nm in ((0, "fp32"), (1, "fp16"), (2, "e4m3"), (3, "e5m2"),
                                          (4, "mxfp8"), (6, "fp16x2"))},
        "phase_ms_switching_step": phases,
        "phase_calls_switching_step": calls,
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms",
                "h2d_bytes_per_step": int(e2e_h2d),
                "d2h_bytes_per_step": int(n * 8)},
        "gpu_launches": int(launches_sw),
        "roofline": roof,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(args, A_host.numpy(), B_host.numpy(),
                                              r_32[-1].iterations)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return result if rank == 0 else None


# ---------------------------------------------------------------- CPU side
def cpu_baseline(args, A: np.ndarray, b: np.ndarray, iters: int, budget_s: float = 20.0):
    """Reference CPU path on a bounded sample: micro_cholesky (FP32,
    unblocked, single thread) on the leading n_s x n_s block, extrapolated by
    (n/n_s)^3, plus the measured cost of one FP64 PCG iteration at full n
    (FP32 GEMV + FP32-factor triangular solves) times the FP32 path's GPU
    iteration count."""
    from oracle import oracle as O

    n = A.shape[0]
    kind = "reference" if O.REF_MICRO.exists() else "port"
    ns = min(n, 1536)
    sub = np.array(A[:ns, :ns], dtype=np.float32, order="F")
    t0 = time.perf_counter()
    if kind == "reference":
        L, rc = O.ref_micro_cholesky(sub)
    else:
        L, rc = O.micro_cholesky(sub)
    t_sub = time.perf_counter() - t0
    t_factor = t_sub * (n / ns) ** 3
    # one PCG iteration at full n: GEMV (n^2 FP32) + two triangular solves
    F = np.asfortranarray(A.astype(np.float32))
    lib = O.lib()
    import ctypes
    x = np.ascontiguousarray(b, dtype=np.float64)
    y = np.zeros(n)
    dp = ctypes.POINTER(ctypes.c_double)
    t0 = time.perf_counter()
    lib.orc_gemv_f32_f64(F.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n, n,
                         x.ctypes.data_as(dp), y.ctypes.data_as(dp))
    lib.orc_potrs_f32_f64(F.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n, n,
                          x.ctypes.data_as(dp), y.ctypes.data_as(dp))
    t_it = time.perf_counter() - t0
    total_ms = (t_factor + (iters + 1) * t_it) * 1e3
    return {"value": round(total_ms, 1), "unit": "ms", "cores": 1, "kind": kind,
            "sample": (f"micro_cholesky on the leading {ns}x{ns} block ({t_sub:.2f} s) "
                       f"extrapolated by (n/{ns})^3 to n={n}, plus {iters + 1} x one measured "
                       f"FP64 PCG iteration at full n ({t_it * 1e3:.0f} ms)")}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    from cholesky_gpu_b200 import matgen
    n = args.n
    A = matgen.spd_matrix(n, args.kappa, 3).numpy()
    b = matgen.rhs(n, 1, 100).numpy()
    vals = []
    for _ in range(max(1, args.steps)):
        cb = cpu_baseline(args, A, b, iters=8)
        vals.append(cb["value"])
    v = statistics.median(vals)
    cb["value"] = v
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 factor, fp64 pcg",
        "data": "synthetic (seeded Q diag(sigma) Q^T, geometric spectrum)",
        "config": {"workload": f"spd n={n} kappa={args.kappa:g} block={args.block} (CPU micro_cholesky)",
                   "n": n, "kappa": args.kappa},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------- other workloads
def _timed(fn, steps, warmup, stream):
    import torch
    for _ in range(warmup):
        fn()
    times, last = [], None
    for _ in range(steps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        last = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return statistics.median(times), last


def _phases(fn):
    """Per-phase device times (library CUDA events) of one call of fn."""
    import torch
    from cholesky_gpu_b200 import _lib
    lib = _lib.load()
    lib.mpchol_profile_enable(1)
    p0 = _lib.Profile()
    lib.mpchol_profile_read(p0, 1)
    fn()
    torch.cuda.synchronize()
    p = _lib.Profile()
    lib.mpchol_profile_read(p, 1)
    lib.mpchol_profile_enable(0)
    return {nm: round(p.ms[i], 4) for i, nm in enumerate(_lib.PHASE_NAMES) if p.calls[i]}


def _base(args, world, value, unit, dtype, data, config, extra):
    out = {"metric": METRIC, "value": round(value, 3), "unit": unit, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(value, 3),
           "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
           "data": data, "config": config}
    out.update(extra)
    return out


def run_rbf(args, world, rank, local):
    """Gaussian RBF kernel matrix: n = 16384 points, 80 % zero coordinates,
    the rest U(0,1) in [0,1]^784 (seeded stand-in for image data);
    l = exact median pairwise distance; nugget 1e-3; 8 rhs.  One step =
    factor + PCG to the tolerance (the kernel-matrix build is timed apart)."""
    import torch
    import cholesky_gpu_b200 as mp
    from cholesky_gpu_b200 import autograd as AG, matgen
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n if args.n != 8192 else 16384
    X = torch.from_numpy(matgen.mnist_like_points(n, 784, 4 + rank)).to(dev)
    ell = matgen.median_pairwise_distance(X)
    stream = torch.cuda.current_stream(dev)
    t_build, (_, K32) = _timed(lambda: AG.rbf_build(X, ell, 1e-3, fp64=False), 1, 1, stream)
    B = matgen.rhs(n, 8, 5 + rank, device=dev)
    prec = args.precision
    mixed = dict(block_size=args.block, precision=prec)
    if prec == "switching":
        # MXFP8 first: the criterion keeps it only where the Schur diagonal allows
        mixed.update(eps_prime=args.eps_prime, ladder=["mxfp8", "fp16", "fp16x2"])
    arms = {prec: mp.Factor(n, **mixed),
            "fp32": mp.Factor(n, block_size=args.block, precision="fp32")}
    res = {}
    for name, f in arms.items():
        def step(f=f):
            f.compute(K32)
            return f.pcg(K32, B, rel_tol=args.tol, max_it=args.max_it, check_every=args.check_every)
        ms, (X_, rep) = _timed(step, args.steps, args.warmup, stream)
        res[name] = (ms, rep, _phases(step))
    ms, rep, _ = res[prec]
    info = arms[prec].info()
    steps_used = {nm: info.steps_by_prec[i] for i, nm in
                  ((0, "fp32"), (1, "fp16"), (2, "e4m3"), (3, "e5m2"), (4, "mxfp8"), (6, "fp16x2"))
                  if info.steps_by_prec[i]}
    return _base(args, world, ms, "ms", f"{'/'.join(steps_used) or prec} factor, fp64 pcg",
                 "synthetic (seeded sparse points in [0,1]^784, RBF kernel)",
                 {"workload": f"rbf n={n} d=784 l=median({ell:.3f}) nugget=1e-3 rhs=8 {prec}",
                  "n": n, "block": args.block, "rhs": 8, "tol": args.tol},
                 {"comparator_fp32_factor_ms": round(res["fp32"][0], 3),
                  "speedup_vs_fp32_factor": round(res["fp32"][0] / ms, 3),
                  "iterations": {k: v[1].iterations for k, v in res.items()},
                  "converged": {k: v[1].converged for k, v in res.items()},
                  "rel_residual": {k: v[1].rel_residual for k, v in res.items()},
                  "kernel_build_ms": round(t_build, 3), "step_precisions": steps_used,
                  "phase_ms": {k: v[2] for k, v in res.items()}})


def run_rbf_grad(args, world, rank, local):
    """Differentiation workload: RBF kernel, n = 8192 points x ~ N(0, I_64),
    l = 4, nugget 1e-2, y ~ N(0,1); one step = forward solve + backward
    (adjoint PCG reusing the factor, fused gradient contraction)."""
    import torch
    from cholesky_gpu_b200 import autograd as AG, matgen
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n if args.n != 8192 else 8192
    X0 = torch.from_numpy(matgen.gaussian_points(n, 64, 6 + rank)).to(dev)
    y = torch.from_numpy(np.random.default_rng(7 + rank).standard_normal(n)).to(dev)
    stream = torch.cuda.current_stream(dev)
    prec = args.precision
    res = {}
    for name in (prec, "fp32"):
        fopts = dict(block_size=args.block, precision=name)
        if name == "switching":
            fopts.update(eps_prime=args.eps_prime, ladder=["e4m3", "fp16", "fp16x2"])

        def step(fopts=fopts):
            Xt = X0.clone().requires_grad_(True)
            ell = torch.tensor(4.0, dtype=torch.float64, requires_grad=True)
            lam = torch.tensor(1e-2, dtype=torch.float64, requires_grad=True)
            x = AG.rbf_solve(Xt, ell, lam, y, rel_tol=1e-12, max_it=args.max_it, **fopts)
            loss = 0.5 * (y * x).sum()
            loss.backward()
            return loss.item(), ell.grad.item(), lam.grad.item()
        res[name] = _timed(step, args.steps, args.warmup, stream)
    ms, (loss, gl, gn) = res[prec]
    return _base(args, world, ms, "ms", f"{prec} factor, fp64 pcg + fp64 gradients",
                 "synthetic (seeded x ~ N(0, I_64))",
                 {"workload": f"rbf-grad n={n} d=64 l=4 nugget=1e-2 {prec}", "n": n,
                  "block": args.block, "tol": 1e-12},
                 {"comparator_fp32_factor_ms": round(res["fp32"][0], 3),
                  "speedup_vs_fp32_factor": round(res["fp32"][0] / ms, 3),
                  "loss": loss, "dL_dl": gl, "dL_dnugget": gn})


def run_batch(args, world, rank, local):
    """512 SPD systems, n_i ~ U[64, 2048], kappa_i log-uniform in [1e2, 1e6]
    (seeded), 4 rhs each; one step = batched factor + lockstep PCG of all."""
    import torch
    import cholesky_gpu_b200 as mp
    from cholesky_gpu_b200 import matgen
    from cholesky_gpu_b200.shard import gather_by_system, max_over_ranks, partition_systems
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    count = 512
    # the same 512 systems for every world size; each rank owns a shard (no
    # data-path collective: systems are independent)
    ns_all = [int(v) for v in matgen.batch_sizes(count, 64, 2048, 8)]
    ks = matgen.batch_kappas(count, 1e2, 1e6, 9)
    mine = partition_systems(ns_all, world)[rank]
    ns = [ns_all[i] for i in mine]
    As = [matgen.spd_matrix(ns_all[i], float(ks[i]), i, device=dev) for i in mine]
    Bs = [matgen.rhs(ns_all[i], 4, 7000 + i, device=dev) for i in mine]
    stream = torch.cuda.current_stream(dev)
    prec = args.precision if args.precision != "switching" else "fp16x2"
    bt = mp.Batch(ns, nrhs=4, block_size=128, precision=prec)

    def step():
        if dist is not None:
            dist.barrier()
        bt.factor(As)
        return bt.pcg(As, Bs, rel_tol=args.tol, max_it=args.max_it, check_every=args.check_every)
    ms, (Xs, reps, st) = _timed(step, args.steps, args.warmup, stream)
    ms = max_over_ranks(ms, dist)
    allrep = gather_by_system({i: (r.iterations, r.converged) for i, r in zip(mine, reps)},
                              count, dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None
    its = [r[0] for r in allrep]
    flops = sum(n ** 3 / 3.0 for n in ns_all)
    return _base(args, world, ms, "ms", f"{prec} factor, fp64 pcg",
                 "synthetic (seeded Q diag(sigma) Q^T per system)",
                 {"workload": f"batch 512 systems n~U[64,2048] kappa~logU[1e2,1e6] rhs=4 {prec}",
                  "systems": count, "block": 128, "rhs": 4, "tol": args.tol,
                  "parallelism": f"systems sharded over {world} GPUs" if world > 1 else "single GPU"},
                 {"scaling": "strong",
                  "solves_per_s": round(count / (ms * 1e-3), 1),
                  "ms_per_system": round(ms / count, 4),
                  "all_converged": all(r[1] for r in allrep),
                  "iterations": {"max": max(its), "median": statistics.median(its)},
                  "factor_tflops_equiv": round(flops / (ms * 1e-3) / 1e12, 2)})


def main():
    args = parse()
    world, rank, local = dist_init(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    elif args.workload == "rbf":
        out = run_rbf(args, world, rank, local)
    elif args.workload == "rbf-grad":
        out = run_rbf_grad(args, world, rank, local)
    elif args.workload == "batch":
        out = run_batch(args, world, rank, local)
    else:
        out = run_gpu(args, world, rank, local)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
