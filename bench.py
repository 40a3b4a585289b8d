"""Time-to-solution benchmark for the mixed-precision Cholesky-preconditioned PCG.

Metric: time to a 1e-10 FP64-checked relative residual ||b - A x|| / ||b|| on
one B200, for the switching mixed-precision factor (MXFP8 / FP16 / FP16X2
trailing updates chosen per step) next to the plain FP32-factor PCG on the
same GPU.

Workload (default, the precision-at-scale configuration): the Gaussian RBF
kernel matrix K_ij = exp(-||x_i - x_j||^2 / (2 l^2)) + 1e-3 delta_ij of
n = 16384 points in [0,1]^784 whose coordinates are 0 with probability 0.8
and U(0,1) otherwise (the seeded stand-in for the image data, which is not
available), l = the exact median pairwise distance, FP32 storage, block 256,
8 right-hand sides ~ N(0,1).  The mixed arm switches per step over the ladder
MXFP8 -> FP16 -> FP16X2 with eps' = 2 (the coherence rule keeps the constant
mode's step off FP8).  One "step" = factor + PCG to 1e-10 of all 8 rhs.  K
(1 GiB) is larger than the 126 MB L2, so every step streams it from HBM; no
separate L2 flush is needed.  `--workload spd` is the n = 8192, kappa = 1e6
SPD configuration; `rbf-grad` and `batch` the differentiation and batching
workloads.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mpchol|reference]

Under torchrun with N > 1 every rank solves its own system (replicas, no
collective on the data path): value = max over ranks of the time to solution.
`--impl reference` runs the reference's own CPU path (its micro_cholesky,
src/micro_chol.hpp, built from the reference sources into oracle/_ref, and a
host FP64 PCG) on the full workload, one step.
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
    ap.add_argument("--workload", default="rbf", choices=["rbf", "spd", "rbf-grad", "batch", "syrk"],
                    help="rbf (default): Gaussian RBF kernel matrix, n=16384 points in [0,1]^784 "
                         "with 80%% zero coordinates, nugget 1e-3, 8 rhs, MXFP8 switching ladder; "
                         "spd: n=8192 Q diag(sigma) Q^T, kappa=1e6, 1 rhs; rbf-grad: forward + "
                         "adjoint gradients of 1/2 y^T K^-1 y, n=8192, d=64; batch: 512 SPD "
                         "systems of order U[64, 2048]; syrk: trailing-update microbenchmark "
                         "against cuBLASLt MXFP8")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--rhs", type=int, default=None)
    ap.add_argument("--kappa", type=float, default=1e6)
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--eps-prime", type=float, default=None)
    ap.add_argument("--eps-coherence", type=float, default=None,
                    help="threshold of the switching rule's coherence test (0: eps')")
    ap.add_argument("--precision", default="switching",
                    help="policy of the mixed arm: switching, e4m3, e5m2, mxfp8, fp16, fp16x2")
    ap.add_argument("--ladder", default=None,
                    help="switching ladder, lowest precision first (its last entry is the "
                         "fallback)")
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--max-it", type=int, default=400)
    ap.add_argument("--check-every", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--factor-only", type=int, default=0, metavar="K",
                    help="run the mixed arm's factorization K times and exit without "
                         "timing or output (an entry point for profilers)")
    ap.add_argument("--tune", action="store_true",
                    help="batch workload: re-run the autotuner on this GPU and write its table")
    ap.add_argument("--tune-out", default=None,
                    help="where --tune writes the table (default: the package's tuned_batch.json)")
    args = ap.parse_args()
    w = WORKLOADS.get(args.workload, {})
    if args.n is None:
        args.n = w.get("n", 8192)
    if args.rhs is None:
        args.rhs = w.get("rhs", 1)
    if args.ladder is None:
        args.ladder = w.get("ladder", "e4m3,fp16,fp16x2")
    if args.eps_prime is None:
        args.eps_prime = w.get("eps", 1e-5)
    if args.eps_coherence is None:
        args.eps_coherence = w.get("eps_c", 0.0)
    return args


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
PREC_LETTER = {0: "S", 1: "h", 2: "e", 3: "f", 4: "M", 6: "X", 7: "a", 8: "b", 9: "q"}
PREC_KEYS = ((0, "fp32"), (1, "fp16"), (2, "e4m3"), (3, "e5m2"), (4, "mxfp8"), (6, "fp16x2"),
             (7, "mxfp6_e2m3"), (8, "mxfp6_e3m2"), (9, "mxfp4"))

# Per-workload defaults of the mixed arm: the switching ladder (lowest
# precision first), eps' and the coherence threshold eps_c.  RBF: eps' = 2
# admits MXFP8 after the constant mode; eps_c = 1/16 keeps the large, coherent
# early updates in FP16 and hands the remaining steps (51 of 63) to MXFP8,
# 5 PCG iterations (eps_c = eps' takes every step in MXFP8 and needs 14).
# SPD kappa = 1e6: FP8 is rejected by the Schur ratio at any useful eps', FP16X2
# carries the factor.
WORKLOADS = {
    "rbf": dict(n=16384, ladder="mxfp8,fp16,fp16x2", eps=2.0, eps_c=0.0625, rhs=8),
    "spd": dict(n=8192, ladder="e4m3,fp16,fp16x2", eps=1e-5, rhs=1),
}


def workload_inputs(args, rank, dev):
    """The system of the time-to-solution workloads, generated outside any
    timed region: (A FP32 n x n on the device, lower triangle valid; B FP64
    n x rhs; description)."""
    import torch
    from cholesky_gpu_b200 import autograd as AG, matgen
    n = args.n
    if args.workload == "rbf":
        # 16384 points in [0,1]^784, 80 % zero coordinates, the rest U(0,1)
        # (the seeded stand-in for the image data); l = exact median pairwise
        # distance; nugget 1e-3; K built on the device in FP64, stored FP32
        X = torch.from_numpy(matgen.mnist_like_points(n, 784, 4 + rank)).to(dev)
        ell = matgen.median_pairwise_distance(X)
        _, A = AG.rbf_build(X, ell, 1e-3, fp64=False)
        del X
        B = matgen.rhs(n, args.rhs, 5 + rank, device=dev)
        desc = {"workload": (f"rbf n={n} d=784 zeros=0.8 l=median({ell:.4f}) nugget=1e-3 "
                             f"rhs={args.rhs} block={args.block} ladder={args.ladder} "
                             f"eps'={args.eps_prime:g} eps_c={args.eps_coherence:g}"),
                "n": n, "d": 784, "lengthscale": round(ell, 6), "nugget": 1e-3}
        data = "synthetic (seeded sparse points in [0,1]^784 standing in for image data; RBF kernel)"
    else:
        A = matgen.spd_matrix(n, args.kappa, 3 + rank, device=dev)
        B = matgen.rhs(n, args.rhs, 100 + rank, device=dev)
        B = B.reshape(n, -1)
        desc = {"workload": (f"spd n={n} kappa={args.kappa:g} rhs={args.rhs} block={args.block} "
                             f"ladder={args.ladder} eps'={args.eps_prime:g}"),
                "n": n, "kappa": args.kappa}
        data = "synthetic (seeded Q diag(sigma) Q^T, geometric spectrum)"
    B = B.reshape(n, -1).contiguous()
    desc.update({"rhs": args.rhs, "block": args.block, "tol": args.tol,
                 "l2": "inputs larger than L2 (A = %d MiB)" % (n * n * 4 // (1 << 20))})
    return A, B, desc, data


def run_gpu(args, world, rank, local):
    import torch
    import cholesky_gpu_b200 as mp
    from cholesky_gpu_b200 import _lib

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
    A, B, desc, data = workload_inputs(args, rank, dev)
    stream = torch.cuda.current_stream(dev)
    ladder = [x.strip() for x in args.ladder.split(",") if x.strip()]
    mixed_opts = dict(block_size=b, precision=args.precision, eps_prime=args.eps_prime,
                      eps_coherence=args.eps_coherence, ladder=ladder)
    # factor objects are created outside the timed region (allocation is setup)
    fobj = {"mixed": mp.Factor(n, **mixed_opts),
            "fp32": mp.Factor(n, block_size=b, precision="fp32")}

    def step(name, f=None):
        f = f or fobj[name]
        f.compute(A)
        return f.pcg(A, B, rel_tol=args.tol, max_it=args.max_it, check_every=args.check_every)

    if args.factor_only > 0:
        for _ in range(args.factor_only):
            fobj["mixed"].compute(A)
        torch.cuda.synchronize()
        return None

    def timed(name, k):
        times, reps = [], []
        for _ in range(k):
            if pg:
                pg.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, rep = step(name)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            reps.append(rep)
        return times, reps

    for _ in range(args.warmup):
        step("mixed")
        step("fp32")
    launches0 = lib.mpchol_kernel_launches()
    with ClockSampler(local, pci_bus_id(torch, local)) as clk:
        t_mx, r_mx = timed("mixed", args.steps)
        launches_mx = lib.mpchol_kernel_launches() - launches0
        t_32, r_32 = timed("fp32", args.steps)
    info_mx = fobj["mixed"].info()

    def mx(v):
        if pg:
            t = torch.tensor([v], dtype=torch.float64, device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            return t.item()
        return v

    ms_mx = mx(statistics.median(t_mx))
    ms_32 = mx(statistics.median(t_32))

    # end to end through the public API with host buffers: Factor.solve_host
    # (mpchol_solve_host) copies A's lower triangle (block columns from the
    # diagonal down, overlapped with the factorization) and B to the device,
    # factors, runs PCG and copies X back -- for both arms
    A_host = A.cpu().pin_memory()
    B_host = B.cpu().pin_memory()
    e2e = {}
    for name in ("mixed", "fp32"):
        ts = []
        for i in range(max(2, min(args.steps, 4)) + 1):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, rep_h = fobj[name].solve_host(A_host, B_host, rel_tol=args.tol, max_it=args.max_it,
                                             check_every=args.check_every)
            e1.record(stream)
            torch.cuda.synchronize()
            if i > 0:
                ts.append(e0.elapsed_time(e1))
            if not rep_h.converged:
                raise RuntimeError(f"{name} host-buffer solve did not converge: {rep_h}")
        e2e[name] = mx(statistics.median(ts))
    e2e_h2d = sum((n - c) * min(b, n - c) for c in range(0, n, b)) * 4 + B_host.numel() * 8

    # per-phase breakdown of one profiled mixed step (events inside the library)
    phases, calls = profiled_phases(lib, lambda: step("mixed"))
    roof = roofline(args, lib, fobj["mixed"].info(), phases, calls, n, b)

    # forced-format arms: time to solution (or the failure) when every step
    # takes one format, with and without larger rounding-error shifts
    arms = {}
    for name, opts in forced_arms(args):
        f = mp.Factor(n, block_size=b, **opts)
        arms[name] = forced_arm(f, lambda f=f: step(None, f), stream)

    steps_used = {nm: info_mx.steps_by_prec[i] for i, nm in PREC_KEYS if info_mx.steps_by_prec[i]}
    result = {
        "metric": METRIC,
        "value": round(ms_mx, 3),
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_mx, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "%s factor, fp64 pcg" % "/".join(steps_used),
        "data": data,
        "config": dict(desc, parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "comparator_fp32_factor_ms": round(ms_32, 3),
        "speedup_vs_fp32_factor": round(ms_32 / ms_mx, 3),
        "e2e": {"value": round(e2e["mixed"], 3), "unit": "ms",
                "h2d_bytes_per_step": int(e2e_h2d), "d2h_bytes_per_step": int(B.numel() * 8)},
        "e2e_comparator_fp32_factor_ms": round(e2e["fp32"], 3),
        "e2e_speedup_vs_fp32_factor": round(e2e["fp32"] / e2e["mixed"], 3),
        "iterations": {"mixed": r_mx[-1].iterations, "fp32": r_32[-1].iterations},
        "rel_residual": {"mixed": r_mx[-1].rel_residual, "fp32": r_32[-1].rel_residual},
        "backward_error": {"mixed": r_mx[-1].backward_error, "fp32": r_32[-1].backward_error},
        "converged": {"mixed": r_mx[-1].converged, "fp32": r_32[-1].converged},
        "step_precisions": steps_used,
        "step_sequence": "".join(PREC_LETTER.get(p, "?") for p in info_mx.step_prec[:-1]),
        "forced_arms": arms,
        "phase_ms_mixed_step": phases,
        "phase_calls_mixed_step": calls,
        "gpu_launches": int(launches_mx),
        "roofline": roof,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        A64 = A_host.numpy()
        result["cpu_baseline"] = cpu_baseline(args, A64, B_host.numpy(), r_32[-1].iterations)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return result if rank == 0 else None


def forced_arms(args):
    """Fixed-format factors timed beside the switching arm.  FP8 everywhere
    (E4M3 and MXFP8, with the default rounding-error shifts and with four
    times larger ones) shows what the switching rule avoids; FP16X2 and FP16
    everywhere bracket it from the precise side."""
    out = [("fp16x2", dict(precision="fp16x2")), ("fp16", dict(precision="fp16"))]
    for p in ("mxfp8", "e4m3"):
        out.append((p, dict(precision=p)))
        out.append((p + "_pert4", dict(precision=p, pert=4.0)))
    # the switching arm's rule with an FP6 or FP4 MX format in the MXFP8 slot
    for low in ("mxfp6e2m3", "mxfp4"):
        out.append(("switching_" + low, dict(precision="switching", eps_prime=args.eps_prime,
                                             eps_coherence=args.eps_coherence,
                                             ladder=[low] + args.ladder.split(",")[1:])))
    return out


def forced_arm(f, solve, stream, k=3):
    """Time (median of k after two warm-ups: the second call captures the
    factorization's graph) and outcome of one forced arm; a factor or solve
    that fails is recorded with its status."""
    import torch
    from cholesky_gpu_b200 import MpcholError
    try:
        solve()
        solve()
        times, rep = [], None
        for _ in range(k):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, rep = solve()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        info = f.info()
        return {"ms": round(statistics.median(times), 3), "iterations": rep.iterations,
                "converged": rep.converged, "rel_residual": rep.rel_residual,
                "n_perturbed": info.n_perturbed}
    except MpcholError as e:
        info = f.info()
        return {"status": _status_name(e.status), "fail_row": info.fail_row,
                "n_perturbed": info.n_perturbed}


def _status_name(st):
    from cholesky_gpu_b200 import _lib
    return _lib.load().mpchol_status_str(st).decode()


def profiled_phases(lib, fn):
    """Per-phase device time and call count of one call of fn (CUDA events the
    library records on the launching streams)."""
    import torch
    from cholesky_gpu_b200 import _lib
    lib.mpchol_profile_enable(1)
    p0 = _lib.Profile()
    lib.mpchol_profile_read(p0, 1)
    fn()
    torch.cuda.synchronize()
    p = _lib.Profile()
    lib.mpchol_profile_read(p, 1)
    lib.mpchol_profile_enable(0)
    phases = {nm: round(p.ms[i], 4) for i, nm in enumerate(_lib.PHASE_NAMES) if p.calls[i]}
    calls = {nm: int(p.calls[i]) for i, nm in enumerate(_lib.PHASE_NAMES) if p.calls[i]}
    return phases, calls


def roofline(args, lib, info, phases, calls, n, b):
    """Rooflines of the bandwidth- and tensor-bound phases of the profiled
    step; the headline is the phase with the largest device time."""
    from cholesky_gpu_b200 import _lib
    hbm, bf16, peak_kind = measured_peaks()
    nr = 1 if args.rhs <= 1 else (2 if args.rhs <= 2 else (4 if args.rhs <= 4 else 8))
    tc_flops, tc_bytes, tc_exec, tc_fmts = 0.0, 0.0, 0, {}
    panel_bytes = {_lib.PREC_FP16: 2, _lib.PREC_E4M3: 1, _lib.PREC_E5M2: 1, _lib.PREC_MXFP8: 1,
                   _lib.PREC_FP16X2: 4}
    for k, pr in enumerate(info.step_prec):
        s0 = k * b
        bs = min(b, n - s0)
        m = n - s0 - bs
        if m <= 0:
            break
        if pr != _lib.PREC_FP32:
            tc_flops += float(m) * (m + 1) * bs       # lower triangle, algorithmic
            # C lower triangle read + written in FP32, the quantized panel read
            # once (plus its E8M0 scales for MXFP8)
            tc_bytes += (float(m) * (m + 1) / 2 * 8 + float(m) * bs * panel_bytes.get(pr, 1)
                         + (float(m) * bs / 32 if pr == _lib.PREC_MXFP8 else 0.0))
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

    tri = n * (n + 1) / 2 * 4 + 3 * n * 8 * nr
    add("trsv", "hbm", "GB/s", hbm, tri, calls.get("trsv", 0),
        f"one triangular solve: lower triangle of L in FP32 + FP64 vectors ({nr} rhs)")
    add("symv", "hbm", "GB/s", hbm, n * (n + 1) / 2 * 4 + 2 * n * 8 * nr, calls.get("symv", 0),
        f"A X from the lower triangle of A in FP32, FP64 vectors ({nr} rhs)")
    if tc_exec:
        # At b = 256 the trailing update moves 8 bytes of C per 2b flops (x3
        # for FP16X2): below the B200 ridge point, so HBM is the binding roof;
        # the useful tensor rate is reported beside it against the dense FP8
        # peak (2 x the measured bf16 rate) when FP8 steps dominate
        fp8 = sum(v for k_, v in tc_fmts.items() if k_ in (_lib.PREC_E4M3, _lib.PREC_E5M2,
                                                             _lib.PREC_MXFP8))
        tpeak = 2 * bf16 if fp8 * 2 > tc_exec else bf16
        add("syrk_tc", "hbm", "GB/s", hbm, tc_bytes / tc_exec, tc_exec,
            "trailing update: C lower triangle read+write (FP32) + quantized panel per "
            "executing step; tensor_tflops = m(m+1)b useful flops / time")
        if "syrk_tc" in by_phase:
            tt = tc_flops / (phases["syrk_tc"] * 1e-3) / 1e12
            by_phase["syrk_tc"]["tensor_tflops"] = round(tt, 1)
            by_phase["syrk_tc"]["tensor_frac"] = round(tt / tpeak, 4)
            by_phase["syrk_tc"]["tensor_peak"] = tpeak
    dom = max(by_phase, key=lambda k_: by_phase[k_]["ms"]) if by_phase else None
    if dom:
        r = by_phase[dom]
        return {"kernel": dom, "bound": r["bound"], "achieved": r["achieved"], "peak": r["peak"],
                "peak_kind": peak_kind, "unit": r["unit"], "frac": r["frac"],
                "algorithmic_per_launch": r["work_per_launch"],
                "traffic": profiled_traffic(dom, n), "by_phase": by_phase}
    return {"kernel": None, "bound": "hbm", "achieved": None, "peak": hbm,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": None, "traffic": None}


# ---------------------------------------------------------------- CPU side
def cpu_pcg(A32: np.ndarray, L32: np.ndarray, B: np.ndarray, tol: float, max_it: int):
    """FP64 PCG (the reference's loop, src/mixed_cholesky.cu:143-217, stopped
    on the true residual) on the host: operator A (FP32 values), M = L L^T with
    the FP32 factor, x0 = M^-1 b.  Returns (iterations, max relative
    residual)."""
    from scipy.linalg import solve_triangular
    A64 = A32.astype(np.float64)
    L64 = np.tril(L32).astype(np.float64)

    def prec(r):
        y = solve_triangular(L64, r, lower=True, check_finite=False)
        return solve_triangular(L64, y, lower=True, trans="T", check_finite=False)

    B = np.asarray(B, dtype=np.float64).reshape(A32.shape[0], -1)
    nb = np.linalg.norm(B, axis=0)
    x = prec(B)
    r = B - A64 @ x
    it = 0
    if np.any(np.linalg.norm(r, axis=0) > tol * nb):
        z = prec(r)
        p = z.copy()
        rho = np.sum(r * z, axis=0)
        while it < max_it:
            Ap = A64 @ p
            alpha = rho / np.sum(p * Ap, axis=0)
            x += alpha * p
            r -= alpha * Ap
            it += 1
            if np.all(np.linalg.norm(r, axis=0) <= tol * nb):
                r = B - A64 @ x                   # confirm on the true residual
                if np.all(np.linalg.norm(r, axis=0) <= tol * nb):
                    break
            z = prec(r)
            rho_new = np.sum(r * z, axis=0)
            p = z + (rho_new / rho) * p
            rho = rho_new
    r = B - A64 @ x
    return it, float(np.max(np.linalg.norm(r, axis=0) / nb))


def cpu_baseline(args, A: np.ndarray, B: np.ndarray, iters: int):
    """The reference's CPU path on a bounded sample (about 10-30 s of CPU
    work): its micro_cholesky (src/micro_chol.hpp:14-44; FP32, unblocked, one
    thread, built from the reference sources into oracle/_ref) on the leading
    n_s x n_s block, scaled by (n/n_s)^3 -- a sample above the host caches, so
    the scaling is close to measured full-size runs (the reference arm,
    `--impl reference`, runs it at full n) -- plus the measured cost of one
    FP64 PCG iteration at full n on the host (FP32 operator and factor, FP64
    vectors, every rhs) times the FP32 arm's iteration count + 1.  Beside it,
    the OpenMP blocked restatement of the same factorization on all host
    cores, sampled and scaled the same way."""
    from oracle import oracle as O
    import ctypes

    n = A.shape[0]
    kind = "reference" if O.REF_MICRO.exists() else "port"
    ns = min(n, 4096)
    sub = np.array(A[:ns, :ns], dtype=np.float32, order="F")
    t0 = time.perf_counter()
    _, rc = O.ref_micro_cholesky(sub) if kind == "reference" else O.micro_cholesky(sub)
    t_sub = time.perf_counter() - t0
    t_factor = t_sub * (n / ns) ** 3
    t0 = time.perf_counter()
    _, rc2 = O.chol_fp32_omp(sub, 256)
    t_omp = time.perf_counter() - t0
    cores = O.num_threads()
    # one PCG iteration at full n for one rhs: GEMV + two triangular solves
    F = np.asfortranarray(A.astype(np.float32))
    lib = O.lib()
    x = np.ascontiguousarray(B.reshape(n, -1)[:, 0], dtype=np.float64)
    y = np.zeros(n)
    dp = ctypes.POINTER(ctypes.c_double)
    fp = ctypes.POINTER(ctypes.c_float)
    t0 = time.perf_counter()
    lib.orc_gemv_f32_f64(F.ctypes.data_as(fp), n, n, x.ctypes.data_as(dp), y.ctypes.data_as(dp))
    lib.orc_potrs_f32_f64(F.ctypes.data_as(fp), n, n, x.ctypes.data_as(dp), y.ctypes.data_as(dp))
    t_it = (time.perf_counter() - t0) * args.rhs
    total_ms = (t_factor + (iters + 1) * t_it) * 1e3
    omp_ms = (t_omp * (n / ns) ** 3 + (iters + 1) * t_it) * 1e3
    return {"value": round(total_ms, 1), "unit": "ms", "cores": 1, "kind": kind,
            "sample": (f"micro_cholesky on the leading {ns}x{ns} block ({t_sub:.2f} s, rc {rc}) "
                       f"scaled by (n/{ns})^3 to n={n}, plus {iters + 1} x one measured FP64 PCG "
                       f"iteration at full n for {args.rhs} rhs ({t_it * 1e3:.0f} ms)"),
            "omp_port": {"value": round(omp_ms, 1), "unit": "ms", "cores": cores, "kind": "port",
                         "sample": (f"OpenMP blocked FP32 restatement (block 256) on the same "
                                    f"{ns}x{ns} block ({t_omp:.2f} s on {cores} threads, rc "
                                    f"{rc2}) scaled by (n/{ns})^3, plus the same PCG cost")}}


def run_reference(args, world, rank):
    """The reference's own CPU path at the full workload: micro_cholesky
    (src/micro_chol.hpp:14-44, built from the reference sources into
    oracle/_ref; one thread, as written) factors the full FP32 matrix, then
    FP64 PCG with that factor runs to the tolerance on the host.  One full
    solve takes minutes, so the arm runs one step (no warm-up) whatever
    --steps asks and says so; the value is that step's measured time."""
    if rank != 0:
        return None
    import torch
    from oracle import oracle as O
    from cholesky_gpu_b200 import matgen
    n = args.n
    t_gen = time.perf_counter()
    if args.workload == "rbf":
        X = torch.from_numpy(matgen.mnist_like_points(n, 784, 4))
        ell = matgen.median_pairwise_distance(X)
        A = matgen.rbf_matrix(X, ell, 1e-3).numpy()
        del X
        B = matgen.rhs(n, args.rhs, 5).numpy().reshape(n, -1)
        workload = (f"rbf n={n} d=784 zeros=0.8 l=median({ell:.4f}) nugget=1e-3 rhs={args.rhs} "
                    f"(host micro_cholesky + FP64 PCG)")
        data = "synthetic (seeded sparse points in [0,1]^784 standing in for image data; RBF kernel)"
    else:
        A = matgen.spd_matrix(n, args.kappa, 3).numpy()
        B = matgen.rhs(n, args.rhs, 100).numpy().reshape(n, -1)
        workload = f"spd n={n} kappa={args.kappa:g} rhs={args.rhs} (host micro_cholesky + FP64 PCG)"
        data = "synthetic (seeded Q diag(sigma) Q^T, geometric spectrum)"
    t_gen = time.perf_counter() - t_gen
    kind = "reference" if O.REF_MICRO.exists() else "port"
    t0 = time.perf_counter()
    L, rc = O.ref_micro_cholesky(A) if kind == "reference" else O.micro_cholesky(A)
    t_fac = time.perf_counter() - t0
    t0 = time.perf_counter()
    its, rel = cpu_pcg(A, L, B, args.tol, args.max_it) if rc == 0 else (0, float("nan"))
    t_pcg = time.perf_counter() - t0
    v = (t_fac + t_pcg) * 1e3
    cb = {"value": round(v, 1), "unit": "ms", "cores": 1, "kind": kind,
          "sample": (f"the full workload, one step: micro_cholesky at n={n} ({t_fac:.1f} s, rc {rc}) "
                     f"+ host FP64 PCG to {args.tol:g} ({its} iterations, {t_pcg:.1f} s, "
                     f"rel residual {rel:.1e})")}
    return {
        "impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms",
        "n_gpus": world, "steps": 1, "warmup": 0, "steps_requested": args.steps,
        "warmup_requested": args.warmup,
        "note": ("one full-size step: the reference's single-threaded micro_cholesky takes "
                 "minutes at this n, so the arm measures one solve instead of extrapolating"),
        "ms_per_step": round(v, 1), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32 factor, fp64 pcg", "data": data,
        "config": {"workload": workload, "n": n, "rhs": args.rhs, "tol": args.tol,
                   "input_generation_s": round(t_gen, 1)},
        "iterations": its, "rel_residual": rel, "converged": bool(rel <= args.tol),
        "cpu_baseline": cb,
        "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
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


def run_rbf_grad(args, world, rank, local):
    """Differentiation workload: RBF kernel, n = 8192 points x ~ N(0, I_64),
    l = 4, nugget 1e-2, y ~ N(0,1); one step = forward solve + backward
    (adjoint PCG reusing the factor, fused gradient contraction)."""
    import torch
    from cholesky_gpu_b200 import autograd as AG, matgen
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
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
    (seeded), 4 rhs each; one step = batched factor + lockstep PCG of all,
    run by the plan the autotuner's table gives for this batch shape
    (cholesky_gpu_b200/tuned_batch.json; --tune re-measures it on this GPU
    and rewrites the table)."""
    import torch
    from cholesky_gpu_b200 import matgen, tune
    from cholesky_gpu_b200.shard import gather_by_system, max_over_ranks, partition_systems
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    count, nrhs = 512, 4
    # the same 512 systems for every world size; each rank owns a shard (no
    # data-path collective: systems are independent)
    ns_all = [int(v) for v in matgen.batch_sizes(count, 64, 2048, 8)]
    ks = matgen.batch_kappas(count, 1e2, 1e6, 9)
    tuned = None
    if args.tune and rank == 0:
        tuned = tune.tune(ns_all, nrhs=nrhs, table=tune.load_table(),
                          log=lambda m: print(m, file=sys.stderr, flush=True))
        tune.save_table(tuned, args.tune_out)
    table = tuned if tuned is not None else tune.load_table()
    plan = tune.plan_for(ns_all, nrhs, table)
    if args.precision != "switching":    # an explicit format overrides the table
        plan = {"mode": "whole", "config": {"block_size": 128, "precision": args.precision}}
    mine = partition_systems(ns_all, world)[rank]
    ns = [ns_all[i] for i in mine]
    As = [matgen.spd_matrix(ns_all[i], float(ks[i]), i, device=dev) for i in mine]
    Bs = [matgen.rhs(ns_all[i], nrhs, 7000 + i, device=dev) for i in mine]
    stream = torch.cuda.current_stream(dev)
    bt = tune.TunedBatch(ns, nrhs=nrhs, plan=plan)

    def step():
        if dist is not None:
            dist.barrier()
        bt.factor(As)
        return bt.pcg(As, Bs, rel_tol=args.tol, max_it=args.max_it, check_every=args.check_every)
    with ClockSampler(local, pci_bus_id(torch, local)) as clk:
        ms, (Xs, reps, st) = _timed(step, args.steps, args.warmup, stream)
    ms = max_over_ranks(ms, dist)
    # end to end: the systems and rhs in page-locked host memory, copied in,
    # factored and solved, the solutions copied back, every step
    Ah = [a.cpu().pin_memory() for a in As]
    Bh = [b.cpu().pin_memory() for b in Bs]
    Xh = [torch.empty(b.shape, dtype=torch.float64).pin_memory() for b in Bs]

    def step_e2e():
        for a, ah in zip(As, Ah):
            a.copy_(ah, non_blocking=True)
        for b, bh in zip(Bs, Bh):
            b.copy_(bh, non_blocking=True)
        X, R, S = step()
        for xh, x in zip(Xh, X):
            xh.copy_(x, non_blocking=True)
        return X, R, S
    ms_e2e, _ = _timed(step_e2e, max(2, min(args.steps, 4)), 1, stream)
    ms_e2e = max_over_ranks(ms_e2e, dist)
    h2d = sum(n * n * 4 + n * nrhs * 8 for n in ns)
    allrep = gather_by_system({i: (r.iterations, r.converged) for i, r in zip(mine, reps)},
                              count, dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None
    its = [r[0] for r in allrep]
    flops = sum(n ** 3 / 3.0 for n in ns_all)
    # roofline of the whole step against HBM: algorithmic bytes of every
    # system's factor (each step's trailing lower triangle read and written
    # in FP32, the panel read) and of its solves (the initial residual and
    # x0 = M^-1 b, then per iteration one operator product and two triangular
    # solves, each a pass over an FP32 lower triangle); small systems keep
    # the batch latency-bound, which the fraction shows
    hbm, _, peak_kind = measured_peaks()
    bsz = plan["config"]["block_size"] if plan["mode"] == "whole" else 128
    alg = 0.0
    for n, it in zip(ns_all, its):
        for k in range(0, n, bsz):
            m = n - k - min(bsz, n - k)
            alg += m * (m + 1) / 2 * 8 + m * min(bsz, n - k) * 4
        alg += (it + 2) * 3 * n * (n + 1) / 2 * 4
    achieved = alg / (ms * 1e-3) / 1e9
    out = _base(args, world, ms, "ms", "tuned batch factor, fp64 pcg",
                "synthetic (seeded Q diag(sigma) Q^T per system)",
                {"workload": f"batch 512 systems n~U[64,2048] kappa~logU[1e2,1e6] rhs=4",
                 "systems": count, "rhs": nrhs, "tol": args.tol, "plan": plan,
                 "parallelism": f"systems sharded over {world} GPUs" if world > 1 else "single GPU"},
                {"scaling": "strong",
                 "solves_per_s": round(count / (ms * 1e-3), 1),
                 "ms_per_system": round(ms / count, 4),
                 "all_converged": all(r[1] for r in allrep),
                 "iterations": {"max": max(its), "median": statistics.median(its)},
                 "factor_tflops_equiv": round(flops / (ms * 1e-3) / 1e12, 2),
                 "e2e": {"value": round(ms_e2e, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
                         "d2h_bytes_per_step": int(sum(n * nrhs * 8 for n in ns))},
                 "roofline": {"kernel": "whole step (factor + PCG of all systems)", "bound": "hbm",
                              "achieved": round(achieved, 1), "peak": hbm, "peak_kind": peak_kind,
                              "unit": "GB/s", "frac": round(achieved / hbm, 4),
                              "algorithmic_per_step": alg, "traffic": None},
                 "clocks": clk.summary()})
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = batch_cpu_baseline(args, As, Bs, ns_all)
    return out


def batch_cpu_baseline(args, As, Bs, ns_all, budget_s: float = 15.0):
    """The reference's CPU path (micro_cholesky + host FP64 PCG, one thread)
    on a seeded sample of the batch's systems until about budget_s of work,
    scaled to all 512 by the sample's share of sum n^3."""
    from oracle import oracle as O
    kind = "reference" if O.REF_MICRO.exists() else "port"
    order = np.random.default_rng(1).permutation(len(As))
    t_tot, done, cube = 0.0, 0, 0.0
    for i in order:
        A = As[i].cpu().numpy()
        B = Bs[i].cpu().numpy()
        t0 = time.perf_counter()
        L, rc = O.ref_micro_cholesky(A) if kind == "reference" else O.micro_cholesky(A)
        if rc == 0:
            cpu_pcg(A, L, B, args.tol, args.max_it)
        t_tot += time.perf_counter() - t0
        done += 1
        cube += float(A.shape[0]) ** 3
        if t_tot > budget_s:
            break
    total = sum(float(n) ** 3 for n in ns_all)
    v = t_tot * total / cube * 1e3
    return {"value": round(v, 1), "unit": "ms", "cores": 1, "kind": kind,
            "sample": (f"micro_cholesky + host FP64 PCG on {done} of the 512 systems "
                       f"({t_tot:.1f} s), scaled by sum n^3")}


def run_syrk(args, world, rank, local):
    """Trailing-update microbenchmark on the RBF workload's shapes (n = 16384):
    C (m x m FP32, lower 128-tiles) -= P P^T with m = n - b (the first step)
    and m = n / 2, for panel widths k = b in {256, 512, 1024}, through
    mpchol_syrk_update in each tensor-core format, beside the reference's
    sm_100 path for the same product -- cuBLASLt block-scaled MXFP8 (E4M3 with
    one E8M0 scale per 32 along K, the reference's LtMxfp8Matmul) reached
    through torch's scaled_mm -- and cuBLAS bf16.  The library GEMMs compute
    the full m x m product into a new FP32 matrix (2 m^2 k flops, no C read);
    the SYRK updates the lower triangle of C in place (m (m+1) k useful
    flops, C read and written).  Codes are random valid values: the timing
    does not depend on them."""
    import torch
    import torch.nn.functional as F
    from cholesky_gpu_b200 import _lib
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)
    hbm, bf16, peak_kind = measured_peaks()
    n = 16384
    g = torch.Generator(device=dev)
    g.manual_seed(1)

    def ev_time(fn, reps=5):
        for _ in range(2):
            fn()
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    def codes8(m, k):
        c = torch.randint(0, 0x7E, (m, k), dtype=torch.uint8, device=dev, generator=g)
        sign = torch.randint(0, 2, (m, k), dtype=torch.uint8, device=dev, generator=g) << 7
        return c | sign

    rows = []
    for k in (256, 512, 1024):
        for m in (n - k, n // 2):
            C = torch.zeros((m, m), dtype=torch.float32, device=dev)
            ent = {"m": m, "k": k}
            for fname, fmt in (("e4m3", _lib.PREC_E4M3), ("mxfp8", _lib.PREC_MXFP8),
                               ("fp16", _lib.PREC_FP16), ("fp16x2", _lib.PREC_FP16X2)):
                if fmt in (_lib.PREC_FP16, _lib.PREC_FP16X2):
                    Q = (torch.randn((2 * m if fmt == _lib.PREC_FP16X2 else m, k), device=dev,
                                     generator=g) * 0.1).half().view(torch.int16)
                else:
                    Q = codes8(m, k)
                S = (torch.full((m, k // 32), 127, dtype=torch.uint8, device=dev)
                     if fmt == _lib.PREC_MXFP8 else torch.zeros(m, dtype=torch.int8, device=dev))
                st = lib.mpchol_syrk_update(C.data_ptr(), m, m, k, fmt, Q.data_ptr(), S.data_ptr(),
                                            None, 0, stream.cuda_stream)
                if st != 0:
                    ent[fname] = {"status": st}
                    continue
                ms = ev_time(lambda: lib.mpchol_syrk_update(C.data_ptr(), m, m, k, fmt, Q.data_ptr(),
                                                            S.data_ptr(), None, 0,
                                                            stream.cuda_stream))
                fl = float(m) * (m + 1) * k
                byt = float(m) * (m + 1) / 2 * 8
                mult = 3 if fmt == _lib.PREC_FP16X2 else 1
                tpk = 2 * bf16 if fmt in (_lib.PREC_E4M3, _lib.PREC_MXFP8) else bf16
                ent[fname] = {"ms": round(ms, 4), "useful_tflops": round(fl / ms / 1e9, 1),
                              "issued_tflops": round(mult * fl / ms / 1e9, 1),
                              "tensor_frac": round(mult * fl / ms / 1e9 / tpk, 4),
                              "hbm_gbs": round(byt / ms / 1e6, 1),
                              "hbm_frac": round(byt / ms / 1e6 / hbm, 4)}
            del C
            # the reference's path: cuBLASLt MXFP8 (block scales 1x32, E8M0), full GEMM
            try:
                a = codes8(m, k).view(torch.float8_e4m3fn)
                bmat = codes8(m, k).view(torch.float8_e4m3fn)
                rows_p = -(-m // 128) * 128
                cols_p = -(-(k // 32) // 4) * 4
                sa = torch.full((rows_p * cols_p,), 1.0, device=dev).to(torch.float8_e8m0fnu)
                sb = torch.full((rows_p * cols_p,), 1.0, device=dev).to(torch.float8_e8m0fnu)

                def lt():
                    return F.scaled_mm(a, bmat.t(), sa, F.ScalingType.BlockWise1x32, sb,
                                       F.ScalingType.BlockWise1x32,
                                       swizzle_a=F.SwizzleType.SWIZZLE_32_4_4,
                                       swizzle_b=F.SwizzleType.SWIZZLE_32_4_4,
                                       output_dtype=torch.float32)
                ms = ev_time(lt)
                ent["cublaslt_mxfp8_gemm"] = {"ms": round(ms, 4),
                                              "tflops": round(2.0 * m * m * k / ms / 1e9, 1),
                                              "tensor_frac": round(2.0 * m * m * k / ms / 1e9 / (2 * bf16), 4)}
            except Exception as e:      # noqa: BLE001 - record why the comparator did not run
                ent["cublaslt_mxfp8_gemm"] = {"error": str(e).splitlines()[0][:200]}
            try:
                ah = torch.randn((m, k), device=dev, generator=g).bfloat16()
                bh = torch.randn((m, k), device=dev, generator=g).bfloat16()
                ms = ev_time(lambda: torch.matmul(ah, bh.t()))
                ent["cublas_bf16_gemm"] = {"ms": round(ms, 4),
                                           "tflops": round(2.0 * m * m * k / ms / 1e9, 1),
                                           "tensor_frac": round(2.0 * m * m * k / ms / 1e9 / bf16, 4)}
            except Exception as e:      # noqa: BLE001
                ent["cublas_bf16_gemm"] = {"error": str(e).splitlines()[0][:200]}
            rows.append(ent)
            torch.cuda.empty_cache()
    return {"metric": "trailing-update time (SYRK vs cuBLASLt MXFP8 GEMM), one B200",
            "unit": "ms", "higher_is_better": False, "n_gpus": world, "data": "synthetic codes",
            "peaks": {"hbm_gbs": hbm, "bf16_tflops": bf16, "fp8_tflops": 2 * bf16, "kind": peak_kind},
            "config": {"workload": "syrk shapes of the rbf n=16384 factorization"}, "shapes": rows}


def main():
    args = parse()
    world, rank, local = dist_init(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    elif args.workload == "rbf-grad":
        out = run_rbf_grad(args, world, rank, local)
    elif args.workload == "batch":
        out = run_batch(args, world, rank, local)
    elif args.workload == "syrk":
        out = run_syrk(args, world, rank, local)
    else:
        out = run_gpu(args, world, rank, local)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
