"""Autotuner for batches of uneven SPD systems.

The batched solver (``Batch``, ``mpchol_batch_*``) serves every system of a
batch with one launch per kernel, so a batch runs with one block size and
one trailing-update format.  Which pair is fastest depends on the orders in
the batch: small systems leave most of a 256-wide block empty and want
b = 64 or 128; large ones amortize the panel work over b = 256; the format
trades tensor-core work for PCG iterations.  This module picks that pair by
measurement -- it factors and solves seeded representative batches with every
candidate on the GPU and keeps the fastest one that converges -- and caches
the choice per size class as JSON, so a later batch of the same shape reuses
it without timing anything.

A batch is tuned as a whole (one configuration, one launch sequence) or
split by size class, each class with its own configuration; the tuner times
both and ``TunedBatch`` runs whichever the table records.  There is no
counterpart in the reference, which solves one system per call.
"""
from __future__ import annotations

import json
import math
import statistics
import time
from pathlib import Path

import numpy as np

# Size classes of the orders: inclusive bounds.
SIZE_CLASSES = ((1, 256), (257, 512), (513, 1024), (1025, 2048), (2049, 1 << 30))

# Candidate configurations: block size and trailing-update format (the
# batched solver takes a fixed tensor-core format).
CANDIDATES = (
    {"block_size": 64, "precision": "fp16x2"},
    {"block_size": 128, "precision": "fp16x2"},
    {"block_size": 256, "precision": "fp16x2"},
    {"block_size": 128, "precision": "fp16"},
    {"block_size": 128, "precision": "mxfp8"},
)
DEFAULT = {"block_size": 128, "precision": "fp16x2"}

# The table shipped with the package: tuned on a B200 for the batch workload
# shape (orders U[64, 2048], 4 rhs, kappa log-uniform in [1e2, 1e6]).
TABLE_PATH = Path(__file__).with_name("tuned_batch.json")


def size_class(n: int) -> int:
    """Index of the size class of order n."""
    for i, (lo, hi) in enumerate(SIZE_CLASSES):
        if lo <= n <= hi:
            return i
    raise ValueError(f"order {n} is outside every size class")


def group_by_class(ns) -> dict[int, list[int]]:
    """System indices grouped by size class (indices in caller order)."""
    groups: dict[int, list[int]] = {}
    for i, n in enumerate(ns):
        groups.setdefault(size_class(int(n)), []).append(i)
    return groups


def table_key(ns, nrhs: int) -> str:
    """Cache key of a batch: the size classes it spans and its rhs count."""
    classes = sorted(group_by_class(ns))
    return f"classes={','.join(map(str, classes))};rhs={nrhs}"


def load_table(path: Path | str | None = None) -> dict:
    p = Path(path) if path is not None else TABLE_PATH
    if not p.exists():
        return {}
    return json.loads(p.read_text())


def save_table(table: dict, path: Path | str | None = None) -> Path:
    p = Path(path) if path is not None else TABLE_PATH
    p.write_text(json.dumps(table, indent=1, sort_keys=True) + "\n")
    return p


def config_name(cfg: dict) -> str:
    return f"b{cfg['block_size']}-{cfg['precision']}"


def plan_for(ns, nrhs: int, table: dict | None = None) -> dict:
    """The execution plan for a batch from the table: {"mode": "whole",
    "config": cfg} or {"mode": "split", "classes": {class: cfg}}; the default
    configuration, whole, when the table has no entry for the batch's shape."""
    table = load_table() if table is None else table
    ent = table.get(table_key(ns, nrhs))
    if ent is None:
        return {"mode": "whole", "config": dict(DEFAULT)}
    if ent["mode"] == "split":
        return {"mode": "split", "classes": {int(k): v for k, v in ent["classes"].items()}}
    return {"mode": "whole", "config": ent["config"]}


def pick(results: dict) -> tuple[str, float] | None:
    """The fastest converged entry of {name: {"ms": t, "converged": bool}}
    (ties: the first in insertion order), or None."""
    best = None
    for name, r in results.items():
        if not r.get("converged") or r.get("ms") is None or not math.isfinite(r["ms"]):
            continue
        if best is None or r["ms"] < best[1]:
            best = (name, r["ms"])
    return best


# ---------------------------------------------------------------- GPU side
class TunedBatch:
    """A batch run by the plan the table gives for its shape: one Batch for
    all systems (whole) or one per size class (split), each with its tuned
    block size and format.  Same calls and results as Batch, in caller
    order."""

    def __init__(self, ns, nrhs: int = 1, table: dict | None = None, plan: dict | None = None,
                 **common):
        from .api import Batch
        self.ns = [int(v) for v in ns]
        self.nrhs = nrhs
        self.plan = plan if plan is not None else plan_for(self.ns, nrhs, table)
        if self.plan["mode"] == "whole":
            self.groups = [(list(range(len(self.ns))), self.plan["config"])]
        else:
            g = group_by_class(self.ns)
            self.groups = [(idx, self.plan["classes"].get(c, DEFAULT)) for c, idx in sorted(g.items())]
        self.batches = [Batch([self.ns[i] for i in idx], nrhs=nrhs, **dict(common, **cfg))
                        for idx, cfg in self.groups]

    def factor(self, As) -> "TunedBatch":
        for (idx, _), bt in zip(self.groups, self.batches):
            bt.factor([As[i] for i in idx])
        return self

    def pcg(self, As, Bs, rel_tol: float = 1e-10, max_it: int = 200, check_every: int = 4):
        Xs = [None] * len(self.ns)
        reps = [None] * len(self.ns)
        status = 0
        for (idx, _), bt in zip(self.groups, self.batches):
            X, R, st = bt.pcg([As[i] for i in idx], [Bs[i] for i in idx], rel_tol=rel_tol,
                              max_it=max_it, check_every=check_every)
            status = status or st
            for j, i in enumerate(idx):
                Xs[i], reps[i] = X[j], R[j]
        return Xs, reps, status


def representative(ns, nrhs: int, seed: int, device="cuda", kappa=(1e2, 1e6)):
    """Seeded SPD systems with the given orders (kappa log-uniform in the
    range) and nrhs N(0,1) right-hand sides."""
    from . import matgen
    ks = matgen.batch_kappas(len(ns), kappa[0], kappa[1], seed)
    As = [matgen.spd_matrix(int(n), float(k), seed * 1000 + i, device=device)
          for i, (n, k) in enumerate(zip(ns, ks))]
    Bs = [matgen.rhs(int(n), nrhs, seed * 1000 + 500 + i, device=device) for i, n in enumerate(ns)]
    return As, Bs


def time_plan(ns, As, Bs, nrhs: int, plan: dict, reps: int = 3, tol: float = 1e-10,
              max_it: int = 200) -> dict:
    """Median device time of factor + PCG of the batch under a plan (after
    one warm-up), and whether every system converged."""
    import torch
    from ._lib import MpcholError
    try:
        tb = TunedBatch(ns, nrhs=nrhs, plan=plan)
        stream = torch.cuda.current_stream()
        times, ok = [], True
        for i in range(reps + 1):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            tb.factor(As)
            _, rr, _ = tb.pcg(As, Bs, rel_tol=tol, max_it=max_it)
            e1.record(stream)
            torch.cuda.synchronize()
            if i > 0:
                times.append(e0.elapsed_time(e1))
            ok = ok and all(r.converged for r in rr)
        return {"ms": statistics.median(times), "converged": ok}
    except MpcholError as e:
        return {"ms": None, "converged": False, "status": e.status}


def tune(ns, nrhs: int = 4, candidates=CANDIDATES, reps: int = 3, sample: int | None = 96,
         seed: int = 11, table: dict | None = None, kappa=(1e2, 1e6), tol: float = 1e-10,
         log=None) -> dict:
    """Tune the plan for batches shaped like ns (orders, rhs count) on the
    current GPU and record it in table (a new dict if None), which is
    returned.  A seeded sample of the orders (at most `sample` systems, every
    size class kept in proportion) stands in for the batch.  Candidates:
    every configuration for the whole batch, and the split plan whose every
    class takes its own fastest configuration."""
    table = {} if table is None else table
    rng = np.random.default_rng(seed)
    ns = [int(v) for v in ns]
    if sample is not None and len(ns) > sample:
        ns_s = sorted(rng.choice(ns, size=sample, replace=False).tolist())
    else:
        ns_s = sorted(ns)
    As, Bs = representative(ns_s, nrhs, seed, kappa=kappa)
    t0 = time.perf_counter()
    whole = {}
    for cfg in candidates:
        whole[config_name(cfg)] = time_plan(ns_s, As, Bs, nrhs, {"mode": "whole", "config": cfg},
                                            reps, tol)
        if log:
            log(f"whole {config_name(cfg)}: {whole[config_name(cfg)]}")
    per_class = {}
    groups = group_by_class(ns_s)
    for c, idx in sorted(groups.items()):
        res = {}
        sub_ns = [ns_s[i] for i in idx]
        sub_A = [As[i] for i in idx]
        sub_B = [Bs[i] for i in idx]
        for cfg in candidates:
            res[config_name(cfg)] = time_plan(sub_ns, sub_A, sub_B, nrhs,
                                              {"mode": "whole", "config": cfg}, reps, tol)
        best = pick(res)
        per_class[c] = {"results": res,
                        "config": next(cfg for cfg in candidates if config_name(cfg) == best[0])
                        if best else dict(DEFAULT)}
        if log:
            log(f"class {c} ({len(idx)} systems): best {best}")
    split_plan = {"mode": "split", "classes": {c: v["config"] for c, v in per_class.items()}}
    split = time_plan(ns_s, As, Bs, nrhs, split_plan, reps, tol)
    best_whole = pick(whole)
    entry = {"sample_orders": [min(ns_s), max(ns_s), len(ns_s)], "nrhs": nrhs,
             "whole": whole, "split_ms": split.get("ms"), "split_converged": split["converged"],
             "per_class": {str(c): {"config": v["config"],
                                    "results": v["results"]} for c, v in per_class.items()},
             "tuning_s": round(time.perf_counter() - t0, 1)}
    use_split = split["converged"] and split["ms"] is not None and (
        best_whole is None or split["ms"] < best_whole[1])
    if use_split:
        entry.update(mode="split", classes={str(c): v["config"] for c, v in per_class.items()})
    else:
        name = best_whole[0] if best_whole else config_name(DEFAULT)
        entry.update(mode="whole",
                     config=next((cfg for cfg in candidates if config_name(cfg) == name), DEFAULT))
    table[table_key(ns, nrhs)] = entry
    return table
