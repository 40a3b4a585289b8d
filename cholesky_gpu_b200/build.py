"""Build recipe for the sm_100a shared library ``libmpchol.so`` (in-tree).

The library is plain C-ABI (``include/mpchol.h``): nvcc compiles every
``csrc/*.cu`` for ``sm_100a`` with the CUDA runtime linked statically, so the
``.so`` has no dependency on torch and travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libmpchol.so"
OBJ = PKG / "_build"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    f"-I{ROOT / 'include'}",
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the sm_100a library cannot be built")
    return exe


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, jobs: int | None = None) -> Path:
    """Compile (incrementally) and link libmpchol.so; returns its path."""
    OBJ.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    objs = []
    cmds = []
    for src in sources():
        obj = OBJ / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmds.append([nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])
    procs = []
    maxjobs = jobs or min(8, os.cpu_count() or 1)
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
        while sum(p.poll() is None for p in procs) >= maxjobs:
            procs[0].wait() if procs[0].poll() is None else None
            procs = [p for p in procs if p.poll() is None] + [p for p in procs if p.poll() is not None]
            break
    failed = []
    for p, cmd in zip(procs, cmds):
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((cmd, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"$ {' '.join(c)}\n{o}" for c, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    if force or cmds or _stale(OUT, objs):
        link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                "-cudart", "static", "-o", str(OUT), *map(str, objs)]
        if verbose:
            print(" ".join(link), flush=True)
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(OUT)
