"""Build libinti_b200.so for sm_100a with nvcc, in-tree.

Each CUDA translation unit under csrc/ is compiled to an object in _build/
(in parallel), then linked into _build/libinti_b200.so.  A unit is rebuilt
when it, or any header it can include, is newer than its object.

    python inti.jl_b200/build.py [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "_build"
INCLUDE = HERE.parent / "include"
LIB = OUT / "libinti_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(src: Path, obj: Path, hdr_mtime: float) -> bool:
    if not obj.exists():
        return True
    m = obj.stat().st_mtime
    return src.stat().st_mtime > m or hdr_mtime > m


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    OUT.mkdir(exist_ok=True)
    nvcc = _nvcc()
    hdr_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    for src in sources():
        obj = OUT / (src.stem + ".o")
        if force or _stale(src, obj, hdr_mtime):
            cmd = [nvcc, *ARCH, *FLAGS, *(extra or []), "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
            jobs.append((src, cmd))

    def run(job):
        src, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, cmd, r

    failed = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for src, cmd, r in ex.map(run, jobs):
            if verbose or r.returncode:
                print(" ".join(cmd), file=sys.stderr)
                if r.stdout:
                    print(r.stdout, file=sys.stderr)
                if r.stderr:
                    print(r.stderr, file=sys.stderr)
            if r.returncode:
                failed.append(src.name)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    objs = [OUT / (s.stem + ".o") for s in sources()]
    if force or jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
