"""Build librpm_b200.so in-tree with nvcc for sm_100a.

Usage: ``python -m rpm_b200.build [-v]``.  The shared library lands in
``rpm_b200/lib/`` so it travels with the source tree; nothing is installed.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
LIBDIR = PACKAGE / "lib"
BUILD = PACKAGE / "_build"
LIBRARY = LIBDIR / "librpm_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-Wall", "-Xcompiler", "-Wno-unused-function"]


def nvcc() -> str:
    for candidate in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and os.path.exists(candidate):
            return candidate
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build librpm_b200")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    """Compile every ``csrc/*.cu`` and link ``lib/librpm_b200.so``; returns its path."""
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list((PACKAGE.parent / "include").glob("*.h"))
    compiler = nvcc()
    objects = []
    jobs = []
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        objects.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [compiler, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
        if verbose or ptxas_info:
            sys.stdout.write(proc.stdout + proc.stderr)
        return proc

    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        list(pool.map(run, jobs))
    if force or jobs or _stale(LIBRARY, objects):
        run([compiler, *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects)])
    return LIBRARY


if __name__ == "__main__":
    args = set(sys.argv[1:])
    print(build(verbose="-v" in args, force="-f" in args, ptxas_info="--ptxas" in args))
