"""Build libsckb200.so in-tree with nvcc for sm_100a (B200).

    python -m spin_colour_kernel_b200.build [--force] [--verbose]

Each csrc/*.cu is compiled to an object in spin_colour_kernel_b200/_build/ and the objects are linked into
spin_colour_kernel_b200/libsckb200.so with the CUDA runtime linked statically, so the library loads beside
PyTorch's own runtime and needs nothing but the driver. Nothing is rebuilt when every object is newer than its
sources and headers.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = PKG / "libsckb200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: set NVCC or put the CUDA toolkit on PATH")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "sck.h", ROOT / "include" / "sck_made.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    cc = nvcc()
    sources = sorted(CSRC.glob("*.cu"))
    headers = _headers()
    jobs = []
    for src in sources:
        obj = OUT / (src.stem + ".o")
        if force or _stale(obj, [src] + headers):
            cmd = [cc, *ARCH, *FLAGS, "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append((src, cmd))

    def run(job):
        src, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r

    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for src, r in ex.map(run, jobs):
            if verbose and r.stderr:
                print(f"--- {src.name}\n{r.stderr}")
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    objs = [OUT / (s.stem + ".o") for s in sources]
    if force or jobs or _stale(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(LIB)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
