"""Build libpandora_gpu.so in-tree with nvcc for sm_100a (B200).

Usage: python build.py [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpandora_gpu.so")
BUILD = os.path.join(HERE, "_build")
# the pass launchers of each group of transform lengths compile in their own unit (passes_n*.cu)
PASS_GROUPS = "abcdefghijk"
SOURCES = (["passes_n%s.cu" % g for g in PASS_GROUPS] +
           ["kernels_passes.cu", "kernels_fluid.cu", "kernels_particles.cu", "pandora_capi.cu", "pandora_static.cu"])
HEADERS = ["fft_core.cuh", "pandora_internal.cuh", "bfrot.cuh", "passes_kernels.cuh", "passes_n.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_mtime() -> float:
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(os.path.dirname(HERE), "include", "pandora_gpu.h"))
    return max(os.path.getmtime(f) for f in files)


def _compile(src: str) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    with open(os.path.join(BUILD, os.path.splitext(src)[0] + ".ptxas.txt"), "w") as f:
        f.write(r.stderr)
    return obj, r.stderr


def build(force: bool = False, jobs: int = 0) -> str:
    jobs = jobs or max(1, min(len(SOURCES), os.cpu_count() or 4))
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _deps_mtime():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = [o for o, _ in ex.map(_compile, SOURCES)]
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0, help="parallel compiles (default: the host's cores)")
    a = ap.parse_args()
    print(build(a.force, a.j))
