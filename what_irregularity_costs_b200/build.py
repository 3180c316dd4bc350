"""Build recipe for the CUDA library (libosn_tsdf_b200.so), in-tree.

nvcc compiles every ``csrc/*.cu`` for sm_100a only and links one shared
library with the CUDA runtime linked statically, so the library loads next to
PyTorch's own runtime without a version clash. ``-fmad=false`` keeps every
float operation unfused; the geometry code also spells its rounding out with
intrinsics, so the flag is a second guard, not the only one.

Run ``python -m what_irregularity_costs_b200.build`` or call ``build()``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libosn_tsdf_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "-I", os.path.join(ROOT, "include"), "-I", CSRC,
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, defines=(), obj_dir: str = OBJ,
          lib: str = LIB) -> str:
    """Compile every csrc/*.cu and link the library. defines: extra -D flags
    (tuning macros such as OSN_BAND_MIN_BLOCKS), with their own object folder
    and library path."""
    os.makedirs(obj_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    exe = nvcc()
    jobs = []
    for src in sources():
        obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + ".o")
        if ptxas_info or _stale(obj, [src] + headers):
            cmd = ([exe] + NVCC_FLAGS + [f"-D{d}" for d in defines] + (["-Xptxas", "-v"] if ptxas_info else [])
                   + ["-c", src, "-o", obj])
            jobs.append(cmd)
    objs = [os.path.join(obj_dir, os.path.basename(s)[:-3] + ".o") for s in sources()]

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or ptxas_info or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if jobs or _stale(lib, objs):
        cmd = [exe] + ARCH + ["-shared", "-o", lib] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return lib


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
    print(LIB)
