"""Build ``libpdlp_b200.so`` (the C-ABI engine) in-tree with nvcc for sm_100a.

    python -m sovereign_moe_b200.build          # or build() from Python
    python -m sovereign_moe_b200.build --bounds-check   # checked engine, for test runs

The library links only the CUDA runtime; there is no torch dependency in the
compiled code.  The output lands next to this file so it travels with the
repository snapshot.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpdlp_b200.so")
SOURCES = ["engine.cu", "kernels.cu", "spmv_plan.cu", "bnr.cu", "crossover.cu"]
HEADERS = ["common.cuh", "engine.cuh", "engine_device.cuh", "engine_passes.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list:
    # nvcc needs a host g++; prefer the system one (some images put another
    # compiler without its runtime specs first on PATH)
    if os.path.exists("/usr/bin/g++"):
        return ["-ccbin", "/usr/bin/g++"]
    return []


STAMP = LIB + ".defines"   # the -D flags the library was built with


def _defines(extra) -> str:
    return " ".join(f for f in (extra or []) if f.startswith("-D"))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    # a library built with extra defines (a checked build) is rebuilt plain
    if os.path.exists(STAMP) and open(STAMP).read().strip():
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(REPO, "include", "pdlp_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra: list | None = None) -> str:
    """Compile the library if any source is newer than it; return its path."""
    if not force and not _stale():
        return LIB
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", *host_compiler(),
           "-I", os.path.join(REPO, "include"), "-I", CSRC,
           "-o", LIB + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES],
           "-lcudart"]
    if extra:
        cmd[1:1] = list(extra)
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{res.stdout}\n{res.stderr}")
    if verbose and (res.stdout or res.stderr):
        print(res.stdout + res.stderr, file=sys.stderr)
    os.replace(LIB + ".tmp", LIB)
    with open(STAMP, "w") as fh:
        fh.write(_defines(extra))
    return LIB


if __name__ == "__main__":
    # --bounds-check: index and row-pointer checks in the engine's tiles
    # (PDLP_ERR_BOUNDS instead of an out-of-range access), for test runs
    extra = []
    if "--ptxas" in sys.argv:
        extra += ["-Xptxas", "-v"]
    if "--bounds-check" in sys.argv:
        extra += ["-DPDLP_BOUNDS_CHECK"]
    print(build(force="--force" in sys.argv or "--bounds-check" in sys.argv, verbose=True,
                extra=extra or None))
