"""Build libpibm.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python -m pureibm_ps2d_fd1d_b200.build

Host set-up code is compiled with -ffp-contract=off so that geometric
quantities match the device kernels' explicitly rounded arithmetic.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libpibm.so")
MAIN = os.path.join(OUT_DIR, "pibm_main")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["kernels.cu", "scalar.cu", "moving.cu", "adjoint.cu", "peak.cu", "api.cu"]
# per-source nvcc flags: the DEM and the moving-geometry rebuild are compiled
# without multiply-add contraction (bit-equal to a serial evaluation)
CU_FLAGS = {"moving.cu": ["--fmad=false"]}
CPP_SOURCES = ["host_setup.cpp"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = _nvcc()
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "pibm.h")]
    if not force and not _stale(LIB, deps):
        build_main()
        return LIB
    jobs = []
    for src in CU_SOURCES:
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        jobs.append((obj, [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                           *CU_FLAGS.get(src, []), "-Xptxas", "-v" if verbose else "-O3", "-c",
                           os.path.join(CSRC, src), "-o", obj]))
    for src in CPP_SOURCES:
        obj = os.path.join(OUT_DIR, src.replace(".cpp", ".o"))
        jobs.append((obj, ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I/usr/local/cuda/include",
                           "-c", os.path.join(CSRC, src), "-o", obj]))
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(subprocess.run, cmd, check=True) for _, cmd in jobs]:
            f.result()
    objs = [obj for obj, _ in jobs]
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    build_main(force=True)
    return LIB


def build_main(force: bool = False) -> str:
    """The C host driver (csrc/pibm_main.c): gcc against include/pibm.h,
    linked to libpibm.so found next to it at run time."""
    src = os.path.join(CSRC, "pibm_main.c")
    if not force and not _stale(MAIN, [src, LIB, os.path.join(HERE, "..", "include", "pibm.h")]):
        return MAIN
    subprocess.run(["gcc", "-O2", "-std=gnu99", "-Wall", "-ffp-contract=off", "-o", MAIN + ".tmp", src,
                    "-L" + OUT_DIR, "-lpibm", "-Wl,-rpath,$ORIGIN", "-lm"], check=True)
    os.replace(MAIN + ".tmp", MAIN)
    return MAIN


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
