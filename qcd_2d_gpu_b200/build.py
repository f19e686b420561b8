"""Build libqcd2d.so in-tree for sm_100a (nvcc, no JIT cache).

    python -m qcd_2d_gpu_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libqcd2d.so")
DRIVER = os.path.join(HERE, "qcd2d")
DRIVER_SRC = [os.path.join(HERE, "driver", f) for f in ("qcd2d_main.c", "refio.c")]

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-shared",
    "-Xcompiler",
    "-fPIC",
]


def sources() -> list[str]:
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh", ".cc"))]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(ROOT, "include", "qcd2d.h")]
    return any(os.path.getmtime(s) > t for s in deps)


UNITS = ["qcd2d.cu", "batch.cu", "pairs.cu", "stats.cc"]


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit for sm_100a in parallel, then link the
    shared library (nvcc -shared)."""
    if not force and not needs_build():
        return LIB
    import concurrent.futures as cf
    import tempfile

    nvcc = os.environ.get("NVCC", "nvcc")
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    with tempfile.TemporaryDirectory(prefix="qcd2d_build_") as tmp:
        objs, cmds = [], []
        for u in UNITS:
            obj = os.path.join(tmp, u + ".o")
            objs.append(obj)
            cmds.append([nvcc] + compile_flags + inc + ["-c", os.path.join(CSRC, u), "-o", obj])
        with cf.ThreadPoolExecutor(max_workers=len(cmds)) as ex:
            futs = []
            for c in cmds:
                if verbose:
                    print(" ".join(c), flush=True)
                futs.append(ex.submit(subprocess.run, c, check=True))
            for f in futs:
                f.result()
        link = [nvcc] + NVCC_FLAGS + ["-o", LIB + ".tmp"] + objs
        if verbose:
            print(" ".join(link), flush=True)
        subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_driver(force: bool = False, verbose: bool = False) -> str:
    """The drop-in program (C), linked against the in-tree libqcd2d.so."""
    build_library(verbose=verbose)
    deps = DRIVER_SRC + [os.path.join(HERE, "driver", "refio.h"), os.path.join(ROOT, "include", "qcd2d.h"), LIB]
    if not force and os.path.exists(DRIVER) and all(os.path.getmtime(d) <= os.path.getmtime(DRIVER) for d in deps):
        return DRIVER
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    cmd = [cc, "-O2", "-std=gnu11", "-Wall", "-I" + os.path.join(ROOT, "include"), "-o", DRIVER + ".tmp"] + DRIVER_SRC + [
        "-L" + HERE, "-lqcd2d", "-Wl,-rpath,$ORIGIN", "-lm"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    build_driver(force="--force" in sys.argv, verbose=True)
    print(LIB)
