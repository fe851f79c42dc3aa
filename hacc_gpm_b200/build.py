"""Build the PM step's native library in-tree.

Compiles every ``csrc/*.cu`` for sm_100a with nvcc (in parallel) and links
``_lib/libhgpm.so`` (C-ABI declared in ``include/hgpm_c.h``; CUDA runtime
linked statically).  Also builds the C++ drop-in driver ``_lib/haccgpm``
(the reference's ``serial()`` run loop over the C-ABI).  Usage:

    python -m hacc_gpm_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libhgpm.so")
DRIVER = os.path.join(LIBDIR, "haccgpm")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"] + ARCH


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "hgpm_c.h"))
    return hs


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    hdrs = _headers()
    cmds = []
    objs = []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJDIR, s[:-3] + ".o")
        objs.append(obj)
        if force or not _newer(obj, [src] + hdrs):
            cmds.append([nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
        if verbose and (r.stdout or r.stderr):
            sys.stderr.write(r.stdout + r.stderr)
        return r

    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        list(ex.map(run, cmds))
    if force or cmds or not os.path.exists(LIB):
        run([nvcc(), "-shared", *ARCH, "-o", LIB, *objs])
    drv_src = os.path.join(HERE, "host", "haccgpm_driver.cpp")
    shim_src = os.path.join(HERE, "host", "haccgpm_serial.cpp")
    if os.path.exists(drv_src):
        deps = [drv_src, shim_src, LIB, os.path.join(HERE, "host", "haccgpm.hpp"), os.path.join(ROOT, "include", "hgpm_c.h")]
        if force or not _newer(DRIVER, [d for d in deps if os.path.exists(d)]):
            run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "host"),
                 "-I", os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include"),
                 drv_src, shim_src, "-L", LIBDIR, "-lhgpm", "-Wl,-rpath,$ORIGIN", "-o", DRIVER])
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))


if __name__ == "__main__":
    main()
