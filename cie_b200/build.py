"""Builds the in-tree CUDA library cie_b200/libciecu.so for sm_100a.

    python -m cie_b200.build            # incremental (object files in cie_b200/_build)
    python -m cie_b200.build --verbose  # also prints ptxas register / spill usage

Every .cu / .cpp under cie_b200/csrc is compiled with nvcc for
`-gencode arch=compute_100a,code=sm_100a` only and linked into one shared
library that exports the C-ABI declared in include/ciecu.h.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libciecu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "--expt-relaxed-constexpr"]


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, name))
    return out


def headers():
    hs = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for name in os.listdir(d):
            if name.endswith((".h", ".cuh", ".hpp")):
                hs.append(os.path.join(d, name))
    return hs


def build(verbose=False, force=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    newest_header = max((os.path.getmtime(h) for h in headers()), default=0)
    objects, commands = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objects.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) > os.path.getmtime(src)
                and os.path.getmtime(obj) > newest_header):
            continue
        cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        if verbose and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        commands.append((src, cmd))
    # translation units compile independently: one nvcc per core, at most 8
    jobs = jobs or max(1, min(8, os.cpu_count() or 1))
    running = []
    for src, cmd in commands:
        print("%s ... %s" % (NVCC, os.path.basename(src)), flush=True)
        running.append((src, subprocess.Popen(cmd)))
        while len(running) >= jobs or (running and src == commands[-1][0]):
            src0, proc = running.pop(0)
            if proc.wait() != 0:
                for _, other in running:
                    other.wait()
                raise subprocess.CalledProcessError(proc.returncode, "nvcc " + os.path.basename(src0))
    if (force or not os.path.exists(LIB)
            or max(os.path.getmtime(o) for o in objects) > os.path.getmtime(LIB)):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objects + ["-lcudart", "-lcuda"]
        subprocess.run(cmd, check=True)
        print("linked", LIB, flush=True)
    return LIB


if __name__ == "__main__":
    p = argparse.ArgumentParser()
    p.add_argument("--verbose", action="store_true")
    p.add_argument("--force", action="store_true")
    a = p.parse_args()
    build(verbose=a.verbose, force=a.force)
    sys.exit(0)
