"""Build the sm_100a shared library libgts_b200.so in-tree with nvcc."""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libgts_b200.so")
CLI = os.path.join(HERE, "gts")
CLI_SRC = os.path.join(HERE, "csrc", "cli.cpp")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) +
                  [p for p in glob.glob(os.path.join(HERE, "csrc", "*.cpp")) if p != CLI_SRC])


def headers():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh")) +
                  glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(CLI):
        return False
    t = min(os.path.getmtime(LIB), os.path.getmtime(CLI))
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [CLI_SRC])


def build_cli() -> str:
    """The GTS command line (drop-in for the reference's bin/GTS)."""
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(HERE, "..", "include"), CLI_SRC,
           "-L", HERE, "-lgts_b200", "-Wl,-rpath,$ORIGIN", "-o", CLI]
    subprocess.run(cmd, check=True)
    return CLI


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = ["nvcc", "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O2",
               "-I", os.path.join(HERE, "..", "include"), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((subprocess.Popen(cmd), src))
        objs.append(obj)
    for p, src in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    cmd = ["nvcc", "-shared", *ARCH, "-o", LIB, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    build_cli()
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
