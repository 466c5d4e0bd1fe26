"""Build the sm_100a shared library in-tree.

    python nutcracker-1_b200/nutcracker_b200/build.py [--force]

(run as a script or loaded by path: importing the ``nutcracker_b200``
package requires the library this script produces).

Compiles every ``csrc/*.cu`` with
``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` and links
``lib/libnutcracker_b200.so``, then the command-line program
``programs/nutcracker.cpp`` into ``bin/nutcracker_b200`` (host C++ against the
library, found through an $ORIGIN-relative rpath).  Objects go to
``_build/``.  Rebuilds only what changed (by mtime against the sources and
headers).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib", "libnutcracker_b200.so")
CLI_SRC = os.path.join(PKG, "programs", "nutcracker.cpp")
CLI = os.path.join(PKG, "bin", "nutcracker_b200")
CXX = os.environ.get("CXX", "g++")
BUILD = os.path.join(PKG, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", CSRC, "-I", os.path.join(REPO, "include")]


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    hdr_t = _newest(hdrs)
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t):
            jobs.append([NVCC] + ARCH + FLAGS + ["-c", s, "-o", o])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed: " + " ".join(cmd[-3:]))
            if verbose and (r.stdout or r.stderr):
                sys.stderr.write(r.stdout + r.stderr)
    if jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    if os.path.exists(CLI_SRC) and (force or not os.path.exists(CLI) or
                                    os.path.getmtime(CLI) < max(os.path.getmtime(CLI_SRC), os.path.getmtime(LIB))):
        os.makedirs(os.path.dirname(CLI), exist_ok=True)
        cmd = [CXX, "-std=c++17", "-O2", "-I", os.path.join(REPO, "include"), CLI_SRC,
               "-L", os.path.dirname(LIB), "-lnutcracker_b200", "-Wl,-rpath,$ORIGIN/../lib", "-o", CLI]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("building the command-line program failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
