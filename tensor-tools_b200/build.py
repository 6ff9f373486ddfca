"""Build libtt_b200.so in-tree for sm_100a.

CUDA sources (csrc/*.cu) go through nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``; the C++ host layer
(csrc/host/*.cpp, csrc/capi/*.cpp) through g++; objects live in ``_build/``
(not committed) and the shared library in ``lib/`` next to this file.
Rebuilds only what changed (source or header newer than its object).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libtt_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v"] + ARCH
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function",
            "-I/usr/local/cuda/include"]


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp"))) + \
        sorted(glob.glob(os.path.join(CSRC, "capi", "*.cpp")))
    return cu, cpp


def _headers():
    hs = glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return hs


def _obj(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(BUILD, rel + ".o")


def _stale(src, obj, newest_header):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or newest_header > t


def _run(cmd):
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    return p.returncode, p.stdout


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cu, cpp = _sources()
    newest_header = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    jobs = []
    for s in cu:
        o = _obj(s)
        if _stale(s, o, newest_header):
            jobs.append([NVCC] + NVFLAGS + ["-c", s, "-o", o])
    for s in cpp:
        o = _obj(s)
        if _stale(s, o, newest_header):
            jobs.append(["g++"] + CXXFLAGS + ["-c", s, "-o", o])
    logs = []
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for cmd, (rc, out) in zip(jobs, ex.map(_run, jobs)):
            logs.append(" ".join(cmd[-3:]) + "\n" + out)
            if rc != 0:
                raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + out)
    objs = [_obj(s) for s in cu + cpp]
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        rc, out = _run([NVCC, "-shared"] + ARCH + ["-o", LIB] + objs +
                       ["-lcudart", "-Xlinker", "-rpath,/usr/local/cuda/lib64"])
        if rc != 0:
            raise RuntimeError("link failed:\n" + out)
    if verbose:
        for l in logs:
            print(l)
    with open(os.path.join(BUILD, "ptxas.log"), "w") as f:
        f.write("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
