"""Build libchdwf.so in-tree for sm_100a with nvcc.

    python -m chiralheisenberg_b200.build        # or: python chiralheisenberg_b200/build.py

Each translation unit under csrc/ is compiled to an object in _build/ and
linked into chiralheisenberg_b200/libchdwf.so.  Objects are rebuilt when the
unit or any header under csrc/ or include/ is newer.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libchdwf.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# host code is compiled without fused multiply-add so the REAL*4/REAL*8
# host arithmetic (Gaussians, correlators, Hamiltonian sums) is reproducible
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr",
              "-I", CSRC, "-I", os.path.join(ROOT, "include")]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> list:
    # nvcc drives the host compiler; prefer the system g++ (the one with OpenMP
    # and a complete runtime) when present
    for cand in ("/usr/bin/g++",):
        if os.path.exists(cand):
            return ["-ccbin", cand]
    return []


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max([os.path.getmtime(h) for h in hs] + [0.0])


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hm = _headers_mtime()
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hm):
            continue
        cmd = [nvcc] + _host_cxx() + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
            cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
            cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall",
                   "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
                   "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _wait(procs)
    _wait(procs)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc] + _host_cxx() + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart",
                                                                             "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


def _wait(procs):
    failed = []
    while procs:
        src, p = procs.pop(0)
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, text))
        elif text.strip():
            sys.stderr.write(text)
    if failed:
        for src, text in failed:
            sys.stderr.write(f"--- {src}\n{text}\n")
        raise RuntimeError("nvcc failed for: " + ", ".join(os.path.basename(s) for s, _ in failed))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
