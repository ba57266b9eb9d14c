"""Build recipe for liblinalg_b200.so (sm_100a only).

    python -m linalglib_b200.build          # incremental
    python -m linalglib_b200.build --force  # rebuild everything

Every CUDA source under csrc/ is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` with -lineinfo, the C++ API sources
(csrc/cxx/*.cpp) by nvcc's host compiler, and both are linked into one shared
library next to this file, so the built .so travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblinalg_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-I", INCLUDE, "-I", CSRC,
          "-Xcompiler", "-fPIC,-fvisibility=hidden", "--expt-relaxed-constexpr",
          "-ccbin", "/usr/bin/g++"]


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "cxx", "*.cpp")))
    return cu, cpp


def _headers():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hs += glob.glob(os.path.join(INCLUDE, "**", "*.h"), recursive=True)
    return hs


def _obj(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(BUILD, rel + ".o")


def _compile(src, force, verbose):
    obj = _obj(src)
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
    else:
        # host C++ (the C++ API); default visibility so namespace linalg is exported
        cmd = ["/usr/bin/g++", "-O3", "-std=c++17", "-fPIC", "-Wall", "-I", INCLUDE, "-I", CSRC,
               "-I", "/usr/local/cuda/include", "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj, None


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile and link; returns the library path.  Raises RuntimeError on failure."""
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = _sources()
    if ptxas_info:
        COMMON.append("-Xptxas=-v")
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), cu + cpp))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("liblinalg_b200 build failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda", "-ccbin", "/usr/bin/g++"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_info))


if __name__ == "__main__":
    main()
