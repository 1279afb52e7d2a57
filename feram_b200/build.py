"""Build the in-tree C-ABI library ``feram_b200/libferam_gpu.so`` for sm_100a.

    python feram_b200/build.py            # production build
    python feram_b200/build.py --checked  # bounds-checked build -> libferam_gpu_checked.so

nvcc compiles the CUDA translation unit for ``compute_100a``/``sm_100a``
(no other architectures), g++ compiles the host-side C++ (parser, driver),
and nvcc links the shared library.  Two CUDA translation units: the MD
step (csrc/fg_api.cu) and the warm-start network (csrc/ws_net.cu).  It
cross-compiles without a GPU.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... ({r.returncode})")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return r


def build(checked: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    nvcc = _nvcc()
    out_dir = os.path.join(HERE, "_build", "checked" if checked else "release")
    os.makedirs(out_dir, exist_ok=True)
    defs = ["-DFG_BOUNDS_CHECK=1"] if checked else []
    objs = []
    # fg_api.cu: the MD step; ws_net.cu: the warm-start network (tcgen05)
    for src in ("fg_api.cu", "ws_net.cu"):
        cu_obj = os.path.join(out_dir, src.replace(".cu", ".o"))
        cu_flags = [nvcc, "-c", os.path.join(HERE, "csrc", src), "-o", cu_obj, *ARCH, "-O3", "-lineinfo",
                    "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", *defs]
        if ptxas_v:
            cu_flags += ["-Xptxas", "-v"]
        _run(cu_flags, verbose or ptxas_v)
        objs.append(cu_obj)
    cxx = shutil.which("g++") or "g++"
    for src in ("feram_host.cpp", "feram_driver.cpp"):
        obj = os.path.join(out_dir, src.replace(".cpp", ".o"))
        _run([cxx, "-c", os.path.join(HERE, "host", src), "-o", obj, "-O2", "-std=c++17", "-fPIC",
              "-ffp-contract=off", f"-I{os.path.join(ROOT, 'include')}", "-I/usr/local/cuda/include"], verbose)
        objs.append(obj)
    name = "libferam_gpu_checked.so" if checked else "libferam_gpu.so"
    lib = os.path.join(HERE, name)
    _run([nvcc, "-shared", *ARCH, "-o", lib, *objs, "-lcudart"], verbose)
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--checked", action="store_true", help="bounds-checked kernels")
    ap.add_argument("--all", action="store_true", help="release and checked builds")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/smem usage")
    a = ap.parse_args()
    if a.all:
        print(build(False, a.verbose, a.ptxas))
        print(build(True, a.verbose, False))
    else:
        print(build(a.checked, a.verbose, a.ptxas))


if __name__ == "__main__":
    main()
