"""Builds libmc3.so (CUDA kernels for sm_100a + C++ host code) and the
MotionCor3 command line in place, next to this file.

Usage: python -m motioncor3_b200.build [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmc3.so")
CLI = os.path.join(HERE, "MotionCor3")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), "nvcc"):
        if shutil.which(c) or os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # Prefer the system compiler; some images point $CXX at a wrapper that
    # lacks runtime spec files.
    for c in ("/usr/bin/g++", "g++"):
        if shutil.which(c) or os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "mc3.h"))
    return hs


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc, cxx = _nvcc(), _cxx()
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
    if not os.path.isdir(cuda_inc):
        cuda_inc = "/usr/local/cuda/include"
    hdrs = _headers()
    cmds = []
    objs = []
    for f in sorted(os.listdir(SRC)):
        src = os.path.join(SRC, f)
        if f == "cli.cpp":
            continue
        if f.endswith(".cu"):
            obj = os.path.join(OBJ, f + ".o")
            cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-ccbin", cxx, "-c", src, "-o", obj]
        elif f.endswith(".cpp"):
            obj = os.path.join(OBJ, f + ".o")
            cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-I", cuda_inc, "-c", src, "-o", obj]
        else:
            continue
        objs.append(obj)
        if force or _stale(obj, [src, *hdrs]):
            cmds.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)

    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        list(ex.map(run, cmds))
    vscript = os.path.join(OBJ, "exports.map")
    with open(vscript, "w") as fh:
        fh.write("{ global: mc3_*; local: *; };\n")
    if force or cmds or _stale(LIB, objs):
        # only the C ABI is exported; the static CUDA runtime stays private
        run([nvcc, *ARCH, "-shared", "-ccbin", cxx, "-o", LIB, *objs, "-lpthread", "-lz",
             "-Xlinker", f"--version-script={vscript}"])
    cli_src = [os.path.join(SRC, "cli.cpp"), os.path.join(SRC, "mrc.cpp")]
    if force or _stale(CLI, [*cli_src, LIB, *hdrs]):
        run([cxx, "-O2", "-std=c++17", "-I", cuda_inc, *cli_src, "-o", CLI, LIB,
             "-Wl,-rpath,$ORIGIN"])
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.jobs, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
