"""Build the B200 kernel-suite shared libraries in-tree (``tealeaf_b200/lib``).

Each library is a plain C-ABI ``.so`` (no torch types) compiled for sm_100a:

* ``libtealeaf_b200_2d.so`` -- the 2D suite (reference 2d/kernel_interface.h)
* ``libtealeaf_b200_3d.so`` -- the 3D suite (reference 3d/kernel_interface.h)

Every source is compiled with ``-fmad=false``: each multiply and add of the
FP64 drop-in rounds separately, in the reference's expression order, and the
FP32 kernels of the precision form contract only where they call fma
explicitly (``fma_t`` in refine2d.cuh).
The CUDA runtime is linked statically so the libraries load in any process
(a C host, ctypes) without a matching libcudart on the library path.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
OBJ_DIR = PKG / "_build"
INCLUDE = REPO / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I%s" % INCLUDE, "-I%s" % CSRC]

LIBS = {
    "tealeaf_b200_2d": ["suite2d.cu", "driver2d.cu", "noalloc2d.cu", "mixed2d.cu", "batch2d.cu"],
    "tealeaf_b200_3d": ["suite3d.cu", "driver3d.cu", "adjoint3d.cu"],
}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx():
    # nvcc needs a host compiler with the standard C++ headers; the system g++ has them.
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(map(str, cmd)), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _deps():
    return (list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.h"))
            + list(INCLUDE.glob("*.h")))


def build(verbose: bool = False, force: bool = False):
    """Compile every library; returns the list of .so paths."""
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    cc = ["-ccbin", _host_cxx()]
    jobs = []
    for lib, srcs in LIBS.items():
        for src in srcs:
            obj = OBJ_DIR / (Path(src).stem + ".o")
            if force or _stale(obj, [CSRC / src] + _deps()):
                jobs.append([nvcc()] + cc + ARCH + NVCC_FLAGS + ["-fmad=false", "-c", CSRC / src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    built = []
    for lib, srcs in LIBS.items():
        if not srcs:
            continue
        objs = [OBJ_DIR / (Path(s).stem + ".o") for s in srcs]
        target = LIB_DIR / ("lib%s.so" % lib)
        if force or _stale(target, objs):
            _run([nvcc()] + cc + ARCH + ["-shared", "-cudart", "static", "-o", target] + objs
                 + ["-lpthread", "-ldl", "-lrt"])
        built.append(target)
    return built


if __name__ == "__main__":
    for p in build(verbose="-v" in sys.argv, force="-f" in sys.argv):
        print(p)
