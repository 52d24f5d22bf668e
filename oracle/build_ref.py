"""Build recipe for the checker binaries (test infrastructure).

The reference TeaLeaf C sources are compiled directly with gcc from where they
lie in the read-only reference tree (the reference's own make system is not
used). Outputs go only to ``oracle/_ref`` (git-ignored, but shipped with the
repository snapshot to the GPU machine, where the reference tree is absent).
``build_oracle()`` compiles this directory's own C restatement
(``tl_oracle.c``) into ``oracle/_build/libtl_oracle.so``.

Products in ``oracle/_ref`` (``D`` = 2d or 3d, ``F`` = flavour):

* ``tealeaf{D}_omp3{F}``  -- the unmodified reference program (its own
                             ``main``) with the reference omp3 kernel suite.
* ``harness{D}_omp3{F}``  -- ``oracle/ref_harness.c`` + reference host/drivers
                             + reference omp3 suite: per-step iteration counts
                             and field summaries.
* ``harness{D}_b200``     -- ``oracle/ref_harness.c`` + reference host/drivers,
                             compiled against the B200 suite's
                             ``chunk_extension.h`` and linked with the B200
                             shared library: the drop-in proof.
* ``layout{D}``           -- prints ``offsetof``/``sizeof`` of the reference
                             ``Chunk``/``Settings``/``State`` structs.
* ``decompose{D}``        -- ``oracle/decompose_probe.c`` + reference host and
                             omp3 objects: the reference's ``decompose_field``
                             for every rank of an N-rank run.
* ``harness{D}_omp3_mpi`` -- the parity harness with the reference host built
                             for several ranks (no ``-DNO_MPI``) over
                             ``oracle/minimpi`` (the MPI calls of ``comms.c``
                             on Unix sockets between processes): the reference's
                             own multi-rank runs, launched by
                             ``oracle.oracle.run_reference_ranks``.
* ``harness{D}_b200_mpi`` -- the same multi-rank host linked with the B200
                             library instead of the omp3 suite.

Compiler flags follow the reference GNU flags (2d/make.flags:10: -O3
-funroll-loops -std=gnu99, plus -fopenmp) with ``-DNO_MPI -DENABLE_PROFILING``.
``-march=native`` is replaced by ``-march=x86-64-v3`` because the binaries are
built here and run on another host. Flavour ``""`` (parity) adds
``-ffp-contract=off`` (every a*b+c rounded twice, as in the B200 FP64 kernels
built with -fmad=false); flavour ``"_fast"`` keeps the stock contraction and
is the one timed as the CPU baseline.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
OUT = HERE / "_ref"
ORACLE_LIB = HERE / "_build" / "libtl_oracle.so"
REF = Path(os.environ.get("TEALEAF_REF", "/root/reference"))

# The system gcc carries libgomp; a CC from the environment may not.
CC = os.environ.get("TL_CC", "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc")
CFLAGS_STOCK = ["-O3", "-march=x86-64-v3", "-funroll-loops", "-std=gnu99", "-fopenmp",
                "-DNO_MPI", "-DENABLE_PROFILING", "-w"]
FLAVOURS = {"": ["-ffp-contract=off"], "_fast": []}

MPI_DIR = HERE / "minimpi"

SUITE_DIR = {"2d": REPO / "tealeaf_b200" / "suite" / "2d",
             "3d": REPO / "tealeaf_b200" / "suite" / "3d"}
LIB_DIR = REPO / "tealeaf_b200" / "lib"
LIB_NAME = {"2d": "tealeaf_b200_2d", "3d": "tealeaf_b200_3d"}


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(map(str, cmd)), r.stdout, r.stderr))


def build_oracle() -> Path:
    """Compile the C restatement (serial, strict IEEE) into a shared library."""
    src = HERE / "tl_oracle.c"
    ORACLE_LIB.parent.mkdir(parents=True, exist_ok=True)
    if _stale(ORACLE_LIB, [src]):
        _run([CC, "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=gnu99", "-o", ORACLE_LIB, src, "-lm"])
    return ORACLE_LIB


class _Job:
    def __init__(self, src, obj, incs, flags):
        self.src, self.obj, self.incs, self.flags = Path(src), Path(obj), [str(i) for i in incs], list(flags)


def _compile_all(jobs, parallel):
    todo = []
    for j in jobs:
        deps = [j.src] + [p for inc in j.incs for p in Path(inc).glob("*.h")]
        if _stale(j.obj, deps):
            j.obj.parent.mkdir(parents=True, exist_ok=True)
            todo.append([CC] + j.flags + ["-I%s" % i for i in j.incs] + ["-c", j.src, "-o", j.obj])
    with cf.ThreadPoolExecutor(max_workers=parallel) as ex:
        list(ex.map(_run, todo))


def _ext_include_dir(dim: str, suite: str) -> Path:
    """Directory that provides ``chunk_extension.h`` to the host sources.

    2D host headers include ``chunk_extension.h`` from the kernel-suite path
    (2d/chunk.h:7, 2d/Makefile:40-41). 3D host headers include
    ``build/chunk_extension.h`` (3d/chunk.h:5), which the reference make copies
    from the suite (3d/Makefile:38); the same copy is made here into ``_ref``.
    """
    src_dir = (REF / dim / "c_kernels" / "omp3") if suite == "omp3" else SUITE_DIR[dim]
    if dim == "2d":
        return src_dir
    inc = OUT / ("inc3d_" + suite)
    (inc / "build").mkdir(parents=True, exist_ok=True)
    dst = inc / "build" / "chunk_extension.h"
    src = src_dir / "chunk_extension.h"
    if _stale(dst, [src]):
        shutil.copyfile(src, dst)
    return inc


def _host_jobs(dim, suite, flav):
    root = REF / dim
    incs = [_ext_include_dir(dim, suite), root]
    flags = CFLAGS_STOCK + FLAVOURS[flav] + (["-DTL3D"] if dim == "3d" else [])
    srcs = sorted(root.glob("*.c")) + sorted((root / "drivers").glob("*.c"))
    objdir = OUT / "obj" / ("%s_host_%s%s" % (dim, suite, flav))
    return [_Job(s, objdir / (s.parent.name + "__" + s.stem + ".o"), incs, flags) for s in srcs]


def _omp3_jobs(dim, flav):
    kdir = REF / dim / "c_kernels" / "omp3"
    incs = [_ext_include_dir(dim, "omp3"), REF / dim, kdir]
    flags = CFLAGS_STOCK + FLAVOURS[flav]
    objdir = OUT / "obj" / ("%s_omp3%s" % (dim, flav))
    return [_Job(s, objdir / (s.stem + ".o"), incs, flags) for s in sorted(kdir.glob("*.c"))]


def _link(target: Path, objs, libs=(), force=False):
    if force or _stale(target, objs):
        _run([CC] + CFLAGS_STOCK + [str(o) for o in objs] + list(libs) + ["-lm", "-lrt", "-o", target])


def build_reference(dims=("2d", "3d"), with_b200=True, parallel=8) -> Path:
    """Compile the reference programs, the harnesses and the layout probes."""
    if not (REF / "2d" / "kernel_interface.h").exists():
        raise FileNotFoundError("reference sources not found at %s" % REF)
    OUT.mkdir(parents=True, exist_ok=True)
    for dim in dims:
        d_flags = ["-DTL3D"] if dim == "3d" else []
        mpi_flags = [f for f in CFLAGS_STOCK if f != "-DNO_MPI"] + FLAVOURS[""] + d_flags
        jobs = []
        plan = {}
        for flav in FLAVOURS:
            host = _host_jobs(dim, "omp3", flav)
            omp3 = _omp3_jobs(dim, flav)
            harness = _Job(HERE / "ref_harness.c", OUT / "obj" / ("%s_harness_omp3%s.o" % (dim, flav)),
                           [_ext_include_dir(dim, "omp3"), REF / dim], CFLAGS_STOCK + FLAVOURS[flav] + d_flags)
            jobs += host + omp3 + [harness]
            plan[flav] = (host, omp3, harness)
        layout = _Job(HERE / "layout_probe.c", OUT / "obj" / ("%s_layout.o" % dim),
                      [_ext_include_dir(dim, "omp3"), REF / dim], CFLAGS_STOCK + d_flags)
        probe = _Job(HERE / "decompose_probe.c", OUT / "obj" / ("%s_decompose.o" % dim),
                     [_ext_include_dir(dim, "omp3"), REF / dim], CFLAGS_STOCK + d_flags)
        jobs += [layout, probe]
        if with_b200:
            host_b200 = [j for j in _host_jobs(dim, "b200", "") if j.src.name != "main.c"]
            harness_b200 = _Job(HERE / "ref_harness.c", OUT / "obj" / ("%s_harness_b200.o" % dim),
                                [_ext_include_dir(dim, "b200"), REF / dim],
                                CFLAGS_STOCK + FLAVOURS[""] + d_flags)
            host_b200_mpi = [_Job(j.src, OUT / "obj" / ("%s_host_b200_mpi" % dim) / j.obj.name, j.incs + [MPI_DIR],
                                  [f for f in j.flags if f != "-DNO_MPI"]) for j in host_b200]
            harness_b200_mpi = _Job(HERE / "ref_harness.c", OUT / "obj" / ("%s_harness_b200_mpi.o" % dim),
                                    [_ext_include_dir(dim, "b200"), REF / dim, MPI_DIR], mpi_flags)
            jobs += host_b200 + [harness_b200] + host_b200_mpi + [harness_b200_mpi]
        host_mpi = [_Job(j.src, OUT / "obj" / ("%s_host_omp3_mpi" % dim) / j.obj.name, j.incs + [MPI_DIR],
                         [f for f in j.flags if f != "-DNO_MPI"])
                    for j in _host_jobs(dim, "omp3", "") if j.src.name != "main.c"]
        harness_mpi = _Job(HERE / "ref_harness.c", OUT / "obj" / ("%s_harness_omp3_mpi.o" % dim),
                           [_ext_include_dir(dim, "omp3"), REF / dim, MPI_DIR], mpi_flags)
        minimpi = _Job(MPI_DIR / "minimpi.c", OUT / "obj" / ("%s_minimpi.o" % dim), [MPI_DIR],
                       ["-O2", "-std=gnu99", "-D_POSIX_C_SOURCE=200809L"])
        jobs += host_mpi + [harness_mpi, minimpi]
        _compile_all(jobs, parallel)

        for flav, (host, omp3, harness) in plan.items():
            host_objs = [j.obj for j in host]
            no_main = [j.obj for j in host if j.src.name != "main.c"]
            k_objs = [j.obj for j in omp3]
            _link(OUT / ("tealeaf%s_omp3%s" % (dim, flav)), host_objs + k_objs)
            _link(OUT / ("harness%s_omp3%s" % (dim, flav)), [harness.obj] + no_main + k_objs)
        _link(OUT / ("layout%s" % dim), [layout.obj])
        host, omp3, _ = plan[""]
        _link(OUT / ("decompose%s" % dim), [probe.obj] + [j.obj for j in host if j.src.name != "main.c"]
              + [j.obj for j in omp3])
        _link(OUT / ("harness%s_omp3_mpi" % dim), [harness_mpi.obj] + [j.obj for j in host_mpi]
              + [j.obj for j in omp3] + [minimpi.obj])
        if with_b200:
            lib = LIB_DIR / ("lib%s.so" % LIB_NAME[dim])
            if not lib.exists():
                raise FileNotFoundError("build the B200 library first: %s" % lib)
            _link(OUT / ("harness%s_b200" % dim), [harness_b200.obj] + [j.obj for j in host_b200],
                  [lib, "-Wl,-rpath,$ORIGIN/../../tealeaf_b200/lib"], force=True)
            _link(OUT / ("harness%s_b200_mpi" % dim), [harness_b200_mpi.obj] + [j.obj for j in host_b200_mpi]
                  + [minimpi.obj], [lib, "-Wl,-rpath,$ORIGIN/../../tealeaf_b200/lib"], force=True)
    return OUT


if __name__ == "__main__":
    build_oracle()
    print(build_reference(with_b200="--no-b200" not in sys.argv))
