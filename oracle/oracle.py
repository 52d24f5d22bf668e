"""Python access to the checkers (TEST INFRASTRUCTURE, never the product).

* ``OracleLib``: ctypes bindings of ``libtl_oracle.so``, the serial C
  restatement in ``tl_oracle.c`` (per-kernel functions and whole runs).
* ``run_reference``: runs a reference-host harness binary from ``oracle/_ref``
  (omp3 suite, or the B200 suite behind the unchanged host) on a tea.in and
  parses per-step iteration counts and field summaries.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
LIB_PATH = HERE / "_build" / "libtl_oracle.so"

SOLVER_IDS = {"jacobi": 0, "cg": 1, "cheby": 2, "ppcg": 3}


class OSettings(C.Structure):
    _fields_ = [("dims", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("halo_depth", C.c_int),
                ("xmin", C.c_double), ("ymin", C.c_double), ("zmin", C.c_double),
                ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
                ("dt_init", C.c_double), ("eps", C.c_double), ("eps_lim", C.c_double),
                ("max_iters", C.c_int), ("end_step", C.c_int), ("solver", C.c_int),
                ("coefficient", C.c_int), ("presteps", C.c_int), ("ppcg_inner_steps", C.c_int),
                ("error_switch", C.c_int), ("check_result", C.c_int), ("summary_frequency", C.c_int),
                ("preconditioner", C.c_int)]


class OState(C.Structure):
    _fields_ = [("density", C.c_double), ("energy", C.c_double), ("x_min", C.c_double),
                ("y_min", C.c_double), ("z_min", C.c_double), ("x_max", C.c_double),
                ("y_max", C.c_double), ("z_max", C.c_double), ("radius", C.c_double),
                ("geometry", C.c_int)]


class OStep(C.Structure):
    _fields_ = [("total_iters", C.c_int), ("cg_iters", C.c_int), ("cheby_iters", C.c_int),
                ("ppcg_iters", C.c_int), ("jacobi_iters", C.c_int), ("est_iters", C.c_int),
                ("error", C.c_double), ("eigmin", C.c_double), ("eigmax", C.c_double),
                ("exact_error", C.c_double), ("vol", C.c_double), ("mass", C.c_double),
                ("ie", C.c_double), ("temp", C.c_double)]


@dataclass
class StepResult:
    """Per-timestep outcome in the reference's own terms."""
    iterations: Dict[str, int] = field(default_factory=dict)   # "CG", "Cheby", "PPCG", "Jacobi"
    summary: List[float] = field(default_factory=list)         # vol, mass, ie, temp
    seconds: float = 0.0
    extra: Dict[str, float] = field(default_factory=dict)


_P = C.POINTER(C.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_P)


class OracleLib:
    """ctypes view of libtl_oracle.so."""

    def __init__(self, path: Path = LIB_PATH):
        if not Path(path).exists():
            from oracle.build_ref import build_oracle  # build on demand (gcc is in the image)
            build_oracle()
        self.lib = C.CDLL(str(path))
        d, i = C.c_double, C.c_int
        self.lib.oracle_run.argtypes = [C.POINTER(OSettings), C.POINTER(OState), i, C.POINTER(OStep), _P]
        self.lib.oracle_run.restype = i
        for name in ("o2_cg_init",):
            getattr(self.lib, name).restype = d
        for name in ("o2_cg_calc_w", "o2_cg_calc_ur", "o2_calculate_2norm", "o2_jacobi_iterate",
                     "o3_cg_init", "o3_cg_calc_w", "o3_cg_calc_ur", "o3_calculate_2norm",
                     "o3_jacobi_iterate"):
            getattr(self.lib, name).restype = d
        self.lib.o_eigenvalue_bounds.restype = i
        self.lib.o_cheby_est_iterations.restype = i
        self.lib.o_cheby_est_iterations.argtypes = [d, d, d, d]

    def __getattr__(self, name):
        return getattr(self.lib, name)

    # -- whole runs --------------------------------------------------------
    @staticmethod
    def _settings(config):
        s = OSettings()
        s.dims = config.dims
        s.nx, s.ny = config.grid_x_cells, config.grid_y_cells
        s.nz = config.grid_z_cells if config.dims == 3 else 1
        s.halo_depth = config.halo_depth
        s.xmin, s.ymin, s.zmin = config.grid_x_min, config.grid_y_min, config.grid_z_min
        s.xmax, s.ymax, s.zmax = config.grid_x_max, config.grid_y_max, config.grid_z_max
        s.dt_init, s.eps, s.eps_lim = config.dt_init, config.eps, config.eps_lim
        s.max_iters, s.end_step, s.solver = config.max_iters, config.end_step, config.solver
        s.coefficient, s.presteps, s.ppcg_inner_steps = config.coefficient, config.presteps, config.ppcg_inner_steps
        s.error_switch, s.check_result = int(config.error_switch), int(config.check_result)
        s.summary_frequency = config.summary_frequency
        s.preconditioner = config.preconditioner_type
        return s

    @staticmethod
    def _states(states):
        arr = (OState * len(states))()
        for n, st in enumerate(states):
            arr[n] = OState(st.density, st.energy, st.x_min, st.y_min, st.z_min, st.x_max,
                            st.y_max, st.z_max, st.radius, st.geometry)
        return arr

    # -- the CPU adjoint (3D CG timestep) ----------------------------------
    def adjoint3d(self, config, states, box, adj_tol: float):
        """(J, dJ/dlog(density) as an (nz, ny, nx) array) after end_step timesteps."""
        s, arr = self._settings(config), self._states(states)
        out = np.zeros((s.nz, s.ny, s.nx))
        J = C.c_double()
        b = (C.c_double * 6)(*box)
        rc = self.lib.oracle_adjoint3d(C.byref(s), arr, len(states), b, C.c_double(adj_tol), C.byref(J), _ptr(out))
        if rc != 0:
            raise RuntimeError("oracle adjoint failed with code %d" % rc)
        return J.value, out

    def objective3d(self, config, states, box, cell: int = -1, log_scale: float = 0.0) -> float:
        """J with density[cell] (interior index, x fastest) scaled by exp(log_scale)."""
        s, arr = self._settings(config), self._states(states)
        J = C.c_double()
        b = (C.c_double * 6)(*box)
        rc = self.lib.oracle_objective3d(C.byref(s), arr, len(states), b, C.c_long(cell), C.c_double(log_scale),
                                         C.byref(J))
        if rc != 0:
            raise RuntimeError("oracle objective failed with code %d" % rc)
        return J.value

    def run(self, config, states, want_energy: bool = False):
        """Run initialise + end_step timesteps; config/states from tealeaf_b200.config."""
        s = self._settings(config)
        arr = self._states(states)
        steps = (OStep * config.end_step)()
        hd = config.halo_depth
        if config.dims == 3:
            n = (s.nx + 2 * hd) * (s.ny + 2 * hd) * (s.nz + 2 * hd)
        else:
            n = (s.nx + 2 * hd) * (s.ny + 2 * hd)
        energy = np.zeros(n) if want_energy else None
        rc = self.lib.oracle_run(C.byref(s), arr, len(states), steps, _ptr(energy) if want_energy else None)
        if rc != 0:
            raise RuntimeError("oracle run failed with code %d" % rc)
        out = []
        names = {0: "Jacobi", 1: "CG", 2: "Cheby", 3: "PPCG"}
        for st in steps:
            it = {}
            if config.solver == 0:
                it["Jacobi"] = st.jacobi_iters
            else:
                it["CG"] = st.cg_iters
            if config.solver == 2:
                it["Cheby"] = st.cheby_iters
            if config.solver == 3:
                it["PPCG"] = st.ppcg_iters
            out.append(StepResult(iterations=it, summary=[st.vol, st.mass, st.ie, st.temp],
                                  extra={"error": st.error, "eigmin": st.eigmin, "eigmax": st.eigmax,
                                         "exact_error": st.exact_error, "est_iters": st.est_iters}))
        return (out, energy) if want_energy else out


_ITER_RE = re.compile(r"^(CG|Cheby|PPCG|Jacobi):\s+(\d+) iterations")


def parse_harness_output(text: str) -> List[StepResult]:
    steps: List[StepResult] = []
    cur: Dict[str, int] = {}
    for line in text.splitlines():
        m = _ITER_RE.match(line.strip())
        if m:
            cur[m.group(1)] = int(m.group(2))
            continue
        if line.startswith("TLSTEP"):
            parts = line.split()
            steps.append(StepResult(iterations=dict(cur), summary=[float(v) for v in parts[2:6]],
                                    seconds=float(parts[6])))
            cur = {}
    return steps


def harness_path(dims: int, suite: str = "omp3", fast: bool = False) -> Path:
    name = "harness%dd_%s%s" % (dims, suite, "_fast" if fast and suite == "omp3" else "")
    return REF_DIR / name


def run_reference(tea_in_text: str, dims: int = 2, suite: str = "omp3", threads: Optional[int] = None,
                  fast: bool = False, max_iters: Optional[int] = None, timeout: float = 3600.0,
                  env_extra: Optional[dict] = None, warm: Optional[tuple] = None) -> List[StepResult]:
    """Run a reference-host harness in a scratch directory and parse its output.
    `max_iters` caps every timestep's solve; `warm` = (steps, cap) gives the
    first `steps` timesteps a cap of their own (warm-up steps)."""
    exe = harness_path(dims, suite, fast)
    if not exe.exists():
        raise FileNotFoundError("%s is missing (build with oracle/build_ref.py)" % exe)
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    if env_extra:
        env.update(env_extra)
    with tempfile.TemporaryDirectory(prefix="tl_ref_") as tmp:
        Path(tmp, "tea.in").write_text(tea_in_text)
        cmd = [str(exe), "tea.in"] + ([str(max_iters)] if max_iters is not None else [])
        if warm is not None and max_iters is not None:
            cmd += [str(int(warm[0])), str(int(warm[1]))]
        r = subprocess.run(cmd, cwd=tmp, env=env, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("%s failed (%d):\n%s\n%s" % (exe.name, r.returncode, r.stdout[-4000:], r.stderr[-4000:]))
        return parse_harness_output(r.stdout)


def run_reference_ranks(tea_in_text: str, dims: int, ranks: int, threads: int = 1,
                        timeout: float = 600.0, suite: str = "omp3") -> List[StepResult]:
    """The reference program's own multi-rank run: `ranks` processes of the
    parity harness built over oracle/minimpi, each in a scratch directory of
    its own (the reference writes its log there), connected through sockets
    in a shared one; the master rank's per-step iteration counts and summed
    field summaries. Every rank must exit 0. `suite` "b200" runs the same
    host linked with the B200 library (every rank on the default GPU)."""
    exe = REF_DIR / ("harness%dd_%s_mpi" % (dims, suite))
    if not exe.exists():
        raise FileNotFoundError("%s is missing (build with oracle/build_ref.py)" % exe)
    with tempfile.TemporaryDirectory(prefix="tlm", dir="/tmp") as tmp:
        deck = Path(tmp, "tea.in")
        deck.write_text(tea_in_text)
        procs = []
        for r in range(ranks):
            cwd = Path(tmp, "r%d" % r)
            cwd.mkdir()
            env = dict(os.environ, OMP_NUM_THREADS=str(threads), MINIMPI_RANK=str(r), MINIMPI_SIZE=str(ranks),
                       MINIMPI_DIR=tmp, MINIMPI_TIMEOUT=str(int(timeout)))
            procs.append(subprocess.Popen([str(exe), str(deck)], cwd=cwd, env=env, stdout=subprocess.PIPE,
                                          stderr=subprocess.PIPE, text=True))
        outs = []
        try:
            for p in procs:
                outs.append(p.communicate(timeout=timeout))
        finally:
            for p in procs:
                if p.poll() is None:
                    p.kill()
        for r, (p, (out, err)) in enumerate(zip(procs, outs)):
            if p.returncode != 0:
                raise RuntimeError("%s rank %d failed (%d):\n%s\n%s" % (exe.name, r, p.returncode, out[-4000:],
                                                                       err[-4000:]))
        return parse_harness_output(outs[0][0])
