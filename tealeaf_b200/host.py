"""Python host over the reference kernel interface (the ``run_*`` C ABI).

A line-by-line behavioural mirror of the reference host that sits above
``kernel_interface.h``: initialisation (2d/initialise.c:11-31), the timestep
``solve`` (2d/diffuse.c:22-80) and the solver drivers (2d/drivers/*.c,
3d/drivers/*.c), including their halo-flag bookkeeping, accumulate-style
reductions and the 2D/3D difference in the stop test (3D tests sqrt(error)).
It calls the B200 suite only through the exported C functions, exactly as the
C drivers do, so it exercises the drop-in boundary from Python (tests, the
end-to-end bench leg).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import abi
from .config import (CG_SOLVER, CHEBY_SOLVER, JACOBI_SOLVER, PPCG_SOLVER, Config, StateDef,
                     read_config)

FIELD_DENSITY, FIELD_ENERGY0, FIELD_ENERGY1, FIELD_U, FIELD_P, FIELD_SD = range(6)
CG_ITERS_FOR_EIGENVALUES = 20
ERROR_SWITCH_MAX = 1.0
DBL_EPSILON = 2.220446049250313e-16
DBL_MAX = 1.7976931348623157e308
DBL_MIN = 2.2250738585072014e-308

# 2D name -> 3D name of the renamed entry points (3d/kernel_interface.h).
_NAMES3 = {"run_cg_init": "run_cg_solver_init", "run_cg_calc_w": "run_cg_solver_calc_w",
           "run_cg_calc_ur": "run_cg_solver_calc_ur", "run_cg_calc_p": "run_cg_solver_calc_p",
           "run_cheby_init": "run_cheby_solver_init", "run_cheby_iterate": "run_cheby_solver_iterate",
           "run_jacobi_init": "run_jacobi_solver_init", "run_jacobi_iterate": "run_jacobi_solver_iterate",
           "run_copy_u": "run_solver_copy_u", "run_finalise": "run_solver_finalise"}

# Field ids of the staging calls (TL2D_* / TL3D_* in the headers).
FIELD_IDS = {"density0": 0, "density": 1, "energy0": 2, "energy": 3, "u": 4, "u0": 5, "p": 6, "r": 7,
             "mi": 8, "w": 9, "kx": 10, "ky": 11, "sd": 12, "volume": 13, "kz": 14}


@dataclass
class StepResult:
    iterations: Dict[str, int] = field(default_factory=dict)
    summary: List[float] = field(default_factory=list)      # vol, mass, ie, temp
    error: float = 0.0
    exact_error: float = 0.0
    eigmin: float = 0.0
    eigmax: float = 0.0
    est_iterations: int = 0


@dataclass
class RefineResult:
    iterations: int = 0
    residual_updates: int = 0
    converged: bool = False
    rel_residual: float = 0.0
    device_ms: float = 0.0
    summary: List[float] = field(default_factory=list)      # vol, mass, ie, temp
    cg_trips: int = 0      # PPCG: CG trips before the switch (CG: all of them)


class DriverError(RuntimeError):
    pass


def _tqli(d: List[float], e: List[float]) -> None:
    """Implicit-shift QL eigenvalues of a symmetric tridiagonal (in place), as
    used by 2d/drivers/eigenvalue_driver.c:71-121 (published "tqli")."""
    n = len(d)
    for i in range(n - 1):
        e[i] = e[i + 1]
    e[n - 1] = 0.0
    for l in range(n):
        sweeps = 0
        while True:
            m = l
            while m < n - 1:
                dd = abs(d[m]) + abs(d[m + 1])
                if abs(e[m]) + dd == dd:
                    break
                m += 1
            if m == l:
                break
            if sweeps == 30:
                raise DriverError("Too many iterations in TQLI routine")
            sweeps += 1
            g = (d[l + 1] - d[l]) / (2.0 * e[l])
            r = math.sqrt((g * g) + 1.0)
            g = d[m] - d[l] + e[l] / (g + (-abs(r) if g < 0 else abs(r)))
            s = c = 1.0
            p = 0.0
            i = m - 1
            while i >= l:
                f = s * e[i]
                b = c * e[i]
                r = math.sqrt(f * f + g * g)
                e[i + 1] = r
                if r == 0.0:
                    d[i + 1] -= p
                    e[m] = 0.0
                    i -= 1
                    continue
                s = f / r
                c = g / r
                g = d[i + 1] - p
                r = (d[i] - g) * s + 2.0 * c * b
                p = s * r
                d[i + 1] = g + p
                g = c * r - b
                i -= 1
            d[l] = d[l] - p
            e[l] = g
            e[m] = 0.0


def eigenvalue_bounds(alphas, betas, n):
    """eigenvalue_driver_initialise (2d/drivers/eigenvalue_driver.c:11-67)."""
    diag = [0.0] * n
    off = [0.0] * n
    for i in range(n):
        diag[i] = 1.0 / alphas[i]
        if i > 0:
            diag[i] += betas[i - 1] / alphas[i - 1]
        if i < n - 1:
            off[i + 1] = math.sqrt(betas[i]) / alphas[i]
    _tqli(diag, off)
    lo, hi = DBL_MAX, DBL_MIN
    for v in diag:
        lo = min(lo, v)
        hi = max(hi, v)
    if lo < 0.0 or hi < 0.0:
        raise DriverError("Calculated negative eigenvalues.")
    return lo * 0.95, hi * 1.05


def cheby_est_iterations(eigmin, eigmax, error, bb):
    """cheby_calc_est_iterations (2d/drivers/cheby_driver.c:146-160): single
    precision logarithms and roundf, evaluated through the C library."""
    libm = _libm()
    cn = eigmax / eigmin
    it_alpha = DBL_EPSILON * bb / (4.0 * error)
    gamm = (math.sqrt(cn) - 1.0) / (math.sqrt(cn) + 1.0)
    q = libm.logf(it_alpha) / (2.0 * libm.logf(gamm))
    return int(libm.roundf(q))


_LIBM = None


def _libm():
    global _LIBM
    if _LIBM is None:
        _LIBM = C.CDLL("libm.so.6")
        _LIBM.logf.argtypes = [C.c_float]
        _LIBM.logf.restype = C.c_float
        _LIBM.roundf.argtypes = [C.c_float]
        _LIBM.roundf.restype = C.c_float
    return _LIBM


class Host:
    """One chunk, one rank (-DNO_MPI), every face external."""

    def __init__(self, tea_in: str, dims: int = 2):
        self.dims = dims
        self.lib = self._load_lib()
        self.cfg, self.states = read_config(tea_in, dims)
        c = self.cfg
        if c.kernel_language not in (None, 0):
            raise DriverError("only C kernels are provided")
        self._keep = []  # ctypes buffers referenced by the structs
        self.chunk = (abi.Chunk2D if dims == 2 else abi.Chunk3D)()
        self.settings = (abi.Settings2D if dims == 2 else abi.Settings3D)()
        self._fill_settings()
        self._initialise_chunk()
        self.initialise_application()
        if dims == 2 and c.preconditioner_type:
            self.lib.tl2d_set_preconditioner(C.byref(self.chunk), c.preconditioner_type)
            abi.check(self.lib, dims)

    # -- plumbing ------------------------------------------------------------
    def _load_lib(self):
        return abi.load(self.dims)

    def _call(self, name, *args):
        if self.dims == 3:
            name = _NAMES3.get(name, name)
        getattr(self.lib, name)(C.byref(self.chunk), C.byref(self.settings), *args)
        abi.check(self.lib, self.dims)

    def _fill_settings(self):
        s, c = self.settings, self.cfg
        s.rank = 0
        s.end_step, s.presteps, s.max_iters = c.end_step, c.presteps, c.max_iters
        s.coefficient, s.ppcg_inner_steps = c.coefficient, c.ppcg_inner_steps
        s.summary_frequency, s.halo_depth = c.summary_frequency, c.halo_depth
        s.num_states = len(self.states)
        s.num_chunks = s.num_chunks_per_rank = s.num_ranks = 1
        flags = (C.c_bool * 6)()
        self._keep.append(flags)
        s.fields_to_exchange = C.cast(flags, C.POINTER(C.c_bool))
        s.error_switch, s.check_result, s.preconditioner = c.error_switch, c.check_result, c.preconditioner
        s.eps, s.dt_init, s.end_time, s.eps_lim = c.eps, c.dt_init, c.end_time, c.eps_lim
        s.solver = c.solver
        if self.dims == 2:
            name = C.create_string_buffer((c.solver_name or "").encode(), 256)
            self._keep.append(name)
            s.solver_name = C.cast(name, C.c_char_p)
        s.kernel_language = 0
        s.grid_x_cells, s.grid_y_cells = c.grid_x_cells, c.grid_y_cells
        s.grid_x_min, s.grid_y_min, s.grid_x_max, s.grid_y_max = c.grid_x_min, c.grid_y_min, c.grid_x_max, c.grid_y_max
        s.dx, s.dy = c.dx, c.dy
        if self.dims == 3:
            s.grid_z_cells, s.grid_z_min, s.grid_z_max, s.dz = c.grid_z_cells, c.grid_z_min, c.grid_z_max, c.dz

    def _initialise_chunk(self):
        """initialise_chunk + decompose_field for one chunk (2d/chunk.c:4-30, 2d/initialise.c:34-134)."""
        ch, c, hd = self.chunk, self.cfg, self.cfg.halo_depth
        ch.x = c.grid_x_cells + 2 * hd
        ch.y = c.grid_y_cells + 2 * hd
        if self.dims == 3:
            ch.z = c.grid_z_cells + 2 * hd
        ch.dt_init = c.dt_init
        nb = (C.c_int * 6)(*([-1] * 6))
        ext = abi.ChunkExtension()
        self._keep += [nb, ext]
        ch.neighbours = C.cast(nb, C.POINTER(C.c_int))
        ch.ext = C.pointer(ext)
        ch.left, ch.right = 0, c.grid_x_cells
        ch.bottom, ch.top = 0, c.grid_y_cells
        if self.dims == 3:
            ch.back, ch.front = 0, c.grid_z_cells

    @property
    def flags(self):
        return self.settings.fields_to_exchange

    def reset_fields_to_exchange(self):
        for i in range(6):
            self.flags[i] = False

    def halo_update(self, depth):
        """halo_update_driver (2d/drivers/halo_update_driver.c:6-25); remote halos are compiled out."""
        if any(self.flags[i] for i in range(6)):
            self._call("run_local_halos", depth)

    def initialise_application(self):
        """2d/initialise.c:11-31 after read_config."""
        self._call("run_kernel_initialise")
        self._call("run_set_chunk_data")
        st_t = abi.State2D if self.dims == 2 else abi.State3D
        arr = (st_t * len(self.states))()
        for n, sd in enumerate(self.states):
            rec = arr[n]
            rec.defined, rec.density, rec.energy = sd.defined, sd.density, sd.energy
            rec.x_min, rec.y_min, rec.x_max, rec.y_max = sd.x_min, sd.y_min, sd.x_max, sd.y_max
            rec.radius, rec.geometry = sd.radius, sd.geometry
            if self.dims == 3:
                rec.z_min, rec.z_max = sd.z_min, sd.z_max
        self._call("run_set_chunk_state", arr)
        self.reset_fields_to_exchange()
        self.flags[FIELD_DENSITY] = self.flags[FIELD_ENERGY0] = self.flags[FIELD_ENERGY1] = True
        self.halo_update(2)
        self._call("run_store_energy")

    def finalise(self):
        if getattr(self, "chunk", None) is not None and self.chunk.ext and self.chunk.ext.contents.suite:
            self.lib.run_kernel_finalise(C.byref(self.chunk), C.byref(self.settings))

    def __del__(self):
        try:
            self.finalise()
        except Exception:
            pass

    # -- scalar-returning calls ------------------------------------------------
    def _acc(self, name, *args):
        v = C.c_double(0.0)
        self._call(name, *args, C.byref(v))
        return v.value

    def _sum(self, value: float) -> float:
        """sum_over_ranks (2d/comms.c:55-61), called where the reference
        drivers call it; on one rank the value itself."""
        return value

    def field_summary(self):
        v = [C.c_double(0.0) for _ in range(4)]
        self._call("run_field_summary", *[C.byref(x) for x in v])
        return [self._sum(x.value) for x in v]

    def norm(self, which: str) -> float:
        ptr = getattr(self.chunk, which if self.dims == 2 else "vec_" + which)
        return self._acc("run_calculate_2norm", ptr)

    def _post_trip(self, error):
        return math.sqrt(error) if self.dims == 3 else error

    # -- CG (2d/drivers/cg_driver.c) --------------------------------------------
    def cg_init_driver(self, rx, ry, rz):
        args = (rx, ry) if self.dims == 2 else (rx, ry, rz)
        rro = self._sum(self._acc("run_cg_init", *args))
        self.reset_fields_to_exchange()
        self.flags[FIELD_U] = self.flags[FIELD_P] = True
        self.halo_update(1)
        self._call("run_copy_u")
        return rro

    def cg_main_step(self, tt, rro):
        pw = self._sum(self._acc("run_cg_calc_w"))
        alpha = rro / pw
        self.chunk.cg_alphas[tt] = alpha
        rrn = self._sum(self._acc("run_cg_calc_ur", alpha))
        beta = rrn / rro
        self.chunk.cg_betas[tt] = beta
        self._call("run_cg_calc_p", beta)
        return rrn, rrn  # (rro, error)

    def cg_driver(self, rx, ry, rz, res: StepResult):
        error = 1e10
        rro = self.cg_init_driver(rx, ry, rz)
        tt = 0
        while tt < self.cfg.max_iters:
            rro, error = self.cg_main_step(tt, rro)
            self.halo_update(1)
            error = self._post_trip(error)
            if abs(error) < self.cfg.eps:
                break
            tt += 1
        res.iterations["CG"] = tt
        return error

    def _switch(self, n_inner, tt, error):
        c = self.cfg
        if n_inner:
            return True
        if c.error_switch:
            return error < c.eps_lim and tt > CG_ITERS_FOR_EIGENVALUES
        return tt > c.presteps and error < ERROR_SWITCH_MAX

    def _cheby_coefs(self, count):
        """cheby_coef_driver (2d/drivers/cheby_driver.c:163-183)."""
        ch = self.chunk
        ch.theta = (ch.eigmax + ch.eigmin) / 2.0
        delta = (ch.eigmax - ch.eigmin) / 2.0
        sigma = ch.theta / delta
        rho_old = 1.0 / sigma
        for i in range(count):
            rho_new = 1.0 / (2.0 * sigma - rho_old)
            ch.cheby_alphas[i] = rho_new * rho_old
            ch.cheby_betas[i] = 2.0 * rho_new / delta
            rho_old = rho_new

    def _eigenvalues(self, n):
        ch = self.chunk
        ch.eigmin, ch.eigmax = eigenvalue_bounds(ch.cg_alphas, ch.cg_betas, n)

    # -- Chebyshev (2d/drivers/cheby_driver.c) ------------------------------------
    def cheby_driver(self, rx, ry, rz, res: StepResult):
        error = 1e10
        rro = self.cg_init_driver(rx, ry, rz)
        est, nch, tt = 0, 0, 0
        ch = self.chunk
        while tt < self.cfg.max_iters:
            if not self._switch(nch, tt, error):
                rro, error = self.cg_main_step(tt, rro)
            else:
                nch += 1
                if nch == 1:
                    self._eigenvalues(tt)
                    self._cheby_coefs(self.cfg.max_iters - tt)
                    bb = self._sum(self.norm("u0"))
                    self._call("run_cheby_init")
                    self.reset_fields_to_exchange()
                    self.flags[FIELD_U] = True
                    self.halo_update(1)
                    self._call("run_cheby_iterate", ch.cheby_alphas[nch], ch.cheby_betas[nch])
                    error = self._sum(self.norm("r"))
                    est = cheby_est_iterations(ch.eigmin, ch.eigmax, error, bb)
                else:
                    calc_norm = nch >= est and (tt + 1) % 10 == 0
                    self._call("run_cheby_iterate", ch.cheby_alphas[nch], ch.cheby_betas[nch])
                    if calc_norm:
                        error = self._sum(self.norm("r"))
            self.halo_update(1)
            error = self._post_trip(error)
            if abs(error) < self.cfg.eps:
                break
            tt += 1
        res.iterations["CG"] = tt - nch + 1
        res.iterations["Cheby"] = nch
        res.est_iterations = est
        res.eigmin, res.eigmax = ch.eigmin, ch.eigmax
        return error

    # -- PPCG (2d/drivers/ppcg_driver.c) ------------------------------------------
    def ppcg_driver(self, rx, ry, rz, res: StepResult):
        error = 1e10
        rro = self.cg_init_driver(rx, ry, rz)
        npp, tt = 0, 0
        ch = self.chunk
        while tt < self.cfg.max_iters:
            if not self._switch(npp, tt, error):
                rro, error = self.cg_main_step(tt, rro)
            else:
                npp += 1
                if npp == 1:
                    self._eigenvalues(tt)
                    self._cheby_coefs(self.cfg.ppcg_inner_steps)
                    self._call("run_calculate_residual")
                    self.reset_fields_to_exchange()
                    self.flags[FIELD_P] = True
                    self.halo_update(1)
                    # ppcg_init_driver sums rro over the ranks once more, although
                    # it already is the mesh's sum (2d/drivers/ppcg_driver.c:83,
                    # 3d/drivers/ppcg_solver_driver.c:84): N ranks scale it by N
                    rro = self._sum(rro)
                pw = self._sum(self._acc("run_cg_calc_w"))
                alpha = rro / pw
                self._acc("run_cg_calc_ur", alpha)
                self._call("run_ppcg_init")
                self.reset_fields_to_exchange()
                self.flags[FIELD_SD] = True
                for pp in range(self.cfg.ppcg_inner_steps):
                    self.halo_update(1)
                    self._call("run_ppcg_inner_iteration", ch.cheby_alphas[pp], ch.cheby_betas[pp])
                self.reset_fields_to_exchange()
                self.flags[FIELD_P] = True
                rrn = self._sum(self.norm("r"))
                beta = rrn / rro
                self._call("run_cg_calc_p", beta)
                error = rrn
                rro = rrn
            self.halo_update(1)
            error = self._post_trip(error)
            if abs(error) < self.cfg.eps:
                break
            tt += 1
        res.iterations["CG"] = tt - npp + 1
        res.iterations["PPCG"] = npp
        res.eigmin, res.eigmax = ch.eigmin, ch.eigmax
        return error

    # -- Jacobi (2d/drivers/jacobi_driver.c) --------------------------------------
    def jacobi_driver(self, rx, ry, rz, res: StepResult):
        args = (rx, ry) if self.dims == 2 else (rx, ry, rz)
        self._call("run_jacobi_init", *args)
        self._call("run_copy_u")
        self.reset_fields_to_exchange()
        self.flags[FIELD_U] = True
        error = 1e10
        tt = 0
        while tt < self.cfg.max_iters:
            v = C.c_double(error)
            self._call("run_jacobi_iterate", C.byref(v))
            error = v.value
            if tt % 50 == 0:
                self.halo_update(1)
                self._call("run_calculate_residual")
                error += self.norm("r")
            error = self._sum(error)
            self.halo_update(1)
            error = self._post_trip(error)
            if abs(error) < self.cfg.eps:
                break
            tt += 1
        res.iterations["Jacobi"] = tt
        return error

    # -- one timestep (2d/diffuse.c:22-80) ----------------------------------------
    def solve(self, tt: int) -> StepResult:
        c = self.cfg
        res = StepResult()
        dt = c.dt_init
        rx = dt / (c.dx * c.dx)
        ry = dt / (c.dy * c.dy)
        rz = dt / (c.dz * c.dz) if self.dims == 3 else 0.0
        self.reset_fields_to_exchange()
        self.flags[FIELD_ENERGY1] = self.flags[FIELD_DENSITY] = True
        self.halo_update(2)
        drivers = {JACOBI_SOLVER: self.jacobi_driver, CG_SOLVER: self.cg_driver,
                   CHEBY_SOLVER: self.cheby_driver, PPCG_SOLVER: self.ppcg_driver}
        res.error = drivers[c.solver](rx, ry, rz, res)
        # solve_finished_driver (2d/drivers/solve_finished_driver.c:7-43)
        if c.check_result:
            self._call("run_calculate_residual")
            res.exact_error = self._sum(self.norm("r"))
        self._call("run_finalise")
        self.flags[FIELD_ENERGY1] = True
        self.halo_update(1)
        res.summary = self.field_summary()
        return res

    # -- device-resident timestep (tl2d_solve_step) ----------------------------------
    def solve_device(self, tt: int, summary: bool = True) -> StepResult:
        """One timestep with the solver loop kept on the GPU (same results as solve());
        `summary` appends the field summary (vol, mass, ie, temp) to the result."""
        fn = getattr(self.lib, "tl%dd_solve_step" % self.dims)
        stats = abi.StepStats()
        fn(C.byref(self.chunk), C.byref(self.settings), tt, C.byref(stats))
        abi.check(self.lib, self.dims)
        res = StepResult(error=stats.error, exact_error=stats.exact_error, eigmin=stats.eigmin,
                         eigmax=stats.eigmax, est_iterations=stats.est_iters)
        s = self.cfg.solver
        res.iterations["CG"] = stats.cg_iters
        if s == CHEBY_SOLVER:
            res.iterations["Cheby"] = stats.cheby_iters
        elif s == PPCG_SOLVER:
            res.iterations["PPCG"] = stats.ppcg_iters
        elif s == JACOBI_SOLVER:
            res.iterations = {"Jacobi": stats.jacobi_iters}
        if summary:
            res.summary = self.field_summary()
        return res

    # -- iterative-refinement timestep (tl2d_refine_solve_step) -------------------------
    def refine_step(self, tt: int, rel_tol: float, precision: int, summary: bool = True) -> RefineResult:
        """One timestep whose solve stops at ||u0 - A u|| / ||u0|| <= rel_tol (FP64
        residual); precision 32 = FP32-stored CG (or PPCG when the deck selects it) with FP64
        refinement, 64 = the same iteration with FP64 storage."""
        if self.dims != 2:
            raise DriverError("the refinement form is 2D")
        st = abi.RefineStats()
        rc = self.lib.tl2d_refine_solve_step(C.byref(self.chunk), C.byref(self.settings), tt, rel_tol,
                                             precision, C.byref(st))
        abi.check(self.lib, self.dims)
        if rc:
            raise DriverError("tl2d_refine_solve_step returned %d" % rc)
        res = RefineResult(st.iterations, st.residual_updates, bool(st.converged), st.rel_residual, st.device_ms,
                           cg_trips=st.cg_trips)
        if summary:
            res.summary = self.field_summary()
        return res

    # -- 3D adjoint (tl3d_adjoint_gradient) ----------------------------------------
    def adjoint_gradient(self, steps: int, every: int, box, rel_tol: float):
        """(J, dJ/dlog(density) as an (nz, ny, nx) array, stats) for J = sum over the
        box of volume*density*u after `steps` timesteps from the current state."""
        if self.dims != 3:
            raise DriverError("the adjoint is 3D")
        c = self.cfg
        out = np.zeros((c.grid_z_cells, c.grid_y_cells, c.grid_x_cells))
        st = abi.AdjointStats()
        b = (C.c_double * 6)(*box)
        rc = self.lib.tl3d_adjoint_gradient(C.byref(self.chunk), C.byref(self.settings), steps, every, b, rel_tol,
                                            out.ctypes.data_as(C.c_void_p), C.byref(st))
        abi.check(self.lib, self.dims)
        if rc:
            raise DriverError("tl3d_adjoint_gradient returned %d" % rc)
        return st.J, out, st

    def run_device(self, steps: Optional[int] = None) -> List[StepResult]:
        n = self.cfg.end_step if steps is None else steps
        return [self.solve_device(tt) for tt in range(n)]

    def run(self, steps: Optional[int] = None) -> List[StepResult]:
        n = self.cfg.end_step if steps is None else steps
        return [self.solve(tt) for tt in range(n)]

    # -- host buffers ---------------------------------------------------------------
    @property
    def shape(self):
        ch = self.chunk
        return (ch.y, ch.x) if self.dims == 2 else (ch.z, ch.y, ch.x)

    def download(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        fn = getattr(self.lib, "tl%dd_download_field" % self.dims)
        fn(C.byref(self.chunk), C.byref(self.settings), FIELD_IDS[name], out.ctypes.data_as(C.c_void_p), out.size)
        abi.check(self.lib, self.dims)
        return out

    def upload(self, name: str, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.size == int(np.prod(self.shape))
        fn = getattr(self.lib, "tl%dd_upload_field" % self.dims)
        fn(C.byref(self.chunk), C.byref(self.settings), FIELD_IDS[name], a.ctypes.data_as(C.c_void_p), a.size)
        abi.check(self.lib, self.dims)
