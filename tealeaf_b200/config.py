"""tea.in reader: the host-side settings and states of a TeaLeaf run.

Mirrors the reference parser so that the B200 host and the reference host read
identical numbers from the same file:

* defaults: 2d/settings.c:6-60 (3d/settings.c);
* keys: 2d/parse_config.c:77-192 -- a key matches when the line *starts with*
  it after leading blanks (``starts_with``, :289-314) and its value is the
  first alphanumeric token after the key text (``read_value``, :317-340);
  keys are tried in the reference order, so ``epslim`` wins over ``eps``;
  ``x_cells``/``y_cells`` are only read while they still hold the default
  (:102-107);
* states: 2d/parse_config.c:195-286 -- state extents are moved inwards by a
  hundredth of a cell (``xmin + dx/100``, ``xmax - dx/100``), circles and
  spheres included (their centre is ``xmin``/``ymin``/``zmin``).
"""
from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path
from typing import List, Optional, Tuple

JACOBI_SOLVER, CG_SOLVER, CHEBY_SOLVER, PPCG_SOLVER = 0, 1, 2, 3
CONDUCTIVITY, RECIP_CONDUCTIVITY = 1, 2
# 2D geometry enum (2d/settings.h:131-136); 3D uses CUBOID/SPHERICAL/POINT (same values).
RECTANGULAR, CIRCULAR, POINT = 0, 1, 2
INT32_MAX = 2147483647


@dataclass
class Config:
    """Settings of one run (field names follow the reference ``Settings``)."""
    dims: int = 2
    grid_x_min: float = 0.0
    grid_y_min: float = 0.0
    grid_z_min: float = 0.0
    grid_x_max: float = 100.0
    grid_y_max: float = 100.0
    grid_z_max: float = 100.0
    grid_x_cells: int = 10
    grid_y_cells: int = 10
    grid_z_cells: int = 10
    dt_init: float = 0.1
    max_iters: int = 1000
    eps: float = 1.0e-15
    end_time: float = 10.0
    end_step: int = INT32_MAX
    summary_frequency: int = 10
    solver: int = CG_SOLVER
    solver_name: str = ""
    coefficient: int = CONDUCTIVITY
    error_switch: bool = False
    presteps: int = 30
    eps_lim: float = 1.0e-5
    check_result: bool = True
    ppcg_inner_steps: int = 10
    preconditioner: bool = False
    # Jacobi preconditioner of the device-resident CG: 0 none, 1 jac_diag,
    # 2 jac_block. The reference C parser only reads `preconditioner_on`
    # (2d/parse_config.c:136-138), which selects jac_diag here;
    # `preconditioner_type = jac_diag | jac_block | none` is the reference
    # README's tl_preconditioner_type (README.md:127-133).
    preconditioner_type: int = 0
    num_chunks_per_rank: int = 1
    halo_depth: int = 2
    kernel_language: Optional[int] = None   # never defaulted by the reference
    dx: float = 0.0
    dy: float = 0.0
    dz: float = 0.0

    @property
    def cells(self) -> int:
        n = self.grid_x_cells * self.grid_y_cells
        return n * self.grid_z_cells if self.dims == 3 else n


@dataclass
class StateDef:
    """One ``state`` line after parsing (reference ``State``)."""
    density: float
    energy: float
    x_min: float = 0.0
    y_min: float = 0.0
    z_min: float = 0.0
    x_max: float = 0.0
    y_max: float = 0.0
    z_max: float = 0.0
    radius: float = 0.0
    geometry: int = RECTANGULAR
    defined: bool = True


def _starts_with(word: str, line: str) -> bool:
    n = 0
    for ch in line:
        if n == 0 and ch.isspace():
            continue
        if ch != word[n]:
            return False
        n += 1
        if n == len(word):
            return True
    return False


def _read_value(line: str, word: str) -> str:
    n = 0
    for ll, ch in enumerate(line):
        if n == len(word):
            if ch.isalpha() or ch.isdigit():
                return line[ll:].split()[0]
        else:
            n = n + 1 if ch == word[n] else 0
    raise ValueError("Failed to find a value for key '%s'" % word)


def _atof(s: str) -> float:
    """C atof on the token (longest valid numeric prefix)."""
    for end in range(len(s), 0, -1):
        try:
            return float(s[:end])
        except ValueError:
            continue
    return 0.0


def _atoi(s: str) -> int:
    digits = ""
    for i, ch in enumerate(s):
        if ch.isdigit() or (i == 0 and ch in "+-"):
            digits += ch
        else:
            break
    try:
        return int(digits)
    except ValueError:
        return 0


def read_config(text: str, dims: int = 2) -> Tuple[Config, List[StateDef]]:
    """Parse tea.in text the way 2d/parse_config.c (or 3d) does."""
    c = Config(dims=dims)
    lines = text.splitlines(keepends=True)
    for line in lines:
        def sd(key, attr):
            if _starts_with(key, line):
                setattr(c, attr, _atof(_read_value(line, key)))
                return True
            return False

        def si(key, attr):
            if _starts_with(key, line):
                setattr(c, attr, _atoi(_read_value(line, key)))
                return True
            return False

        if sd("initial_timestep", "dt_init") or sd("end_time", "end_time") or si("end_step", "end_step"):
            continue
        if sd("xmin", "grid_x_min") or sd("ymin", "grid_y_min"):
            continue
        if dims == 3 and sd("zmin", "grid_z_min"):
            continue
        if sd("xmax", "grid_x_max") or sd("ymax", "grid_y_max"):
            continue
        if dims == 3 and sd("zmax", "grid_z_max"):
            continue
        # 2D reads the cell counts only while they hold the default
        # (2d/parse_config.c:102-107); 3D always does (3d/parse_config.c:111-116).
        if (dims == 3 or c.grid_x_cells == 10) and si("x_cells", "grid_x_cells"):
            continue
        if (dims == 3 or c.grid_y_cells == 10) and si("y_cells", "grid_y_cells"):
            continue
        if dims == 3 and si("z_cells", "grid_z_cells"):
            continue
        if (si("summary_frequency", "summary_frequency") or si("presteps", "presteps")
                or si("ppcg_inner_steps", "ppcg_inner_steps") or sd("epslim", "eps_lim")
                or si("max_iters", "max_iters") or sd("eps", "eps")
                or si("num_chunks_per_rank", "num_chunks_per_rank") or si("halo_depth", "halo_depth")):
            continue
        switches = [("check_result", "check_result", True), ("errswitch", "error_switch", True),
                    ("preconditioner_on", "preconditioner", True)]
        hit = False
        for key, attr, val in switches:
            if _starts_with(key, line):
                setattr(c, attr, val)
                hit = True
                break
        if hit:
            continue
        if _starts_with("preconditioner_type", line):
            v = _read_value(line, "preconditioner_type").strip().lower()
            c.preconditioner_type = {"jac_diag": 1, "jac_block": 2}.get(v, 0)
            c.preconditioner = c.preconditioner_type != 0
            continue
        if _starts_with("use_fortran_kernels", line):
            c.kernel_language = 1
            continue
        if _starts_with("use_c_kernels", line):
            c.kernel_language = 0
            continue
        solvers = [("use_jacobi", JACOBI_SOLVER, "Jacobi"), ("use_cg", CG_SOLVER, "CG"),
                   ("use_chebyshev", CHEBY_SOLVER, "Chebyshev"), ("use_ppcg", PPCG_SOLVER, "PPCG")]
        for key, sv, name in solvers:
            if _starts_with(key, line):
                c.solver, c.solver_name = sv, name
                hit = True
                break
        if hit:
            continue
        if _starts_with("coefficient_density", line):
            c.coefficient = CONDUCTIVITY
            continue
        if _starts_with("coefficient_inverse_density", line):
            c.coefficient = RECIP_CONDUCTIVITY
            continue

    c.dx = (c.grid_x_max - c.grid_x_min) / float(c.grid_x_cells)
    c.dy = (c.grid_y_max - c.grid_y_min) / float(c.grid_y_cells)
    if dims == 3:
        c.dz = (c.grid_z_max - c.grid_z_min) / float(c.grid_z_cells)

    # states (2d/parse_config.c:195-286)
    num_states = 0
    for line in lines:
        if _starts_with("state", line):
            num_states = max(num_states, _atoi(_read_value(line, "state")))
    states: List[Optional[StateDef]] = [None] * num_states
    for line in lines:
        if not _starts_with("state", line):
            continue
        sn = _atoi(_read_value(line, "state"))
        if states[sn - 1] is not None:
            raise ValueError("State number %d defined twice." % sn)
        st = StateDef(density=_atof(_read_value(line, "density")), energy=_atof(_read_value(line, "energy")))
        if sn > 1:
            st.x_min = _atof(_read_value(line, "xmin")) + c.dx / 100.0
            st.y_min = _atof(_read_value(line, "ymin")) + c.dy / 100.0
            if dims == 3:
                st.z_min = _atof(_read_value(line, "zmin")) + c.dz / 100.0
            st.x_max = _atof(_read_value(line, "xmax")) - c.dx / 100.0
            st.y_max = _atof(_read_value(line, "ymax")) - c.dy / 100.0
            if dims == 3:
                st.z_max = _atof(_read_value(line, "zmax")) - c.dz / 100.0
            geom = _read_value(line, "geometry")
            if geom == ("cuboid" if dims == 3 else "rectangle"):
                st.geometry = RECTANGULAR
            elif geom == ("spherical" if dims == 3 else "circular"):
                st.geometry = CIRCULAR
                st.radius = _atof(_read_value(line, "radius"))
            elif geom == "point":
                st.geometry = POINT
        states[sn - 1] = st
    if c.preconditioner and c.preconditioner_type == 0:
        c.preconditioner_type = 1   # preconditioner_on alone: jac_diag
    return c, [s if s is not None else StateDef(0.0, 0.0, defined=False) for s in states]


def read_config_file(path, dims: int = 2) -> Tuple[Config, List[StateDef]]:
    return read_config(Path(path).read_text(), dims)
