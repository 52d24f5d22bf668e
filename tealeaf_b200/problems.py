"""Seeded synthetic TeaLeaf problems, written as tea.in text.

The reference ships one hand-written geometry (2d/tea.in, 3d/tea.in) and no
generator; the workloads used here come from this module so that the
reference omp3 program and the B200 suite read byte-identical input files.

Generator (numpy PCG64, seed recorded in the header comment of the file):
  * state 1 is the ambient material (density 100, energy 1e-4);
  * rectangles/boxes: lower corner uniform in the domain, side lengths uniform
    in [0.5, 5], upper corner clipped to the domain; density 0.1, energy
    uniform in [0.1, 25];
  * circles: centre uniform in the domain, radius uniform in [0.3, 2];
    written as ``geometry=circular xmin=cx ymin=cy xmax=cx ymax=cy radius=r``
    (the parser needs all four extents, 2d/parse_config.c:253-262);
  * later states overwrite earlier ones (2d/c_kernels/omp3/set_chunk_state.c:24);
  * coefficient: reciprocal conductivity (1/density) throughout.

Numbers are written with ``repr`` so C ``atof`` and Python ``float`` read the
same doubles.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import List, Optional, Sequence

import numpy as np

SOLVER_KEYS = {"jacobi": "use_jacobi", "cg": "use_cg", "cheby": "use_chebyshev", "ppcg": "use_ppcg"}


@dataclass
class Problem:
    """One TeaLeaf run description (dims 2 or 3)."""
    dims: int
    cells: Sequence[int]
    states: List[str]                 # state lines without the leading "state N"
    domain_max: float = 10.0
    solver: str = "cg"
    eps: float = 1e-15
    max_iters: int = 20000
    end_step: int = 10
    dt: float = 0.004
    presteps: int = 30
    ppcg_inner_steps: int = 10
    coefficient: str = "inverse_density"
    check_result: bool = True
    summary_frequency: int = 10
    halo_depth: int = 2
    eps_lim: float = 1e-4
    error_switch: bool = False
    preconditioner: str = "none"      # CG: none, jac_diag or jac_block
    name: str = ""
    seed: Optional[int] = None

    def with_(self, **kw) -> "Problem":
        return replace(self, **kw)

    def tea_in(self) -> str:
        axes = "xyz"[: self.dims]
        out = ["*tea", "! %s seed=%s" % (self.name, self.seed)]
        for n, body in enumerate(self.states, start=1):
            out.append("state %d %s" % (n, body))
        out.append("")
        for a in axes:
            out.append("%smin = 0.0" % a)
        for a in axes:
            out.append("%smax = %r" % (a, float(self.domain_max)))
        for a, n in zip(axes, self.cells):
            out.append("%s_cells = %d" % (a, n))
        out.append("")
        out.append(SOLVER_KEYS[self.solver])
        out.append("use_c_kernels")
        if self.check_result:
            out.append("check_result")
        if self.error_switch:
            out.append("errswitch")
        if self.preconditioner != "none":
            out.append("preconditioner_on")
            out.append("preconditioner_type = %s" % self.preconditioner)
        out.append("coefficient_" + self.coefficient)
        out.append("")
        out.append("eps = %r" % self.eps)
        out.append("max_iters = %d" % self.max_iters)
        out.append("initial_timestep = %r" % self.dt)
        out.append("end_step = %d" % self.end_step)
        out.append("end_time = 100.0")
        out.append("summary_frequency = %d" % self.summary_frequency)
        out.append("halo_depth = %d" % self.halo_depth)
        out.append("num_chunks_per_rank = 1")
        out.append("presteps = %d" % self.presteps)
        out.append("ppcg_inner_steps = %d" % self.ppcg_inner_steps)
        out.append("epslim = %r" % self.eps_lim)
        out.append("*endtea")
        return "\n".join(out) + "\n"


AMBIENT = "density=100.0 energy=0.0001"


def _box(rng, dims, lo_max, side_lo=0.5, side_hi=5.0):
    lo = [float(rng.uniform(0.0, lo_max)) for _ in range(dims)]
    hi = [min(l + float(rng.uniform(side_lo, side_hi)), lo_max) for l in lo]
    return lo, hi


def _energy(rng):
    return float(rng.uniform(0.1, 25.0))


def seeded(dims: int, cells: Sequence[int], seed: int, n_rect: int, n_circ: int = 0,
           domain_max: float = 10.0, **kw) -> Problem:
    """Ambient + n_rect boxes (+ n_circ circles, 2D) from one PCG64 stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    states = [AMBIENT]
    rect_word = "cuboid" if dims == 3 else "rectangle"
    for _ in range(n_rect):
        lo, hi = _box(rng, dims, domain_max)
        e = _energy(rng)
        ext = " ".join("%smin=%r" % (a, v) for a, v in zip("xyz", lo))
        ext += " " + " ".join("%smax=%r" % (a, v) for a, v in zip("xyz", hi))
        states.append("density=0.1 energy=%r geometry=%s %s" % (e, rect_word, ext))
    for _ in range(n_circ):
        c = [float(rng.uniform(0.0, domain_max)) for _ in range(dims)]
        rad = float(rng.uniform(0.3, 2.0))
        e = _energy(rng)
        ext = " ".join("%smin=%r" % (a, v) for a, v in zip("xyz", c))
        ext += " " + " ".join("%smax=%r" % (a, v) for a, v in zip("xyz", c))
        word = "spherical" if dims == 3 else "circular"
        states.append("density=0.1 energy=%r geometry=%s %s radius=%r" % (e, word, ext, rad))
    return Problem(dims=dims, cells=tuple(cells), states=states, domain_max=domain_max,
                   seed=seed, **kw)


# ---- the named workloads -------------------------------------------------

def plain_2d(n: int = 512, seed: int = 1, steps: int = 10, solver: str = "cg") -> Problem:
    """512^2 CPU-runnable case: 4 rectangles, CG, eps 1e-15, dt 0.004, 10 steps."""
    return seeded(2, (n, n), seed, 4, 0, solver=solver, end_step=steps, name="plain_2d_%d" % n)


def dropin_2d(n: int = 4096, seed: int = 2, steps: int = 10, solver: str = "cg") -> Problem:
    """4096^2 drop-in case: 8 rectangles + 4 circles; CG / Chebyshev (30 presteps) / PPCG (10 inner)."""
    return seeded(2, (n, n), seed, 8, 4, solver=solver, end_step=steps, presteps=30,
                  ppcg_inner_steps=10, name="dropin_2d_%d_%s" % (n, solver))


def mixed_2d(n: int = 8192, seed: int = 3, steps: int = 10) -> Problem:
    """8192^2 mixed-precision case: 16 rectangles."""
    return seeded(2, (n, n), seed, 16, 0, solver="cg", end_step=steps, name="mixed_2d_%d" % n)


def adjoint_3d(n: int = 256, seed: int = 4, steps: int = 20) -> Problem:
    """3D adjoint case: 6 boxes on [0,10]^3, CG, 20 steps."""
    return seeded(3, (n, n, n), seed, 6, 0, solver="cg", end_step=steps, name="adjoint_3d_%d" % n)


def batched_2d(count: int = 64, seed: int = 5, lo: int = 128, hi: int = 2048,
               steps: int = 1) -> List[Problem]:
    """Batch of independent 2D problems: sides log-uniform in [lo, hi], 3 rectangles each, eps 1e-12."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for b in range(count):
        nx = int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))
        ny = int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))
        sub_seed = int(rng.integers(0, 2**31 - 1))
        out.append(seeded(2, (nx, ny), sub_seed, 3, 0, solver="cg", eps=1e-12, end_step=steps,
                          name="batched_2d_%d" % b))
    return out
