"""Pins the CPU adjoint of the oracle (oracle_adjoint3d in oracle/tl_oracle.c)
before the B200 adjoint is compared with it.

The reference has no adjoint, so the pin is the reference's own forward
timestep (the oracle's restatement of 3d/c_kernels/omp3/cg_solver.c, itself
pinned to the reference program) differentiated by central differences:
J(log rho_c + h) - J(log rho_c - h) over 2h, h = 1e-6. A central difference
is exact to O(h^2) but carries the rounding of J: |dJ| ~ eps * |J| / h, the
noise floor each comparison is allowed on top of the stated 1e-6 relative.
"""
import numpy as np
import pytest

from tealeaf_b200 import problems
from tealeaf_b200.config import read_config

BOX = [6.0, 9.0, 6.0, 9.0, 6.0, 9.0]
H = 1e-6
RTOL = 1e-6


def _case(steps=3):
    prob = problems.seeded(3, (12, 10, 8), 21, 6, 0, solver="cg", eps=1e-14, end_step=steps, name="adj_small")
    return read_config(prob.tea_in(), 3)


def test_cpu_adjoint_matches_central_differences(oracle_lib):
    cfg, states = _case()
    J, g = oracle_lib.adjoint3d(cfg, states, BOX, 1e-14)
    assert J > 0.0
    gf = g.ravel()
    rng = np.random.default_rng(7)
    cells = list(np.argsort(-np.abs(gf))[:6]) + list(rng.integers(0, gf.size, 6))
    noise = 8.0 * np.finfo(float).eps * abs(J) / (2 * H)
    for c in cells:
        jp = oracle_lib.objective3d(cfg, states, BOX, int(c), H)
        jm = oracle_lib.objective3d(cfg, states, BOX, int(c), -H)
        fd = (jp - jm) / (2 * H)
        assert abs(fd - gf[c]) <= RTOL * abs(gf[c]) + noise, (c, gf[c], fd)


def test_cpu_objective_unperturbed_matches_adjoint_J(oracle_lib):
    cfg, states = _case(steps=2)
    J, _ = oracle_lib.adjoint3d(cfg, states, BOX, 1e-12)
    assert oracle_lib.objective3d(cfg, states, BOX) == J
