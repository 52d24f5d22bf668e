"""Iterative-refinement timestep (tl2d_refine_solve_step) on the B200.

Stated accuracy of the form: every timestep stops at a relative FP64
residual ||u0 - A u||_2 / ||u0||_2 <= 1e-10 (checked on the residual the
suite recomputes in FP64 after the solve), in both precisions. Against the
FP64 oracle (the C restatement of the reference solve, run to r.r < 1e-28,
i.e. far below the 1e-10 residual) the field summary of either form is held
to: vol and mass exact (they do not depend on the solve), temp within
TEMP_RTOL relative, step after step (the energy of each step feeds the next).
"""
import numpy as np
import pytest

from tealeaf_b200 import problems
from tealeaf_b200.config import read_config
from tealeaf_b200.host import DriverError, Host

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10
TEMP_RTOL = 1e-9   # temp vs the oracle's converged solve, after 3 timesteps


def _problem(steps=3, eps=1e-15, n=(160, 120)):
    return problems.seeded(2, n, 11, 16, 0, solver="cg", eps=eps, end_step=steps, name="refine_small")


@pytest.fixture(scope="module")
def oracle_steps(oracle_lib):
    cfg, states = read_config(_problem(eps=1e-28).tea_in(), 2)
    return oracle_lib.run(cfg, states)


@pytest.mark.parametrize("precision", [64, 32])
def test_refine_reaches_residual_and_matches_oracle(precision, oracle_steps):
    h = Host(_problem().tea_in(), 2)
    try:
        for tt, ref in enumerate(oracle_steps):
            r = h.refine_step(tt, REL_TOL, precision)
            assert r.converged, (precision, tt, r)
            assert 0.0 < r.rel_residual <= REL_TOL
            assert r.iterations > 0 and r.residual_updates >= 1
            vol, mass, ie, temp = r.summary
            assert vol == ref.summary[0] and mass == ref.summary[1]
            assert ie == pytest.approx(ref.summary[2], rel=1e-14)
            assert abs(temp / ref.summary[3] - 1.0) < TEMP_RTOL, (precision, tt, temp, ref.summary[3])
    finally:
        h.finalise()


def test_fp32_and_fp64_forms_agree_and_fp32_updates_residual():
    a, b = Host(_problem().tea_in(), 2), Host(_problem().tea_in(), 2)
    try:
        for tt in range(3):
            r64 = a.refine_step(tt, REL_TOL, 64)
            r32 = b.refine_step(tt, REL_TOL, 32)
            # several FP64 residual replacements over ten decades of reduction
            assert r32.residual_updates >= 5
            # the FP32-stored CG needs at most a modest number of extra iterations
            assert r32.iterations <= 1.5 * r64.iterations + 20, (r32.iterations, r64.iterations)
            assert abs(r32.summary[3] / r64.summary[3] - 1.0) < TEMP_RTOL
            ua, ub = a.download("u"), b.download("u")
            hd = 2
            ia, ib = ua[hd:-hd, hd:-hd], ub[hd:-hd, hd:-hd]
            assert np.linalg.norm(ia - ib) / np.linalg.norm(ia) < 1e-8
    finally:
        a.finalise()
        b.finalise()


def test_refine_rejects_bad_arguments():
    h = Host(_problem(steps=1).tea_in(), 2)
    try:
        with pytest.raises(Exception):
            h.refine_step(0, REL_TOL, 16)
    finally:
        h.finalise()


# Forward-error bound of a solve stopped at relative residual REL_TOL:
# |du|/|u| <= cond(A) * REL_TOL. The oracle's PPCG run of this deck estimates
# eigmax / eigmin = 672 / 1.18 (Lanczos, with the 5% margins), so cond < 600.
TEMP_RTOL_BOUND = 600 * REL_TOL


def _ppcg_problem(steps=3, **kw):
    return _problem(steps=steps).with_(solver="ppcg", name="refine_ppcg_small", **kw)


@pytest.mark.parametrize("precision,inner,error_switch", [(64, 10, False), (32, 10, False), (32, 1, False),
                                                          (64, 10, True)])
def test_refined_ppcg_reaches_residual_and_matches_oracle(precision, inner, error_switch, oracle_steps):
    """PPCG with FP64 refinement converges to the same solution as the oracle's
    tight CG (same operator), in fewer outer steps than CG takes trips."""
    p = _ppcg_problem(ppcg_inner_steps=inner, presteps=10, error_switch=error_switch)
    h, c = Host(p.tea_in(), 2), Host(_problem().tea_in(), 2)
    try:
        for tt, ref in enumerate(oracle_steps):
            r = h.refine_step(tt, REL_TOL, precision)
            rc = c.refine_step(tt, REL_TOL, precision, summary=False)
            assert r.converged, (precision, inner, tt, r)
            assert 0.0 < r.rel_residual <= REL_TOL
            assert r.residual_updates >= 1
            vol, mass, ie, temp = r.summary
            assert vol == ref.summary[0] and mass == ref.summary[1]
            assert abs(temp / ref.summary[3] - 1.0) < TEMP_RTOL_BOUND, (precision, inner, tt, temp, ref.summary[3])
            if inner == 10:
                # ten inner steps per outer step: far fewer outer steps than CG trips
                assert r.iterations < 0.6 * rc.iterations, (r.iterations, rc.iterations)
    finally:
        h.finalise()
        c.finalise()


def test_refined_ppcg_rejects_bad_inner_steps():
    h = Host(_ppcg_problem(steps=1, ppcg_inner_steps=0).tea_in(), 2)
    try:
        with pytest.raises(Exception):
            h.refine_step(0, REL_TOL, 32)
    finally:
        h.finalise()


@pytest.mark.parametrize("precision,inner", [(32, 2), (32, 6), (32, 7), (32, 12), (64, 10)])
def test_blocked_preconditioner_matches_one_step_chain(precision, inner):
    """The temporally blocked preconditioner (up to 5 inner steps per launch)
    against one launch per inner step. The fields are the same operations in
    the same order; only r.z is summed over another partition, so the runs
    may part in the last bits of beta: same CG phase, outer steps within 2,
    both at the residual bound, temp within TEMP_RTOL of each other."""
    p = _ppcg_problem(ppcg_inner_steps=inner, presteps=10)
    a, b = Host(p.tea_in(), 2), Host(p.tea_in(), 2)
    try:
        b.lib.tl2d_set_temporal_blocking(b.chunk, 0)
        for tt in range(3):
            ra = a.refine_step(tt, REL_TOL, precision)
            rb = b.refine_step(tt, REL_TOL, precision)
            assert ra.converged and rb.converged
            assert ra.cg_trips == rb.cg_trips
            assert abs(ra.iterations - rb.iterations) <= 2, (ra.iterations, rb.iterations)
            assert abs(ra.summary[3] / rb.summary[3] - 1.0) < TEMP_RTOL
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("precision,solver", [(32, "cg"), (64, "cg"), (32, "ppcg"), (64, "ppcg")])
def test_tma_sweeps_match_direct_loads(precision, solver):
    """The refinement sweeps fed by TMA row loads and the ones reading their
    operands directly give the same solve bit for bit (same tiles, rows and
    reduction partials), on a mesh of ragged tiles (600 = 2 x 256 + 88 FP32
    columns, 4 x 128 + 88 FP64) over three timesteps."""
    p = problems.seeded(2, (600, 157), 19, 8, 2, solver=solver, eps=1e-15, end_step=3, name="rftma")
    if solver == "ppcg":
        p = p.with_(presteps=10)
    a, b = Host(p.tea_in(), 2), Host(p.tea_in(), 2)
    try:
        b.lib.tl2d_set_tma(b.chunk, 0)
        for tt in range(3):
            ra = a.refine_step(tt, REL_TOL, precision)
            rb = b.refine_step(tt, REL_TOL, precision)
            assert (ra.iterations, ra.cg_trips, ra.residual_updates) == (rb.iterations, rb.cg_trips,
                                                                       rb.residual_updates)
            assert ra.rel_residual == rb.rel_residual
            assert ra.summary == rb.summary
    finally:
        a.finalise()
        b.finalise()
