"""Parity at the configuration sizes (B200 only).

The golden runs in ``golden/ref_runs_big.json`` come from the reference omp3
program (strict-IEEE build) on:
  * the 4096^2 drop-in deck (8 rectangles + 4 circles, reciprocal
    conductivity, eps 1e-15, dt 0.004), two timesteps each with CG,
    Chebyshev (30 presteps) and PPCG (10 inner steps);
  * the 3D 256^3 deck of the adjoint configuration (6 boxes, CG), two steps;
  * the reference's shipped geometry at the sizes of its own known answers:
    2d/tea.problems:2 (4096^2, 1 step), :3 (1024^2, 20 steps),
    3d/tea.problems:3 (64^3, 20 steps), :4 (256^3, 5 steps); and :5 (256^3,
    20 steps), checked against the known answer alone.

Three paths drive the suite: the device-resident driver (tl2d_solve_step /
tl3d_solve_step), the Python mirror of the reference drivers over run_*, and
the reference's own C host and drivers linked with the B200 library. Per-step
iteration counts must be equal and the field summaries within 1e-12 relative
(the reference's known answers at their own 1e-5, field_summary_driver.c:43-51).

On the 4096^2 deck the reference's Chebyshev and PPCG do not reach eps 1e-15
within 20000 iterations per step, so those runs are capped at max_iters 2000
and 1000 on both sides (the cap is in the tea.in): the counts then pin the
CG presteps and the switch, and the summaries pin the capped solve.
"""
import json

import pytest

from oracle.oracle import harness_path, run_reference
from tealeaf_b200.host import Host

pytestmark = pytest.mark.gpu

RTOL = 1e-12          # field summaries against the reference program
KNOWN_ANSWER = 1e-5   # the reference's own check on the final temperature


def golden(golden_dir):
    return {c["name"]: c for c in json.loads((golden_dir / "ref_runs_big.json").read_text())}


def compare(steps, gold, rtol=RTOL):
    assert len(steps) == len(gold["steps"])
    for n, (s, g) in enumerate(zip(steps, gold["steps"])):
        assert s.iterations == g["iterations"], "step %d" % (n + 1)
        for a, b in zip(s.summary, g["summary"]):
            assert a == pytest.approx(float(b), rel=rtol), "step %d" % (n + 1)


def known_answer(steps, gold):
    exp = gold["tea_problems"]
    assert exp is not None
    temp = steps[-1].summary[3]
    assert abs(100.0 * (temp / exp) - 100.0) < 100.0 * KNOWN_ANSWER, (temp, exp)


def run_device(g):
    h = Host(g["tea_in"], dims=g["dims"])
    try:
        return h.run_device()
    finally:
        h.finalise()


def run_python_host(g):
    h = Host(g["tea_in"], dims=g["dims"])
    try:
        return h.run()
    finally:
        h.finalise()


DEVICE_CASES = ["dropin_2d_4096_cg_2steps", "dropin_2d_4096_cheby_2steps", "dropin_2d_4096_ppcg_2steps",
                "adjoint_3d_256_cg_2steps", "shipped_2d_4096_1", "shipped_2d_1024_20", "shipped_3d_64_20",
                "shipped_3d_256_5"]


@pytest.mark.parametrize("name", DEVICE_CASES)
def test_device_driver_at_configuration_sizes(name, golden_dir):
    g = golden(golden_dir)[name]
    steps = run_device(g)
    compare(steps, g)
    if g.get("tea_problems") is not None:
        known_answer(steps, g)


@pytest.mark.parametrize("name", ["dropin_2d_4096_cg_2steps", "dropin_2d_4096_ppcg_2steps",
                                  "adjoint_3d_256_cg_2steps", "shipped_2d_4096_1"])
def test_kernel_interface_at_configuration_sizes(name, golden_dir):
    """run_* driven by the Python mirror of the reference drivers."""
    g = golden(golden_dir)[name]
    steps = run_python_host(g)
    compare(steps, g)
    if g.get("tea_problems") is not None:
        known_answer(steps, g)


@pytest.mark.parametrize("name", ["dropin_2d_4096_cg_2steps", "dropin_2d_4096_cheby_2steps",
                                  "dropin_2d_4096_ppcg_2steps", "adjoint_3d_256_cg_2steps",
                                  "shipped_2d_1024_20"])
def test_reference_host_at_configuration_sizes(name, golden_dir):
    """The unchanged reference C host and drivers, linked with the B200 library."""
    g = golden(golden_dir)[name]
    if not harness_path(g["dims"], "b200").exists():
        pytest.skip("oracle/_ref/harness%dd_b200 not built" % g["dims"])
    steps = run_reference(g["tea_in"], dims=g["dims"], suite="b200")
    compare(steps, g)


def test_known_answer_3d_256_20_steps(golden_dir):
    """3d/tea.problems:5 -- 256^3 over 20 steps, final temperature at 1e-5."""
    g = golden(golden_dir)["shipped_3d_256_20"]
    known_answer(run_device(g), g)
