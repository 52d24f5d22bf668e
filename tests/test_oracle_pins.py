"""Pins the oracle (the C restatement in oracle/tl_oracle.c) before it is trusted.

* Against the reference's OWN known answers: 2d/tea.problems and
  3d/tea.problems (final temperature, 1e-5 relative, the reference's
  tolerance, 2d/drivers/field_summary_driver.c:43-51).
* Against the reference omp3 program run on seeded inputs (golden fixtures,
  tests/golden/ref_runs.json): per-step iteration counts exactly, field
  summaries within 1e-12 relative.
"""
import json
from pathlib import Path

import pytest

from tealeaf_b200.config import read_config

GOLDEN = Path(__file__).resolve().parent / "golden"
RTOL = 1e-12


def cases():
    return {c["name"]: c for c in json.loads((GOLDEN / "ref_runs.json").read_text())}


# Cases the serial oracle finishes in seconds.
PINNED = ["shipped_2d_64_1", "shipped_3d_25_20", "shipped_3d_32_20",
          "odd_2d_97x61_cg", "odd_2d_97x61_cheby", "odd_2d_97x61_ppcg", "odd_2d_97x61_jacobi",
          "odd_3d_40x36x28_cg", "odd_3d_40x36x28_cheby", "odd_3d_40x36x28_ppcg", "odd_3d_40x36x28_jacobi",
          "plain_2d_512_cg"]


@pytest.mark.parametrize("name", PINNED)
def test_oracle_matches_reference_program(name, oracle_lib):
    c = cases()[name]
    cfg, states = read_config(c["tea_in"], c["dims"])
    steps = oracle_lib.run(cfg, states)
    assert len(steps) == len(c["steps"])
    for n, (s, g) in enumerate(zip(steps, c["steps"])):
        assert s.iterations == g["iterations"], "step %d" % (n + 1)
        for a, b in zip(s.summary, g["summary"]):
            assert a == pytest.approx(float(b), rel=RTOL), "step %d" % (n + 1)


@pytest.mark.parametrize("name", ["shipped_2d_64_1", "shipped_3d_25_20", "shipped_3d_32_20"])
def test_oracle_reproduces_tea_problems(name, oracle_lib):
    c = cases()[name]
    assert c["tea_problems"] is not None
    cfg, states = read_config(c["tea_in"], c["dims"])
    temp = oracle_lib.run(cfg, states)[-1].summary[3]
    assert abs(100.0 * (temp / c["tea_problems"]) - 100.0) < 0.001


def test_eigenvalue_and_chebyshev_helpers(oracle_lib):
    """The Lanczos/QL bounds and the iteration estimate agree between the
    oracle's C and the Python host's restatement (same libm for logf/roundf)."""
    import ctypes as C

    from tealeaf_b200.host import cheby_est_iterations, eigenvalue_bounds
    alphas = [0.9 / (1.0 + 0.01 * i) for i in range(25)]
    betas = [0.5 * (0.97 ** i) for i in range(25)]
    lo, hi = eigenvalue_bounds(alphas, betas, 25)
    a = (C.c_double * 25)(*alphas)
    b = (C.c_double * 25)(*betas)
    olo, ohi = C.c_double(), C.c_double()
    assert oracle_lib.o_eigenvalue_bounds(a, b, 25, C.byref(olo), C.byref(ohi)) == 0
    assert (lo, hi) == (olo.value, ohi.value)
    for err, bb in ((1e-3, 10.0), (3e-6, 2.5e2), (0.7, 1e4)):
        assert cheby_est_iterations(lo, hi, err, bb) == oracle_lib.o_cheby_est_iterations(lo, hi, err, bb)
