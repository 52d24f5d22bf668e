"""Generate the committed golden fixtures from the reference program.

Runs HERE only (it needs the reference sources to build ``oracle/_ref``):

    python tests/golden/make_golden.py            # small/medium cases
    python tests/golden/make_golden.py --big      # configuration-size cases (slow)
    python tests/golden/make_golden.py --big --only NAME[,NAME]   # regenerate some of them

Writes
  * ``layout_2d.txt`` / ``layout_3d.txt`` -- offsetof/sizeof of the reference
    Chunk/Settings/State structs (oracle/layout_probe.c compiled against the
    reference headers);
  * ``ref_runs.json`` / ``ref_runs_big.json`` -- per-step iteration counts and
    field summaries (vol, mass, ie, temp; %.17e) of the reference omp3 program
    (strict-IEEE build, oracle/build_ref.py) on seeded tea.in files, with the
    tea.in text itself so tests can replay it anywhere;
  * the reference's own known answers (2d/tea.problems, 3d/tea.problems) for
    the shipped geometry, next to the omp3 result for the same case.
"""
from __future__ import annotations

import json
import re
import subprocess
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from oracle.build_ref import OUT, REF, build_reference  # noqa: E402
from oracle.oracle import run_reference  # noqa: E402
from tealeaf_b200 import problems  # noqa: E402


def shipped_case(dims: int, n: int, steps: int):
    """The reference's shipped tea.in resized to n cells per side."""
    text = (REF / ("%dd" % dims) / "tea.in").read_text()
    for ax in "xyz"[:dims]:
        text = re.sub(r"%s_cells\s*=\s*\d+" % ax, "%s_cells = %d" % (ax, n), text)
    text = re.sub(r"end_step\s*=\s*\d+", "end_step = %d" % steps, text)
    expected = None
    for line in (REF / ("%dd" % dims) / "tea.problems").read_text().splitlines():
        parts = line.split()
        if not parts:
            continue
        cells = [int(v) for v in parts[:dims]]
        if cells == [n] * dims and int(parts[dims]) == steps:
            expected = float(parts[dims + 1])
    return text, expected


def small_cases():
    cases = []
    for n, steps in ((64, 1), (512, 20)):
        text, exp = shipped_case(2, n, steps)
        cases.append(dict(name="shipped_2d_%d_%d" % (n, steps), dims=2, tea_in=text, tea_problems=exp))
    for n in (25, 32):
        text, exp = shipped_case(3, n, 20)
        cases.append(dict(name="shipped_3d_%d_20" % n, dims=3, tea_in=text, tea_problems=exp))
    for solver in ("cg", "cheby", "ppcg"):
        p = problems.plain_2d(512, seed=1, steps=10, solver=solver)
        cases.append(dict(name="plain_2d_512_%s" % solver, dims=2, tea_in=p.tea_in()))
    for solver in ("cg", "cheby", "ppcg", "jacobi"):
        p = problems.seeded(2, (97, 61), 11, 3, 2, solver=solver, end_step=3, name="odd_2d")
        if solver == "jacobi":
            p = p.with_(eps=1e-10)
        cases.append(dict(name="odd_2d_97x61_%s" % solver, dims=2, tea_in=p.tea_in()))
    for solver in ("cg", "cheby", "ppcg", "jacobi"):
        p = problems.seeded(3, (40, 36, 28), 12, 3, 1, solver=solver, end_step=3, name="odd_3d")
        if solver == "cheby":
            p = p.with_(max_iters=600)   # the 3D Chebyshev stop test never fires (sqrt each trip)
        if solver == "jacobi":
            p = p.with_(eps=1e-6)
        cases.append(dict(name="odd_3d_40x36x28_%s" % solver, dims=3, tea_in=p.tea_in()))
    return cases


def big_cases():
    """The configuration sizes: the 4096^2 drop-in deck with each solver, the
    3D 256^3 deck of the adjoint configuration, and the reference's own known
    answers at their full sizes (2d/tea.problems:2-3, 3d/tea.problems:3-4).

    On the 4096^2 deck the reference's Chebyshev and PPCG do not reach eps
    1e-15 within 20000 iterations per step, and their CG presteps only bring
    the error below the switch threshold (1) after thousands of iterations.
    Their runs here use the reference's error switch instead (`errswitch`,
    epslim 1e30: the switch after CG_ITERS_FOR_EIGENVALUES = 20 CG trips,
    2d/drivers/cheby_driver.c:30-32) and are capped at max_iters 2000
    (Chebyshev) and 200 (PPCG), on both sides, so the reference run stays
    affordable and the comparison covers the CG presteps, the eigenvalue
    bounds, the Chebyshev coefficients and the capped Chebyshev / PPCG solve."""
    cases = []
    p = problems.dropin_2d(4096, seed=2, steps=2, solver="cg")
    cases.append(dict(name="dropin_2d_4096_cg_2steps", dims=2, tea_in=p.tea_in()))
    for solver, cap in (("cheby", 2000), ("ppcg", 200)):
        p = problems.dropin_2d(4096, seed=2, steps=2, solver=solver).with_(max_iters=cap, error_switch=True,
                                                                          eps_lim=1e30)
        cases.append(dict(name="dropin_2d_4096_%s_2steps" % solver, dims=2, tea_in=p.tea_in()))
    p = problems.adjoint_3d(256, seed=4, steps=2)
    cases.append(dict(name="adjoint_3d_256_cg_2steps", dims=3, tea_in=p.tea_in()))
    for n, steps in ((4096, 1), (1024, 20)):
        text, exp = shipped_case(2, n, steps)
        cases.append(dict(name="shipped_2d_%d_%d" % (n, steps), dims=2, tea_in=text, tea_problems=exp))
    for n, steps in ((64, 20), (256, 5)):
        text, exp = shipped_case(3, n, steps)
        cases.append(dict(name="shipped_3d_%d_%d" % (n, steps), dims=3, tea_in=text, tea_problems=exp))
    return cases


def known_answer_cases():
    """Known answers checked on the GPU only (no reference run is recorded:
    3d/tea.problems:5 is 256^3 over 20 steps, a long CPU run)."""
    text, exp = shipped_case(3, 256, 20)
    return [dict(name="shipped_3d_256_20", dims=3, tea_in=text, tea_problems=exp, steps=None,
                 generator="3d/tea.problems known answer only")]


def run_cases(cases, threads=8):
    out = []
    for c in cases:
        t0 = time.time()
        steps = run_reference(c["tea_in"], c["dims"], "omp3", threads=threads, timeout=24 * 3600)
        c = dict(c)
        c["steps"] = [dict(iterations=s.iterations, summary=["%.17e" % v for v in s.summary]) for s in steps]
        c["seconds"] = round(time.time() - t0, 3)
        c["generator"] = "oracle/_ref/harness%dd_omp3 (reference omp3, -ffp-contract=off), OMP_NUM_THREADS=%d" % (
            c["dims"], threads)
        print("%-36s %7.1fs  %s" % (c["name"], c["seconds"], c["steps"][-1]), flush=True)
        out.append(c)
    return out


def main():
    build_reference(with_b200=False)
    for dims in (2, 3):
        txt = subprocess.run([str(OUT / ("layout%dd" % dims))], capture_output=True, text=True, check=True).stdout
        (HERE / ("layout_%dd.txt" % dims)).write_text(txt)
    only = None
    if "--only" in sys.argv:
        only = set(sys.argv[sys.argv.index("--only") + 1].split(","))
    if "--big" in sys.argv:
        path = HERE / "ref_runs_big.json"
        if only:
            # regenerate the named cases in place, keep the others
            old = {c["name"]: c for c in json.loads(path.read_text())}
            for c in run_cases([c for c in big_cases() if c["name"] in only]):
                old[c["name"]] = c
            for c in known_answer_cases():
                old.setdefault(c["name"], c)
            order = [c["name"] for c in big_cases() + known_answer_cases()]
            cases = [old[n] for n in order if n in old]
        else:
            cases = run_cases(big_cases()) + known_answer_cases()
        path.write_text(json.dumps(cases, indent=1) + "\n")
    else:
        (HERE / "ref_runs.json").write_text(json.dumps(run_cases(small_cases()), indent=1) + "\n")


if __name__ == "__main__":
    main()
