"""Writes ref_ranks.json: the reference program's own multi-rank runs (its
host built for several ranks over oracle/minimpi, its omp3 kernels on one
thread each, oracle/build_ref.py), per case the deck, the rank count and,
per timestep, the master rank's iteration counts and summed field summary.

    python tests/golden/make_ranks_golden.py
"""
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from tealeaf_b200 import problems  # noqa: E402


def decks():
    s = problems.seeded
    return [
        ("r2_cg", 2, s(2, (48, 40), 51, 3, 1, solver="cg", end_step=2, name="r2_cg").tea_in(), (2, 3, 4)),
        ("r2_cheby", 2, s(2, (48, 40), 52, 3, 1, solver="cheby", end_step=2, name="r2_cheby").tea_in(), (2, 4)),
        ("r2_ppcg", 2, s(2, (48, 40), 53, 3, 1, solver="ppcg", end_step=2, name="r2_ppcg").tea_in(), (2, 3)),
        ("r2_jacobi", 2, s(2, (24, 20), 54, 2, 1, solver="jacobi", end_step=1, name="r2_jac").with_(
            max_iters=400).tea_in(), (2, 3)),
        ("r2_cg_odd", 2, s(2, (61, 37), 58, 4, 2, solver="cg", end_step=2, name="r2_cg_odd").tea_in(), (5, 6)),
        ("r3_cg", 3, s(3, (20, 16, 14), 55, 3, 1, solver="cg", end_step=2, name="r3_cg").tea_in(), (2, 4)),
        ("r3_cheby", 3, s(3, (20, 16, 14), 56, 3, 1, solver="cheby", end_step=1, name="r3_ch").with_(
            max_iters=300).tea_in(), (3,)),
        ("r3_ppcg", 3, s(3, (20, 16, 14), 57, 3, 1, solver="ppcg", end_step=1, name="r3_pp").tea_in(), (4,)),
    ]


def main():
    from oracle.build_ref import build_reference
    from oracle.oracle import run_reference_ranks
    build_reference(with_b200=False)
    out = []
    for name, dims, text, worlds in decks():
        for world in worlds:
            steps = run_reference_ranks(text, dims, world)
            out.append({"name": "%s_%dranks" % (name, world), "dims": dims, "ranks": world, "tea_in": text,
                        "steps": [{"iterations": s.iterations, "summary": s.summary} for s in steps]})
    (HERE / "ref_ranks.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote %d cases" % len(out))


if __name__ == "__main__":
    main()
