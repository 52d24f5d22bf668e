"""Writes decompose_ref.json: the reference's own decomposition of a set of
meshes over N ranks (decompose_field, compiled from the reference sources
with oracle/decompose_probe.c by oracle/build_ref.py into
oracle/_ref/decompose{2d,3d}). Each case lists, per rank, the chunk's
first cell and cell count along each axis and its neighbours.

    python tests/golden/make_decompose_golden.py
"""
import json
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

CASES_2D = [(10, 7, 4), (37, 23, 6), (41, 3, 5), (100, 100, 2), (100, 100, 4), (200, 100, 8), (64, 64, 16),
            (97, 61, 12), (13, 11, 7), (4096, 4096, 8), (1000, 10, 10), (33, 65, 9), (5, 5, 1), (48, 40, 3),
            (512, 512, 6), (7, 300, 5)]
CASES_3D = [(9, 8, 7, 12), (40, 30, 20, 8), (17, 13, 11, 3), (30, 30, 30, 8), (30, 30, 30, 2),
            (64, 32, 16, 8), (25, 25, 25, 27), (256, 256, 256, 8), (20, 16, 14, 4), (50, 10, 10, 6),
            (37, 19, 23, 12), (128, 64, 32, 16)]


def probe(dims, case):
    exe = REPO / "oracle" / "_ref" / ("decompose%dd" % dims)
    out = subprocess.run([str(exe)] + [str(v) for v in case], capture_output=True, text=True, check=True).stdout
    ranks = []
    for line in out.splitlines():
        v = [int(t) for t in line.split()]
        if dims == 2:
            r, left, right, bottom, top = v[:5]
            nb = v[5:9]
            ranks.append({"rank": r, "lo": [left, bottom], "cells": [right - left, top - bottom], "neighbours": nb})
        else:
            r, left, right, bottom, top, back = v[:6]
            nb = v[6:12]
            ranks.append({"rank": r, "lo": [left, bottom, back], "cells": [right - left, top - bottom, None],
                          "neighbours": nb})
    if dims == 3:   # z extent from the reference's own back planes: the front neighbour's, or the mesh end
        for c in ranks:
            f = c["neighbours"][5]
            c["cells"][2] = (ranks[f]["lo"][2] if f >= 0 else case[2]) - c["lo"][2]
    return ranks


def main():
    from oracle.build_ref import build_reference
    build_reference(with_b200=False)
    cases = []
    for case in CASES_2D:
        cases.append({"cells": list(case[:2]), "ranks": case[2], "chunks": probe(2, case)})
    for case in CASES_3D:
        cases.append({"cells": list(case[:3]), "ranks": case[3], "chunks": probe(3, case)})
    (HERE / "decompose_ref.json").write_text(json.dumps(cases, indent=None, separators=(",", ":")) + "\n")
    print("wrote %d cases" % len(cases))


if __name__ == "__main__":
    main()
