"""The device-resident timestep (tl2d_solve_step) on the B200.

* Same answers as the reference omp3 program (golden fixtures): per-step
  iteration counts exactly, field summaries within 1e-12.
* Same memory state as the kernel-interface path driven like the reference
  drivers: after every timestep every field is bit-identical (both paths use
  the same sweeps, launch shapes and reduction trees).
"""
import json

import numpy as np
import pytest

from tealeaf_b200 import problems
from tealeaf_b200.host import Host

pytestmark = pytest.mark.gpu

RTOL = 1e-12
FIELDS = ("u", "u0", "p", "r", "w", "kx", "ky", "sd", "energy", "density")


def golden(golden_dir):
    return {c["name"]: c for c in json.loads((golden_dir / "ref_runs.json").read_text())}


@pytest.mark.parametrize("name", ["shipped_2d_64_1", "odd_2d_97x61_cg", "odd_2d_97x61_cheby",
                                  "odd_2d_97x61_ppcg", "plain_2d_512_cg", "plain_2d_512_cheby"])
def test_device_driver_matches_reference(name, golden_dir):
    g = golden(golden_dir)[name]
    h = Host(g["tea_in"], dims=2)
    try:
        steps = h.run_device()
    finally:
        h.finalise()
    assert len(steps) == len(g["steps"])
    for n, (s, ref) in enumerate(zip(steps, g["steps"])):
        assert s.iterations == ref["iterations"], "step %d" % (n + 1)
        for a, b in zip(s.summary, ref["summary"]):
            assert a == pytest.approx(float(b), rel=RTOL), "step %d" % (n + 1)


@pytest.mark.parametrize("solver", ["cg", "cheby", "ppcg"])
def test_device_driver_memory_state_equals_run_path(solver):
    prob = problems.seeded(2, (71, 53), 31, 3, 2, solver=solver, end_step=2, name="state")
    text = prob.tea_in()
    a, b = Host(text, 2), Host(text, 2)
    try:
        for tt in range(2):
            ra = a.solve(tt)
            rb = b.solve_device(tt)
            assert ra.iterations == rb.iterations
            assert ra.summary == rb.summary
            assert ra.exact_error == rb.exact_error
            for f in FIELDS:
                assert np.array_equal(a.download(f), b.download(f)), (solver, tt, f)
            flags_a = [a.flags[i] for i in range(6)]
            flags_b = [b.flags[i] for i in range(6)]
            assert flags_a == flags_b
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("solver", ["cheby", "ppcg"])
def test_temporal_blocking_is_bit_identical(solver):
    """Chebyshev trips / PPCG inner steps run temporally blocked in shared
    memory give the same memory state, bit for bit, as one launch per step,
    on a mesh of many tiles with ragged edges."""
    prob = problems.seeded(2, (203, 141), 17, 5, 2, solver=solver, end_step=2, name="blocked")
    text = prob.tea_in()
    a, b = Host(text, 2), Host(text, 2)
    try:
        b.lib.tl2d_set_temporal_blocking(b.chunk, 0)
        for tt in range(2):
            ra = a.solve_device(tt)
            rb = b.solve_device(tt)
            assert ra.iterations == rb.iterations
            assert ra.summary == rb.summary
            for f in FIELDS:
                assert np.array_equal(a.download(f), b.download(f)), (solver, tt, f)
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("solver,path", [("cg", "device"), ("cg", "run"), ("ppcg", "device")])
def test_tma_w_sweep_is_bit_identical(solver, path):
    """The CG w sweep fed by TMA row loads (even row length: 300 + 4) and the
    one reading its operands directly give the same memory state, bit for
    bit (same strips, rows and reduction partials), on a mesh with ragged
    strips (300 = 2 x 128 + 44 columns) and a ragged last block row."""
    prob = problems.seeded(2, (300, 157), 23, 5, 2, solver=solver, end_step=2, name="tma2")
    text = prob.tea_in()
    a, b = Host(text, 2), Host(text, 2)
    try:
        b.lib.tl2d_set_tma(b.chunk, 0)
        for tt in range(2):
            ra = a.solve_device(tt) if path == "device" else a.solve(tt)
            rb = b.solve_device(tt) if path == "device" else b.solve(tt)
            assert ra.iterations == rb.iterations
            assert ra.summary == rb.summary
            for f in FIELDS:
                assert np.array_equal(a.download(f), b.download(f)), (solver, path, tt, f)
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("inner", [10, 7, 1])
def test_run_path_ppcg_queue_is_bit_identical(inner):
    """Through run_* (the reference drivers' call sequence), the PPCG inner
    steps deferred and run temporally blocked give the same memory state, bit
    for bit, as one launch per call (temporal blocking off), for inner-step
    counts that fill, split and underfill the 5-step blocks."""
    prob = problems.seeded(2, (203, 141), 17, 5, 2, solver="ppcg", end_step=2, name="pq").with_(
        ppcg_inner_steps=inner)
    text = prob.tea_in()
    a, b = Host(text, 2), Host(text, 2)
    try:
        b.lib.tl2d_set_temporal_blocking(b.chunk, 0)
        for tt in range(2):
            ra = a.solve(tt)
            rb = b.solve(tt)
            assert ra.iterations == rb.iterations
            assert ra.summary == rb.summary
            assert ra.exact_error == rb.exact_error
            for f in FIELDS:
                assert np.array_equal(a.download(f), b.download(f)), (inner, tt, f)
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("cap", [None, 183, 261])
def test_run_path_cheby_queue_is_bit_identical(cap):
    """Through run_* (the reference drivers' call sequence), the Chebyshev
    trips deferred and run temporally blocked (each trip ending with its
    u += p) give the same iteration counts, summaries and memory state, bit
    for bit, as one launch per call; capped runs stop the queue at trip counts
    that split the 5-trip blocks and between norm checks."""
    prob = problems.seeded(2, (203, 141), 19, 5, 2, solver="cheby", end_step=2, name="cq")
    if cap:
        prob = prob.with_(max_iters=cap)
    text = prob.tea_in()
    a, b = Host(text, 2), Host(text, 2)
    try:
        b.lib.tl2d_set_temporal_blocking(b.chunk, 0)
        for tt in range(2):
            ra = a.solve(tt)
            rb = b.solve(tt)
            assert ra.iterations == rb.iterations
            assert ra.iterations.get("Cheby", 0) > 0
            assert ra.summary == rb.summary
            assert ra.exact_error == rb.exact_error
            for f in FIELDS:
                assert np.array_equal(a.download(f), b.download(f)), (cap, tt, f)
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("dims,trips", [((203, 141), 1), ((203, 141), 5), ((204, 142), 7)])
def test_cg_sweeps_run_the_deferred_trips_first(dims, trips, cheby_then_cg_sweeps):
    """Chebyshev trips still queued when run_cg_calc_w, run_cg_calc_ur and
    run_cg_calc_p are called run before them: the sweeps' dot products and
    the memory state match, bit for bit, a chunk that ran every trip at
    once."""
    text = problems.seeded(2, dims, 43, 5, 2, solver="cheby", end_step=1, name="qcg2").tea_in()
    a, b = Host(text, 2), Host(text, 2)
    try:
        b.lib.tl2d_set_temporal_blocking(b.chunk, 0)
        ra = cheby_then_cg_sweeps(a, trips)
        rb = cheby_then_cg_sweeps(b, trips)
        assert ra == rb
        for f in FIELDS:
            assert np.array_equal(a.download(f), b.download(f)), (dims, trips, f)
    finally:
        a.finalise()
        b.finalise()
