"""Failure paths of the 2D suite on the B200, made without a GPU fault.

The reference's failures are die() calls (2d/shared.c:97-111): a message and
exit(1). The suite keeps that default and, in record mode (the Python loader
switches it on), returns the error code and message to the caller instead.
These tests drive each failure on purpose and check what is reported:

* a bounded device wait that runs out: the shared-memory barrier wait of the
  TMA-fed sweeps, on a barrier that nothing completes (no copy in flight), and
  the persistent batch kernel's phase wait with a limit too short to be met;
  the kernel returns, the host reports the error, the context stays usable;
* host-side errors: max_iters above what the chunk was initialised with
  (error 32), a NaN in the density field, an iteration cap that stops the
  solve early.
"""
import math

import numpy as np
import pytest

from oracle.oracle import OracleLib
from tealeaf_b200 import abi, problems
from tealeaf_b200.batch import Batch
from tealeaf_b200.config import read_config
from tealeaf_b200.host import DriverError, Host

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _oracle_run(tea_in):
    cfg, states = read_config(tea_in, 2)
    return OracleLib().run(cfg, states)


def test_bounded_wait_gives_up_and_is_reported():
    prob = problems.plain_2d(64, seed=3, steps=1, solver="cg")
    h = Host(prob.tea_in(), dims=2)
    try:
        rc = h.lib.tl2d_check_bounded_wait(abi.C.byref(h.chunk), 1000)
        assert rc == 35
        with pytest.raises(abi.SuiteError, match="gave up after 1000 polls"):
            abi.check(h.lib, 2)
        # the chunk's wait-error word stays set: the next solve reports it too
        with pytest.raises(abi.SuiteError, match="error 35"):
            h.solve_device(0)
    finally:
        h.finalise()
    # the context is still usable: a fresh chunk solves and matches the oracle
    h = Host(prob.tea_in(), dims=2)
    try:
        got = h.run_device()
    finally:
        h.finalise()
    want = _oracle_run(prob.tea_in())
    assert got[0].iterations == want[0].iterations
    for a, b in zip(got[0].summary, want[0].summary):
        assert a == pytest.approx(b, rel=RTOL)


def test_bounded_wait_rejects_a_bad_limit():
    prob = problems.plain_2d(32, seed=3, steps=1, solver="cg")
    h = Host(prob.tea_in(), dims=2)
    try:
        assert h.lib.tl2d_check_bounded_wait(abi.C.byref(h.chunk), 0) == 36
        with pytest.raises(abi.SuiteError, match="polls must be"):
            abi.check(h.lib, 2)
    finally:
        h.finalise()


def test_batch_phase_wait_timeout_is_reported_and_the_batch_recovers():
    probs = problems.batched_2d(4, seed=11, lo=64, hi=200, steps=2)
    b = Batch([p.tea_in() for p in probs])
    try:
        b.set_wait_limit(1)          # one SM clock: the first phase wait runs out
        with pytest.raises(abi.SuiteError, match="phase wait of the persistent kernel timed out"):
            b.step()
        b.set_wait_limit(0)          # back to the default limit
        st = b.step()
        assert st.problems == len(probs) and st.converged == len(probs)
        it, rr, conv = b.results()
        assert conv.all() and (rr < 1e-12).all()
    finally:
        b.close()


def test_max_iters_above_the_initialised_tables_is_an_error():
    prob = problems.plain_2d(48, seed=5, steps=1, solver="cg").with_(max_iters=100)
    h = Host(prob.tea_in(), dims=2)
    try:
        h.settings.max_iters = 101
        with pytest.raises(abi.SuiteError, match="error 32: max_iters 101 exceeds"):
            h.solve_device(0)
        h.settings.max_iters = 100
        r = h.solve_device(0)          # the chunk is still usable
        assert r.iterations["CG"] > 0 and math.isfinite(r.summary[3])
    finally:
        h.finalise()


@pytest.mark.parametrize("solver", ["cg", "cheby", "ppcg"])
def test_iteration_cap_stops_like_the_oracle(solver):
    """max_iters far below convergence: the drivers stop at the cap
    (cg_driver.c:18, cheby_driver.c:24, ppcg_driver.c:22) with the same
    counts and summaries as the oracle, through both drivers."""
    prob = problems.plain_2d(128, seed=6, steps=2, solver=solver).with_(max_iters=45, presteps=10)
    want = _oracle_run(prob.tea_in())
    for path in ("device", "run"):
        h = Host(prob.tea_in(), dims=2)
        try:
            got = h.run_device() if path == "device" else h.run()
        finally:
            h.finalise()
        for g, w in zip(got, want):
            assert sum(g.iterations.values()) <= 45 + 1
            assert g.iterations == w.iterations, path
            for a, b in zip(g.summary, w.summary):
                assert a == pytest.approx(b, rel=1e-10 if solver == "ppcg" else RTOL), path


@pytest.mark.parametrize("path", ["device", "run"])
def test_nan_density_runs_to_the_cap_and_propagates(path):
    """A NaN uploaded into one density cell: the reference's stop test
    fabs(error) < eps is false for NaN (cg_driver.c:24), so the solve runs
    to max_iters and the temperature comes out NaN; nothing faults."""
    prob = problems.plain_2d(64, seed=7, steps=1, solver="cg").with_(max_iters=30)
    h = Host(prob.tea_in(), dims=2)
    try:
        d = h.download("density")
        hd = h.cfg.halo_depth
        d[hd + 10, hd + 12] = np.nan
        h.upload("density", d)
        r = h.solve_device(0) if path == "device" else h.solve(0)
        assert r.iterations["CG"] == 30
        assert math.isnan(r.error)
        assert math.isnan(r.summary[3])
        assert not math.isnan(r.summary[0])     # the volume does not depend on the solve
    finally:
        h.finalise()
