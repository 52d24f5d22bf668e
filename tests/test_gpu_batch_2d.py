"""Batched timesteps (tl2d_batch_*) on the B200.

Every problem of a batch of uneven sizes is stopped by its FP64 residual,
r.r < eps (1e-12, the reference's 2D stop test). Two checks per problem:

* against the oracle (the reference's CG, 2d/drivers/cg_driver.c, restated
  in oracle/tl_oracle.c) on the same tea.in: the oracle stops on the
  recursive residual, the batch on the true FP64 residual of an iteration
  whose vectors are stored in FP32. Both residual norms are below
  sqrt(eps) = 1e-6, and A = I + (positive semi-definite diffusion) has
  smallest eigenvalue >= 1, so the two solutions differ by at most 2e-6 in
  norm; temp = sum(V rho u) moves by at most that relative to its size
  (TEMP_RTOL = 1e-6 is checked). FP32 storage costs iterations: the batch
  needs at most 25 % + 10 more than the oracle (ITER_BAND), and never fewer
  than 75 % of them;
* against the same timestep solved alone by the FP64 device driver, with the
  same bounds.

vol, mass and ie do not depend on the solve and match exactly.
"""
import numpy as np
import pytest

from tealeaf_b200 import problems
from tealeaf_b200.batch import Batch
from tealeaf_b200.host import Host

pytestmark = pytest.mark.gpu

TEMP_RTOL = 1e-6


def ITER_BAND(ref_it):
    return 0.75 * ref_it - 1, 1.25 * ref_it + 10


def _oracle(prob, steps):
    from oracle.oracle import OracleLib
    from tealeaf_b200.config import read_config
    cfg, states = read_config(prob.with_(end_step=steps).tea_in(), 2)
    return OracleLib().run(cfg, states)


def _probs(count=6):
    return problems.batched_2d(count, seed=9, lo=40, hi=300, steps=2)


def _sequential(prob, steps):
    h = Host(prob.tea_in(), 2)
    try:
        out = []
        for tt in range(steps):
            r = h.solve_device(tt)
            out.append((r.iterations["CG"], r.summary))
        return out
    finally:
        h.finalise()


def test_batch_matches_sequential_fp64_solves():
    probs = _probs()
    b = Batch([p.tea_in() for p in probs])
    try:
        for tt in range(2):
            st = b.step()
            assert st.problems == len(probs) and st.converged == len(probs)
            assert st.graph == 1
            it, rr, conv = b.results()
            assert conv.all() and (rr < 1e-12).all()
            for k, (p, s) in enumerate(zip(probs, b.summaries())):
                ref_it, ref = _sequential(p, tt + 1)[tt]
                assert s[0] == ref[0] and s[1] == ref[1] and s[2] == ref[2]
                assert abs(s[3] / ref[3] - 1.0) < TEMP_RTOL, (k, tt, s[3], ref[3])
                # FP32 storage costs at most a few extra iterations here
                assert it[k] <= 1.25 * ref_it + 10, (k, it[k], ref_it)
    finally:
        b.close()


def test_batch_matches_the_oracle():
    probs = _probs()
    want = [_oracle(p, 2) for p in probs]
    b = Batch([p.tea_in() for p in probs])
    try:
        for tt in range(2):
            st = b.step()
            assert st.converged == len(probs)
            it, rr, conv = b.results()
            assert conv.all() and (rr < 1e-12).all()
            for k, s in enumerate(b.summaries()):
                ref = want[k][tt]
                for a, r in zip(s[:3], ref.summary[:3]):
                    assert a == pytest.approx(r, rel=1e-15), (k, tt)
                assert abs(s[3] / ref.summary[3] - 1.0) < TEMP_RTOL, (k, tt, s[3], ref.summary[3])
                lo, hi = ITER_BAND(ref.iterations["CG"])
                assert lo <= it[k] <= hi, (k, tt, it[k], ref.iterations["CG"])
    finally:
        b.close()


def test_autotuner_picks_a_candidate_and_step_still_converges():
    probs = _probs(4)
    b = Batch([p.tea_in() for p in probs])
    try:
        before = [h.download("energy") for h in b.hosts]
        cfg = b.tune(trial_iters=5)
        assert cfg["tile_rows"] in (-1, 4, 8, 16, 32, 64) and cfg["grid_blocks"] > 0
        for h, e in zip(b.hosts, before):   # tuning leaves the energy untouched
            assert np.array_equal(h.download("energy"), e)
        st = b.step()
        assert st.converged == len(probs) and st.tile_rows == cfg["tile_rows"]
    finally:
        b.close()


def test_batch_results_do_not_depend_on_the_grid():
    """Tiles are handed to whichever block asks first and blocks move between
    problems, but every dot product is summed from fixed per-tile partials
    in tile order: the same tile height gives bit-identical results for any
    grid size and any schedule."""
    probs = _probs(5)
    out = []
    for grid in (148, 0):
        b = Batch([p.tea_in() for p in probs], tile_rows=8, grid_blocks=grid)
        try:
            st = b.step()
            it, rr, conv = b.results()
            out.append((st.converged, it.copy(), rr.copy(), [h.download("energy") for h in b.hosts]))
        finally:
            b.close()
    (c0, it0, rr0, e0), (c1, it1, rr1, e1) = out
    assert c0 == c1 == len(probs)
    assert np.array_equal(it0, it1) and np.array_equal(rr0, rr1)
    for a, b_ in zip(e0, e1):
        assert np.array_equal(a, b_)


def test_batch_rejects_an_empty_batch():
    from tealeaf_b200 import abi
    lib = abi.load(2)
    handle = lib.tl2d_batch_create(None, None, 0, 0, 0)
    with pytest.raises(Exception):
        abi.check(lib, 2)
    assert not handle
