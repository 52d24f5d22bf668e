"""The decomposed mesh through the B200 suite (tealeaf_b200.decomp.DistHost).

Two ranks run as processes sharing cuda:0: their kernels never wait on each
other, the faces cross as host buffers over gloo between run_* calls.

* Against the reference program's own two-rank runs (tests/golden/
  ref_ranks.json: its host built for several ranks, omp3 kernels): CG,
  Chebyshev, PPCG and Jacobi, iteration counts within one and summaries
  within 1e-10 (the GPU's per-chunk sums differ from the serial ones by
  rounding).
* Against the undivided solve of the same CG deck on the same GPU: the
  solution within 1e-10.
* The device-resident timestep refuses the decomposed chunk.
* The reference's own multi-rank host linked with the B200 library against
  the same host's omp3 two-rank runs.
"""
import datetime
import json
import socket
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from tealeaf_b200 import problems

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q, text, steps):
    try:
        import torch.distributed as dist
        from tealeaf_b200 import abi, decomp
        from tealeaf_b200.host import Host
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        h = decomp.DistHost(text, 2)
        out = [h.solve(tt) for tt in range(steps)]
        u = h.gather_interior("u")
        refused = None
        if world > 1:   # the library's own check, past DistHost's
            try:
                Host.solve_device(h, steps)
            except abi.SuiteError as exc:
                refused = str(exc)
        q.put((rank, ([(dict(r.iterations), list(r.summary)) for r in out], u, refused)))
        h.finalise()
        dist.barrier()
        dist.destroy_process_group()
    except Exception as exc:
        q.put((rank, "%s: %s" % (type(exc).__name__, exc)))


def _run(world, text, steps, timeout=240):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, text, steps)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        out = [q.get(timeout=timeout) for _ in range(world)]
    finally:
        for p in procs:
            p.join(timeout=timeout)
            if p.is_alive():
                p.kill()
    for r, payload in out:
        if isinstance(payload, str):
            pytest.fail("rank %d: %s" % (r, payload))
    return [payload for _, payload in sorted(out, key=lambda t: t[0])]


def _two_rank_cases():
    cases = json.loads((Path(__file__).resolve().parent / "golden" / "ref_ranks.json").read_text())
    return [c for c in cases if c["dims"] == 2 and c["ranks"] == 2]


@pytest.mark.parametrize("case", _two_rank_cases(), ids=lambda c: c["name"])
def test_two_ranks_on_one_gpu_match_the_reference_two_rank_run(case):
    res = _run(2, case["tea_in"], len(case["steps"]))
    for out, _, refused in res:
        assert refused is not None and "error 34" in refused and "four faces are external" in refused
        assert len(out) == len(case["steps"])
        for (its, summary), ref in zip(out, case["steps"]):
            assert its.keys() == ref["iterations"].keys()
            assert all(abs(its[k] - ref["iterations"][k]) <= 1 for k in its)
            assert summary == pytest.approx(ref["summary"], rel=1e-10)
    assert res[0][0] == res[1][0]


def test_two_ranks_on_one_gpu_match_the_undivided_solve():
    text = problems.seeded(2, (160, 128), 61, 3, 1, solver="cg", end_step=2, name="dg_cg").tea_in()
    (one, u1, _), = _run(1, text, 2)
    res = _run(2, text, 2)
    for out, u, _ in res:
        assert np.allclose(u, u1, rtol=1e-10, atol=0.0)
        for (its, summary), (its1, summary1) in zip(out, one):
            assert its.keys() == its1.keys()
            assert all(abs(its[k] - its1[k]) <= 1 for k in its)
            assert summary == pytest.approx(summary1, rel=1e-10)
    assert res[0][0] == res[1][0]


@pytest.mark.parametrize("case", _two_rank_cases(), ids=lambda c: c["name"])
def test_reference_multi_rank_host_on_the_b200_library(case):
    """The reference's own host built for several ranks (its comms over the
    MPI stand-in oracle/minimpi), linked with the B200 library instead of the
    omp3 suite: its remote_halo_driver packs into its own host buffers through
    run_pack_or_unpack. Two ranks sharing cuda:0 against the same host's omp3
    two-rank run: iteration counts within one, summaries within 1e-10."""
    from oracle.oracle import run_reference_ranks
    steps = run_reference_ranks(case["tea_in"], 2, 2, suite="b200", timeout=240)
    assert len(steps) == len(case["steps"])
    for s, ref in zip(steps, case["steps"]):
        assert s.iterations.keys() == ref["iterations"].keys()
        assert all(abs(s.iterations[k] - ref["iterations"][k]) <= 1 for k in s.iterations)
        assert s.summary == pytest.approx(ref["summary"], rel=1e-10)
