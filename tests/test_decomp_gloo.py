"""The decomposed mesh (tealeaf_b200.decomp) on the CPU, gloo ranks over
127.0.0.1.

* decompose: every chunk as the reference's own decompose_field
  (2d/initialise.c:34-134, 3d/initialise.c:34-174, compiled from its sources)
  places it for 28 meshes; chunks that tile the mesh once, remainders to the
  first chunks, neighbours that face each other.
* FaceExchange: after one exchange every halo layer on an internal face
  holds the neighbour's interior cells, for 2D and 3D meshes and 2 to 4
  ranks, several fields per message; external faces and corners untouched.
* DistHost: whole timesteps of the reference drivers' sequence through
  run_*, each rank's kernels computed by the oracle's restatement of the
  reference kernels (tests/oracle_suites.py): one rank reproduces the
  oracle's own run bit for bit; 2 to 6 ranks reproduce the reference
  program's own run on as many ranks bit for bit, and the one-rank solve to
  the rounding of their split sums.
"""
import datetime
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tealeaf_b200 import decomp, problems
from tealeaf_b200.config import read_config


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _init(rank, world, port):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    return dist


def _run(target, world, args, timeout=300):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q) + tuple(args)) for r in range(world)]
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


# -- decompose -------------------------------------------------------------------------

def test_chunk_counts_follow_the_reference_search():
    assert decomp.chunk_counts((100, 100), 1) == (1, 1)
    assert decomp.chunk_counts((100, 100), 4) == (2, 2)
    assert decomp.chunk_counts((100, 100), 2) == (1, 2)     # a tie keeps the first factorisation
    assert decomp.chunk_counts((200, 100), 2) == (2, 1)
    assert decomp.chunk_counts((100, 200), 2) == (1, 2)
    assert decomp.chunk_counts((70, 10), 7) == (7, 1)
    assert decomp.chunk_counts((64, 32, 16), 8) == (4, 2, 1)
    assert decomp.chunk_counts((30, 30, 30), 8) == (2, 2, 2)
    assert decomp.chunk_counts((30, 30, 30), 2) == (1, 1, 2)


@pytest.mark.parametrize("cells,n", [((10, 7), 4), ((37, 23), 6), ((41, 3), 5), ((9, 8, 7), 12),
                                     ((40, 30, 20), 8), ((5, 5), 1), ((17, 13, 11), 3)])
def test_chunks_tile_the_mesh_and_face_each_other(cells, n):
    boxes = decomp.decompose(cells, n)
    counts = decomp.chunk_counts(cells, n)
    assert len(boxes) == n
    cover = np.zeros(cells[::-1], dtype=int)
    for b in boxes:
        cover[tuple(slice(l, h) for l, h in zip(b.lo[::-1], b.hi[::-1]))] += 1
        for f, nb in enumerate(b.neighbours):
            axis = f // 2
            if nb == decomp.EXTERNAL_FACE:
                assert b.lo[axis] == 0 if f % 2 == 0 else b.hi[axis] == cells[axis]
                continue
            o = boxes[nb]
            assert o.neighbours[f ^ 1] == b.index
            assert o.hi[axis] == b.lo[axis] if f % 2 == 0 else o.lo[axis] == b.hi[axis]
            for a in range(len(cells)):
                if a != axis:
                    assert (o.lo[a], o.hi[a]) == (b.lo[a], b.hi[a])
    assert (cover == 1).all()
    for a, (cnt, c) in enumerate(zip(counts, cells)):
        spans = sorted({(b.lo[a], b.cells[a]) for b in boxes})
        assert len(spans) == cnt
        widths = [w for _, w in spans]   # the first c % cnt chunks take one cell more
        assert widths == [c // cnt + 1] * (c % cnt) + [c // cnt] * (cnt - c % cnt)
        assert [l for l, _ in spans] == [sum(widths[:k]) for k in range(cnt)]


def test_decompose_matches_the_reference_decompose_field(golden_dir):
    """Every chunk of 28 meshes (2D and 3D, 1 to 27 ranks) as the reference's
    own decompose_field placed it (tests/golden/decompose_ref.json, made by
    tests/golden/make_decompose_golden.py from the reference sources)."""
    import json
    cases = json.loads((golden_dir / "decompose_ref.json").read_text())
    assert len(cases) == 28
    for c in cases:
        boxes = decomp.decompose(c["cells"], c["ranks"])
        got = [{"rank": b.index, "lo": list(b.lo), "cells": list(b.cells), "neighbours": list(b.neighbours)}
               for b in boxes]
        assert got == c["chunks"], (c["cells"], c["ranks"])


def test_more_chunks_than_cells_is_an_error():
    with pytest.raises(ValueError):
        decomp.decompose((3, 3), 16)
    with pytest.raises(ValueError):
        decomp.chunk_counts((8, 8), 0)


# -- FaceExchange -----------------------------------------------------------------------

def _tag(field, gz, gy, gx):
    return field * 0.5 + gx + 1000.0 * gy + 1.0e6 * gz


def _slabs(shape, hd, depth, face):
    """(pack slab, unpack slab) index tuples of one face, array order z, y, x."""
    dims = len(shape)
    axis = dims - 1 - face // 2
    n = shape[axis]
    inner = [slice(hd, s - hd) for s in shape]
    lo = face % 2 == 0
    pack, unpack = list(inner), list(inner)
    pack[axis] = slice(hd, hd + depth) if lo else slice(n - hd - depth, n - hd)
    unpack[axis] = slice(hd - depth, hd) if lo else slice(n - hd, n - hd + depth)
    return tuple(pack), tuple(unpack)


def _exchange_worker(rank, world, port, q, cells, hd, depth):
    try:
        import ctypes as C
        dist = _init(rank, world, port)
        box = decomp.decompose(cells, world)[rank]
        dims = len(cells)
        shape = tuple(c + 2 * hd for c in box.cells[::-1])
        fields = []
        for f in range(3):
            a = np.full(shape, np.nan)
            idx = np.indices(box.cells[::-1])
            g = [idx[k] + box.lo[::-1][k] for k in range(dims)]
            gz, gy, gx = ([np.zeros_like(g[0])] + g) if dims == 2 else g
            a[(slice(hd, -hd),) * dims] = _tag(f, gz, gy, gx)
            fields.append(a)

        def pack(face, d, field, address, is_pack):
            src, dst = _slabs(field.shape, hd, d, face)
            view = field[src] if is_pack else field[dst]
            buf = np.ctypeslib.as_array(C.cast(address, C.POINTER(C.c_double)), shape=(view.size,))
            if is_pack:
                buf[:] = view.ravel()
            else:
                field[dst] = buf.reshape(view.shape)

        ex = decomp.FaceExchange(box)
        assert ex.face_len(0, depth) == depth * int(np.prod(box.cells[1:]))
        ex.run(depth, fields, pack)
        bad = []
        for f, a in enumerate(fields):
            for face, nb in enumerate(box.neighbours):
                _, dst = _slabs(shape, hd, depth, face)
                got = a[dst]
                if nb == decomp.EXTERNAL_FACE:
                    if not np.isnan(got).all():
                        bad.append(("external face written", f, face))
                    continue
                coords = np.indices(shape)[(slice(None),) + dst]
                g = [coords[k] - hd + box.lo[::-1][k] for k in range(dims)]
                gz, gy, gx = ([np.zeros_like(g[0])] + g) if dims == 2 else g
                if not np.array_equal(got, _tag(f, gz, gy, gx)):
                    bad.append(("wrong halo", f, face))
            inside = np.zeros(shape, dtype=bool)   # the interior and the face slabs
            inside[(slice(hd, -hd),) * dims] = True
            for face in range(2 * dims):
                inside[_slabs(shape, hd, depth, face)[1]] = True
            if not np.isnan(a[~inside]).all():
                bad.append(("cells outside the face slabs written", f))
        q.put((rank, bad))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as exc:   # reported to the test, not swallowed
        q.put((rank, "%s: %s" % (type(exc).__name__, exc)))


@pytest.mark.parametrize("cells,world,hd,depth", [((12, 9), 2, 2, 1), ((12, 9), 4, 2, 2), ((13, 11), 3, 2, 2),
                                                  ((8, 7, 6), 2, 2, 2), ((8, 7, 6), 4, 2, 1)])
def test_face_exchange_fills_internal_halos(cells, world, hd, depth):
    for bad in _run(_exchange_worker, world, (cells, hd, depth)):
        assert bad == []


# -- DistHost ---------------------------------------------------------------------------

def _solve_worker(rank, world, port, q, jobs):
    """Solves every (deck, dims, steps) of `jobs` in turn on this rank's chunk."""
    try:
        dist = _init(rank, world, port)
        from oracle_suites import OracleSuite2D, OracleSuite3D
        results = []
        for text, dims, steps in jobs:
            h = decomp.DistHost(text, dims, lib=OracleSuite2D() if dims == 2 else OracleSuite3D())
            out = []
            for tt in range(steps):
                r = h.solve(tt)
                out.append((dict(r.iterations), list(r.summary), r.error))
            results.append((h.box, out, h.gather_interior("u")))
            h.finalise()
        q.put((rank, results))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as exc:
        q.put((rank, "%s: %s" % (type(exc).__name__, exc)))


def _solve(world, jobs):
    """Per job, every rank's (box, per-step results, gathered u)."""
    per_rank = _run(_solve_worker, world, (jobs,))
    return [[per_rank[r][k] for r in range(world)] for k in range(len(jobs))]


CASES = {
    (2, "cg"): problems.seeded(2, (48, 40), 51, 3, 1, solver="cg", end_step=2, name="d_cg").tea_in(),
    (2, "cheby"): problems.seeded(2, (48, 40), 52, 3, 1, solver="cheby", end_step=2, name="d_cheby").tea_in(),
    (2, "ppcg"): problems.seeded(2, (48, 40), 53, 3, 1, solver="ppcg", end_step=2, name="d_ppcg").tea_in(),
    (2, "jacobi"): problems.seeded(2, (24, 20), 54, 2, 1, solver="jacobi", end_step=1, name="d_jac").with_(
        max_iters=400).tea_in(),
    (3, "cg"): problems.seeded(3, (20, 16, 14), 55, 3, 1, solver="cg", end_step=2, name="d3_cg").tea_in(),
    (3, "cheby"): problems.seeded(3, (20, 16, 14), 56, 3, 1, solver="cheby", end_step=1, name="d3_ch").with_(
        max_iters=300).tea_in(),
    (3, "ppcg"): problems.seeded(3, (20, 16, 14), 57, 3, 1, solver="ppcg", end_step=1, name="d3_pp").tea_in(),
}
_ONE_RANK = {}


def _one_rank(dims, solver):
    """The one-rank solve of a deck; every deck's is run in one process, once."""
    if not _ONE_RANK:
        keys = list(CASES)
        jobs = [(CASES[k], k[0], read_config(CASES[k], k[0])[0].end_step) for k in keys]
        for k, res in zip(keys, _solve(1, jobs)):
            _ONE_RANK[k] = res[0]
    return _ONE_RANK[(dims, solver)]


@pytest.mark.parametrize("dims,solver", list(CASES))
def test_one_rank_reproduces_the_oracle_run(dims, solver, oracle_lib):
    text = CASES[(dims, solver)]
    cfg, states = read_config(text, dims)
    ref = oracle_lib.run(cfg, states)
    box, out, _ = _one_rank(dims, solver)
    assert box.neighbours == (-1,) * (2 * dims)
    for (its, summary, _), r in zip(out, ref):
        assert its == r.iterations
        assert summary == r.summary


def _reference_ranks():
    import json
    from pathlib import Path
    return json.loads((Path(__file__).resolve().parent / "golden" / "ref_ranks.json").read_text())


@pytest.mark.parametrize("name", ["r2_cg_odd_5ranks", "r3_ppcg_4ranks"])
def test_reference_multi_rank_harness_reproduces_its_fixture(name):
    """The MPI stand-in and its build, live: the reference's multi-rank
    harness rerun on a fixture's deck gives the fixture again."""
    from oracle.oracle import REF_DIR, run_reference_ranks
    case = next(c for c in _reference_ranks() if c["name"] == name)
    if not (REF_DIR / ("harness%dd_omp3_mpi" % case["dims"])).exists():
        pytest.skip("reference harnesses not built here")
    steps = run_reference_ranks(case["tea_in"], case["dims"], case["ranks"], timeout=120)
    assert [(s.iterations, s.summary) for s in steps] == [(r["iterations"], r["summary"]) for r in case["steps"]]


@pytest.mark.parametrize("world", sorted({c["ranks"] for c in _reference_ranks()}))
def test_ranks_reproduce_the_reference_multi_rank_run(world):
    """Bit for bit against the reference program run as the same number of
    ranks (its host built for several ranks over the MPI stand-in
    oracle/minimpi, omp3 kernels on one thread; tests/golden/ref_ranks.json
    from tests/golden/make_ranks_golden.py): the same chunks, faces, sums in
    rank order, and so the same iteration counts and summed summaries."""
    cases = [c for c in _reference_ranks() if c["ranks"] == world]
    results = _solve(world, [(c["tea_in"], c["dims"], len(c["steps"])) for c in cases])
    for case, per_rank in zip(cases, results):
        for _, out, _ in per_rank:
            assert len(out) == len(case["steps"]), case["name"]
            for (its, summary, _), ref in zip(out, case["steps"]):
                assert its == ref["iterations"], case["name"]
                assert summary == ref["summary"], case["name"]


@pytest.mark.parametrize("dims,solver,world", [(2, "cg", 3), (2, "cheby", 4), (3, "cg", 4)])
def test_ranks_reproduce_the_one_rank_solve(dims, solver, world):
    """Split sums differ from the one-rank sums by rounding only: iteration
    counts equal and summaries and the solution within 1e-11. (Not PPCG:
    the reference sums rro over the ranks a second time when it switches to
    PPCG, ppcg_driver.c:83, so its N-rank PPCG is not its one-rank PPCG.)"""
    text = CASES[(dims, solver)]
    cfg, _ = read_config(text, dims)
    _, one, u1 = _one_rank(dims, solver)
    res, = _solve(world, [(text, dims, cfg.end_step)])
    boxes = [b for b, _, _ in res]
    assert sorted(b.index for b in boxes) == list(range(world))
    assert sum(int(np.prod(b.cells)) for b in boxes) == u1.size
    for _, out, u in res:
        assert np.allclose(u, u1, rtol=1e-11, atol=0.0)
        for (its, summary, err), (its1, summary1, err1) in zip(out, one):
            assert its == its1
            assert summary == pytest.approx(summary1, rel=1e-11)
    # every rank holds the same reduced figures
    for _, out, _ in res[1:]:
        assert out == res[0][1]


def _group_worker(rank, world, port, q, jobs):
    """Ranks {0,1} and {2,3} form two process groups; each solves its job
    (deck, dims, steps) on its own group."""
    try:
        dist = _init(rank, world, port)
        from oracle_suites import OracleSuite2D, OracleSuite3D
        groups = [dist.new_group([0, 1]), dist.new_group([2, 3])]
        mine = rank // 2
        text, dims, steps = jobs[mine]
        h = decomp.DistHost(text, dims, group=groups[mine],
                            lib=OracleSuite2D() if dims == 2 else OracleSuite3D())
        out = []
        for tt in range(steps):
            r = h.solve(tt)
            out.append((dict(r.iterations), list(r.summary)))
        q.put((rank, (mine, h.rank, h.box.index, out)))
        h.finalise()
        dist.barrier()
        dist.destroy_process_group()
    except Exception as exc:
        q.put((rank, "%s: %s" % (type(exc).__name__, exc)))


def test_ranks_of_a_process_group_solve_on_their_own():
    """DistHost on a process group: group ranks own the chunks, faces go to
    the peers' global ranks, sums stay inside the group; two groups of two
    solving different decks at once each reproduce the reference's two-rank
    run of their deck bit for bit."""
    cases = [c for c in _reference_ranks() if c["name"] in ("r2_cg_2ranks", "r3_cg_2ranks")]
    assert len(cases) == 2
    res = _run(_group_worker, 4, ([(c["tea_in"], c["dims"], len(c["steps"])) for c in cases],))
    for rank, (mine, group_rank, chunk, out) in enumerate(res):
        assert mine == rank // 2 and group_rank == rank % 2 and chunk == group_rank
        ref = cases[mine]["steps"]
        assert [(o[0], o[1]) for o in out] == [(r["iterations"], r["summary"]) for r in ref]


def _leaver_worker(rank, world, port, q, text):
    """Rank 1 leaves after set-up; rank 0 starts a timestep, whose first face
    exchange has no peer."""
    import datetime as dt
    import time
    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                                timeout=dt.timedelta(seconds=5))
        from oracle_suites import OracleSuite2D
        h = decomp.DistHost(text, 2, lib=OracleSuite2D())
        if rank == 1:
            q.put((rank, "left"))
            return
        t0 = time.monotonic()
        try:
            h.solve(0)
            q.put((rank, "completed"))
        except Exception as exc:   # the peer is gone: an error, not a hang
            q.put((rank, ("error", type(exc).__name__, time.monotonic() - t0)))
    except Exception as exc:
        q.put((rank, "%s: %s" % (type(exc).__name__, exc)))


def test_a_rank_that_leaves_ends_the_others_with_an_error():
    text = _reference_ranks()[0]["tea_in"]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaver_worker, args=(r, 2, port, q, text)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        out = dict(q.get(timeout=120) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert out[1] == "left"
    kind, _, seconds = out[0]
    assert kind == "error" and seconds < 60
