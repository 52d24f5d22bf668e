"""Host-side check of the TMA ring protocols of the staged sweeps
(tealeaf_b200/csrc: the streaming 2D CG sweeps k_cg_w_stream and
k_cg_ur_stream in stream2d.cuh; walkt and k3_cg_ur_tma in kernels3d.cuh;
k_rf_w_tma and k_rf_ur_tma in rftma2d.cuh; the blocked preconditioner is not
staged).

Streaming protocol (stream2d.cuh): a persistent block owns several strips
and their stages form one sequence. Before consuming stage q every thread
passes a block barrier; then one thread issues stages while fewer than
q + kStages have been issued (the newest, q + kStages - 1, goes into the slot
stage q-1 left), then every thread waits for stage q and reads only stage q
(rows needed later are carried in registers).

Per-strip protocol (the other kernels):

Each kernel walks its rows (or z-planes) in blocks; before block b it waits
on the shared-memory barriers of the stages it reads, synchronises the
block, and one thread issues the stage kStages - 1 ahead into the slot the
previous occupant left. The simulation below replays that schedule for every
strip length the kernels can see and checks, without a GPU, that:

* a stage is issued once, only after every read of the slot's previous
  occupant, and never into a slot the current block reads;
* every read waits on the right barrier phase (parity = uses of the slot);
* every issued stage is waited for before the kernel exits, so no copy is
  still in flight into the block's shared memory when the block ends;
* every row (plane) a block needs lies in a stage it waited for.
"""
import pytest


def simulate(n_units, rows, stages, np_fn, loop_fn, reads_fn, waits_fn):
    """Replays one block. n_units: rows (planes) of the strip; rows: units per
    stage; np_fn(n) -> stages that exist; loop_fn(n) -> loop trips; reads_fn(b)
    -> stages read in trip b; waits_fn(b, np) -> stages waited in trip b."""
    np_ = np_fn(n_units)
    slot_of = {}                 # slot -> stage occupying it
    issued, waited = set(), set()
    last_read = {}               # stage -> last trip that read it
    uses = {}                    # slot -> completed barrier phases

    def issue(stage, trip):
        assert stage not in issued, "stage issued twice"
        slot = stage % stages
        prev = slot_of.get(slot)
        if prev is not None:
            # the previous occupant is read no more from this trip on
            assert last_read.get(prev, -1) < trip, "slot overwritten while still read"
            assert prev in waited, "slot reused before its copy was waited for"
        slot_of[slot] = stage
        issued.add(stage)

    # prologue (one thread): the first stages - 1 stages
    for b in range(min(stages - 1, np_)):
        issue(b, -1)
    for b in range(loop_fn(n_units)):
        for s in waits_fn(b, np_):
            assert s in issued, "wait on a stage never issued (would hang)"
            slot = s % stages
            assert slot_of[slot] == s
            if s not in waited:
                uses[slot] = uses.get(slot, 0) + 1
                waited.add(s)
            # the kernel waits with parity (s // stages) & 1 on the slot's barrier
            assert (s // stages) == uses[slot] - 1
        # __syncthreads(); then the issue of the stage stages - 1 ahead
        nxt = b + stages - 1
        if nxt < np_:
            issue(nxt, b)
        for s in reads_fn(b):
            assert s in waited, "read of a stage not waited for"
            assert slot_of[s % stages] == s, "read of a slot already reissued"
            last_read[s] = b
    assert issued <= waited, "a copy may still be in flight when the block ends"
    return np_


def ceil_div(a, b):
    return -(-a // b)


def simulate_stream(strip_stage_counts, stages):
    """Replays one persistent block of the streaming protocol over strips
    with the given stage counts; returns the stages consumed."""
    total = sum(strip_stage_counts)
    slot_of, issued, waited, uses = {}, [], set(), {}
    done_reading = -1            # every stage <= this one is read no more
    q = 0
    for np_ in strip_stage_counts:
        for _ in range(np_):
            done_reading = q - 1     # block barrier: stage q-1 was consumed by every thread
            while len(issued) < total and len(issued) < q + stages:
                st = len(issued)
                slot = st % stages
                prev = slot_of.get(slot)
                if prev is not None:
                    assert prev <= done_reading, "slot overwritten while still read"
                    assert prev in waited, "slot reused before its copy was waited for"
                slot_of[slot] = st
                issued.append(st)
            assert q in issued, "wait on a stage never issued (would hang)"
            slot = q % stages
            assert slot_of[slot] == q
            uses[slot] = uses.get(slot, 0) + 1
            waited.add(q)
            assert (q // stages) == uses[slot] - 1     # the wait parity the kernel uses
            q += 1
    assert set(issued) == waited, "a copy may still be in flight when the block ends"
    return q


@pytest.mark.parametrize("stages", [3, 4])
def test_streaming_rings(stages):
    rows = 4
    for n in range(1, 70):                     # rows of a full strip
        for last in (n, max(1, n // 3), 1):    # the grid's last row of strips may be shorter
            for nstrips in range(1, 6):
                lens = [n] * (nstrips - 1) + [last]
                # w sweep: rows j0-1 .. j1 of each strip; u/r update: rows j0 .. j1-1
                w_counts = [ceil_div(m + 2, rows) for m in lens]
                assert simulate_stream(w_counts, stages) == sum(w_counts)
                ur_counts = [ceil_div(m, rows) for m in lens]
                assert simulate_stream(ur_counts, stages) == sum(ur_counts)
                # every row a strip needs lies in one of its own stages
                for m, c in zip(lens, w_counts):
                    assert c * rows >= m + 2


@pytest.mark.parametrize("rows,stages", [(4, 3), (4, 4), (8, 3), (2, 5)])
def test_w_sweep_rings(rows, stages):
    # the refinement w sweep: stage b holds strip rows
    # j0-1+rows*b .. ; row block b (rows j0+rows*b ..) reads stages b and b+1
    for n in range(1, 200):
        def reads(b):
            out = set()
            for u in range(rows):
                j = b * rows + u            # row offset from j0
                if j >= n:
                    break
                t = j + 1                   # offset from the first staged row (j0 - 1)
                out.add(t // rows)          # the row itself (left / right ring cells)
                out.add((t + 1) // rows)    # its upper neighbour
                if b == 0 and u == 0:
                    out.add(0)              # the row below the strip
            return out
        simulate(n, rows, stages,
                 np_fn=lambda n: ceil_div(n + 2, rows),
                 loop_fn=lambda n: ceil_div(n, rows),
                 reads_fn=reads,
                 waits_fn=lambda b, np_: [b] + ([b + 1] if b + 1 < np_ else []))


@pytest.mark.parametrize("rows,stages", [(4, 3), (2, 3)])
def test_pointwise_sweep_rings(rows, stages):
    # 3D / refinement u-r updates: stage b holds units rows*b .. ; trip b reads stage b
    for n in range(1, 200):
        simulate(n, rows, stages,
                 np_fn=lambda n: ceil_div(n, rows),
                 loop_fn=lambda n: ceil_div(n, rows),
                 reads_fn=lambda b: {b},
                 waits_fn=lambda b, np_: [b])


def test_walkt_plane_ring():
    # 3D stencil walker: planes i0 .. i1 (i1 the front neighbour), plane q
    # computed from slots q and q+1, 4 stages
    for zr in range(1, 40):
        np_ = zr + 1
        simulate(zr, 1, 4,
                 np_fn=lambda n: n + 1,
                 loop_fn=lambda n: n,
                 reads_fn=lambda q: {q, q + 1},
                 waits_fn=lambda q, np_: [q, q + 1])
        assert np_ >= 2
