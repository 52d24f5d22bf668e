"""Host-side check of the TMA ring protocol the staged sweeps share
(tealeaf_b200/csrc: k_cg_w_fused_tma, k_cg_ur_fused_tma in kernels2d.cuh;
k_pcg_ur_tma in pcg2d.cuh; walkt and k3_cg_ur_tma in kernels3d.cuh;
k_rf_w_tma and k_rf_ur_tma in rftma2d.cuh), and of the TMA-staged blocked
kernel (k_blocked_tma in blocked2d.cuh: one barrier, one region in flight).

Each kernel walks its rows (or z-planes) in blocks; before block b it
synchronises the block, one thread issues the stage kStages - 1 ahead into
the slot the previous occupant left, and every thread then waits on the
shared-memory barriers of the stages it reads. The simulation below replays that schedule for every
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
        # __syncthreads(); the issue of the stage stages - 1 ahead; the waits
        nxt = b + stages - 1
        if nxt < np_:
            issue(nxt, b)
        for s in waits_fn(b, np_):
            assert s in issued, "wait on a stage never issued (would hang)"
            slot = s % stages
            assert slot_of[slot] == s
            if s not in waited:
                uses[slot] = uses.get(slot, 0) + 1
                waited.add(s)
            # the kernel waits with parity (s // stages) & 1 on the slot's barrier
            assert (s // stages) == uses[slot] - 1
        for s in reads_fn(b):
            assert s in waited, "read of a stage not waited for"
            assert slot_of[s % stages] == s, "read of a slot already reissued"
            last_read[s] = b
    assert issued <= waited, "a copy may still be in flight when the block ends"
    return np_


def ceil_div(a, b):
    return -(-a // b)


def test_blocked_region_prefetch():
    """k_blocked_tma: one barrier; tile t's region is issued before the loop
    (t = first) or after every thread has read tile t - G's region (the
    block barrier in the tile function), and waited for with parity of the
    tile's ordinal; every issued region is waited for."""
    for ntiles in range(1, 40):
        for grid in range(1, 12):
            for b in range(min(grid, ntiles)):
                mine = list(range(b, ntiles, grid))
                issued, waited, reads_done = [mine[0]], [], set()
                phase = 0
                for n, t in enumerate(mine):
                    assert issued[-1] == t, "waiting for a region never issued (would hang)"
                    assert n % 2 == phase
                    waited.append(t)
                    reads_done.add(t)      # registers taken, block barrier passed
                    if n + 1 < len(mine):
                        assert t in reads_done   # the staging is free before it is reused
                        issued.append(mine[n + 1])
                    phase ^= 1
                assert issued == waited, "a region copy may still be in flight at exit"


@pytest.mark.parametrize("rows,stages", [(4, 3), (4, 4), (8, 3), (2, 5)])
def test_w_sweep_rings(rows, stages):
    # 2D CG w sweep and the refinement w sweep: stage b holds strip rows
    # j0-1+rows*b .. ; row block b (rows j0+rows*b ..) reads stages b and b+1
    for n in range(1, 300):
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


@pytest.mark.parametrize("rows,stages", [(4, 3), (4, 4), (2, 3), (2, 4)])
def test_pointwise_sweep_rings(rows, stages):
    # 2D / 3D / refinement u-r updates and the PCG u/r/z sweep: stage b holds
    # units rows*b .. ; trip b reads stage b
    for n in range(1, 300):
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


@pytest.mark.parametrize("steps", [1, 2])
def test_blocked3d_plane_ring(steps):
    """The region-plane ring of k3_blocked_tma (blocked3d.cuh): planes
    s_begin .. load_end - 1 staged kPf3 = 2 ahead into kRing3 = 5 slots (slot
    (p - s_begin) % 5, one barrier per slot); step s waits for plane s, then
    (after the barrier) issues plane s + 2, and reads planes s - steps .. s
    (level l reads plane s - l and, for kz, s - l + 1). Checked for every
    segment position and length: each read plane was issued and waited for
    and still holds its slot, each wait uses the slot's use count as parity,
    every issued plane is waited for."""
    R, PF, TB = 5, 2, 2
    for zlo, zhi in [(2, 2 + n) for n in range(1, 140)]:
        for Z0 in range(zlo, zhi, 64):
            Z1 = min(Z0 + 64, zhi)
            H = steps
            s_begin, s_end = max(Z0 - H, zlo), Z1 + H
            load_end = min(Z1 + H, zhi + 1)
            slot_of, uses, issued, waited = {}, [0] * R, set(), set()

            def issue(p):
                q = (p - s_begin) % R
                slot_of[q] = p
                issued.add(p)

            for p in range(s_begin, min(s_begin + PF, load_end)):
                issue(p)
            for s_ in range(s_begin, s_end):
                if s_ < load_end:
                    q = (s_ - s_begin) % R
                    assert slot_of.get(q) == s_
                    assert ((s_ - s_begin) // R) & 1 == uses[q] & 1
                    uses[q] += 1
                    waited.add(s_)
                # after the barrier: the issue two planes ahead
                if s_ + PF < load_end:
                    issue(s_ + PF)
                reads = set()
                if s_ < min(Z1 + H, zhi):
                    reads.add(s_)
                for l in range(1, H + 1):
                    z = s_ - l
                    if max(Z0 - H + l, zlo) <= z < min(Z1 + H - l, zhi):
                        reads |= {z, z + 1}
                for p in reads:
                    assert p in waited, (Z0, Z1, s_, p)
                    assert slot_of[(p - s_begin) % R] == p, (Z0, Z1, s_, p)
            assert issued == waited
            assert TB + 1 + PF == R
