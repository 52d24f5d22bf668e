"""Jacobi-preconditioned CG (2D): jac_diag and jac_block (blocks of 4 rows).

The reference documents both preconditioners (README.md:127-133) without a C
implementation, so the oracle's restatement (oracle/tl_oracle.c,
o2_precond_factor, o2_precond and oc_pcg) is pinned here on its own terms
first: its z solves M z = r for the stated M exactly (to rounding), and PCG
needs fewer iterations than CG on the same deck. The GPU tests then hold the device-resident PCG to the oracle:
per-step iteration counts equal, field summaries within 1e-12 relative.
"""
import ctypes as C

import numpy as np
import pytest

from tealeaf_b200 import problems
from tealeaf_b200.config import read_config

P = C.POINTER(C.c_double)


def ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P)


def _mesh(x, y, seed):
    rng = np.random.default_rng(seed)
    kx = rng.uniform(0.01, 3.0, (y, x))
    ky = rng.uniform(0.01, 3.0, (y, x))
    r = rng.normal(size=(y, x))
    return kx, ky, r


@pytest.mark.parametrize("ny", [12, 13, 14, 15])
def test_oracle_block_solve_satisfies_the_blocks(oracle_lib, ny):
    """jac_block: per column, each 4-row block (the last one shorter when the
    interior height is not a multiple of 4) solves its tridiagonal system."""
    hd, nx = 2, 9
    x, y = nx + 2 * hd, ny + 2 * hd
    kx, ky, r = _mesh(x, y, ny)
    z, mi = np.zeros((y, x)), np.zeros((y, x))
    oracle_lib.o2_precond_factor(x, y, hd, 2, ptr(kx), ptr(ky), ptr(mi))
    oracle_lib.o2_precond(x, y, hd, 2, ptr(ky), ptr(mi), ptr(r), ptr(z))
    for k in range(hd, x - hd):
        for jb in range(hd, y - hd, 4):
            m = min(4, y - hd - jb)
            rows = range(jb, jb + m)
            T = np.zeros((m, m))
            for q, j in enumerate(rows):
                T[q, q] = 1.0 + (kx[j, k + 1] + kx[j, k]) + (ky[j + 1, k] + ky[j, k])
                if q > 0:
                    T[q, q - 1] = T[q - 1, q] = -ky[j, k]
            zb = np.array([z[j, k] for j in rows])
            rb = np.array([r[j, k] for j in rows])
            assert np.allclose(T @ zb, rb, rtol=1e-13, atol=1e-13)
    # the halo is left alone
    assert not z[:hd].any() and not z[:, :hd].any()


def test_oracle_diag_solve_is_the_diagonal(oracle_lib):
    hd, nx, ny = 2, 7, 6
    x, y = nx + 2 * hd, ny + 2 * hd
    kx, ky, r = _mesh(x, y, 3)
    z, mi = np.zeros((y, x)), np.zeros((y, x))
    oracle_lib.o2_precond_factor(x, y, hd, 1, ptr(kx), ptr(ky), ptr(mi))
    oracle_lib.o2_precond(x, y, hd, 1, ptr(ky), ptr(mi), ptr(r), ptr(z))
    sl = (slice(hd, y - hd), slice(hd, x - hd))
    d = 1.0 + (kx[hd:y - hd, hd + 1:x - hd + 1] + kx[sl]) + (ky[hd + 1:y - hd + 1, hd:x - hd] + ky[sl])
    assert np.array_equal(mi[sl], 1.0 / d)      # the reference cuda kernel's mi = 1 / diag(A)
    assert np.array_equal(z[sl], (1.0 / d) * r[sl])


def test_oracle_pcg_converges_in_fewer_iterations(oracle_lib):
    base = problems.plain_2d(96, seed=21, steps=1, solver="cg")
    its = {}
    for pc in ("none", "jac_diag", "jac_block"):
        cfg, states = read_config(base.with_(preconditioner=pc).tea_in(), 2)
        res = oracle_lib.run(cfg, states)
        its[pc] = res[0].iterations["CG"]
        plain_cfg, _ = read_config(base.tea_in(), 2)
    want = oracle_lib.run(plain_cfg, states)[0].summary
    assert its["jac_block"] < its["jac_diag"] <= its["none"], its
    # the same solution to the eps the stop test allows (temp within 1e-9)
    for pc in ("jac_diag", "jac_block"):
        cfg, states = read_config(base.with_(preconditioner=pc).tea_in(), 2)
        got = oracle_lib.run(cfg, states)[0].summary
        assert got[3] == pytest.approx(want[3], rel=1e-9)


CASES = [("odd", (97, 61), 3), ("odd", (130, 77), 2), ("plain", (256, 256), 2)]


@pytest.mark.gpu
@pytest.mark.parametrize("pc", ["jac_diag", "jac_block"])
@pytest.mark.parametrize("kind,cells,steps", CASES)
def test_device_pcg_matches_the_oracle(oracle_lib, pc, kind, cells, steps):
    from tealeaf_b200.host import Host
    prob = problems.seeded(2, cells, 31, 4, 2, solver="cg", end_step=steps, name="pcg").with_(preconditioner=pc)
    text = prob.tea_in()
    cfg, states = read_config(text, 2)
    want = oracle_lib.run(cfg, states)
    h = Host(text, dims=2)
    try:
        got = h.run_device()
    finally:
        h.finalise()
    for n, (g, w) in enumerate(zip(got, want)):
        assert g.iterations == w.iterations, (pc, cells, n)
        for a, b in zip(g.summary, w.summary):
            assert a == pytest.approx(b, rel=1e-12), (pc, cells, n)


@pytest.mark.gpu
def test_preconditioner_setter_rejects_unknown_types():
    from tealeaf_b200 import abi
    from tealeaf_b200.host import Host
    h = Host(problems.plain_2d(32, seed=3, steps=1).tea_in(), dims=2)
    try:
        assert h.lib.tl2d_set_preconditioner(C.byref(h.chunk), 3) == 37
        with pytest.raises(abi.SuiteError, match="jac_block"):
            abi.check(h.lib, 2)
    finally:
        h.finalise()


@pytest.mark.gpu
@pytest.mark.parametrize("pc", ["jac_diag", "jac_block"])
def test_tma_fed_pcg_sweep_is_bit_identical(pc):
    """The TMA-fed u/r/z sweep (k_pcg_ur_tma) and the per-thread-load one
    (k_pcg_ur, tl2d_set_tma(0)) give the same counts, summaries and fields."""
    from tealeaf_b200.host import Host
    prob = problems.seeded(2, (300, 170), 33, 4, 2, solver="cg", end_step=2, name="pcgt").with_(preconditioner=pc)
    a, b = Host(prob.tea_in(), 2), Host(prob.tea_in(), 2)
    try:
        b.lib.tl2d_set_tma(C.byref(b.chunk), 0)
        for tt in range(2):
            ra, rb = a.solve_device(tt), b.solve_device(tt)
            assert ra.iterations == rb.iterations and ra.summary == rb.summary
            for f in ("u", "p", "r", "w", "energy", "mi"):
                assert np.array_equal(a.download(f), b.download(f)), (pc, tt, f)
    finally:
        a.finalise()
        b.finalise()
