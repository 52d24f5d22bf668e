"""3D suite parity on the B200 (7-point stencil, 3d/kernel_interface.h).

* Element-wise: every 3D kernel through the C ABI against the oracle's
  restatement of the reference omp3 3D kernel on the same inputs; bit-exact
  for element-wise kernels, 1e-13 relative for dot products.
* Whole solves: the Python host mirror over run_*, the device-resident
  driver, and the reference's own C host linked with the B200 library,
  against the reference omp3 program (golden fixtures): iteration counts
  exactly, field summaries within 1e-12.
"""
import ctypes as C
import json

import numpy as np
import pytest

from oracle.oracle import OState, harness_path, run_reference
from tealeaf_b200 import problems
from tealeaf_b200.host import Host

pytestmark = pytest.mark.gpu

RTOL = 1e-12
RTOL_DOT = 1e-13
D = C.c_double
P = C.POINTER(C.c_double)


def ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P)


def golden(golden_dir):
    return {c["name"]: c for c in json.loads((golden_dir / "ref_runs.json").read_text())}


def compare(steps, gold, rtol=RTOL):
    assert len(steps) == len(gold["steps"])
    for n, (s, g) in enumerate(zip(steps, gold["steps"])):
        assert s.iterations == g["iterations"], "step %d" % (n + 1)
        for a, b in zip(s.summary, g["summary"]):
            assert a == pytest.approx(float(b), rel=rtol), "step %d" % (n + 1)


@pytest.fixture(scope="module")
def host3():
    prob = problems.seeded(3, (21, 17, 13), 41, 3, 1, solver="cg", end_step=1, name="k3")
    h = Host(prob.tea_in(), dims=3)
    yield h
    h.finalise()


def test_3d_initial_state_and_kernels(host3, oracle_lib):
    h = host3
    c = h.cfg
    x, y, z, hd = h.chunk.x, h.chunk.y, h.chunk.z, c.halo_depth
    shape = (z, y, x)
    vx, vy, vz = np.zeros(x + 1), np.zeros(y + 1), np.zeros(z + 1)
    cx, cy, cz = np.zeros(x), np.zeros(y), np.zeros(z)
    n = x * y * z
    vol, xa, ya, za = np.zeros(n), np.zeros(n + y * z), np.zeros(n + x * z), np.zeros(n + x * y)
    oracle_lib.o3_set_chunk_data(x, y, z, hd, D(c.grid_x_min), D(c.grid_y_min), D(c.grid_z_min), D(c.dx),
                                 D(c.dy), D(c.dz), ptr(vx), ptr(vy), ptr(vz), ptr(cx), ptr(cy), ptr(cz), ptr(vol),
                                 ptr(xa), ptr(ya), ptr(za))
    sts = (OState * len(h.states))()
    for i, s in enumerate(h.states):
        sts[i] = OState(s.density, s.energy, s.x_min, s.y_min, s.z_min, s.x_max, s.y_max, s.z_max, s.radius,
                        s.geometry)
    dens, e0, u = np.zeros(shape), np.zeros(shape), np.zeros(shape)
    oracle_lib.o3_set_chunk_state(x, y, z, ptr(vx), ptr(vy), ptr(vz), ptr(cx), ptr(cy), ptr(cz), ptr(dens),
                                  ptr(e0), ptr(u), len(h.states), sts)
    nb = (C.c_int * 6)(*([-1] * 6))
    for f in (dens, e0):
        oracle_lib.o3_halo_field(x, y, z, hd, 2, nb, ptr(f))
    assert np.array_equal(h.download("density"), dens)
    assert np.array_equal(h.download("energy0"), e0)
    assert np.array_equal(h.download("energy"), e0)
    assert np.array_equal(h.download("u"), u)
    assert np.array_equal(h.download("volume").ravel(), vol)

    # cg_init
    rx, ry, rz = 0.004 / c.dx ** 2, 0.004 / c.dy ** 2, 0.004 / c.dz ** 2
    h.reset_fields_to_exchange()
    h.flags[0] = h.flags[2] = True
    h.halo_update(2)
    dens, en = h.download("density"), h.download("energy")
    want = {k: h.download(k) for k in ("u", "p", "r", "w", "kx", "ky", "kz")}
    oracle_lib.o3_cg_init.restype = D
    rro_o = oracle_lib.o3_cg_init(x, y, z, hd, c.coefficient, D(rx), D(ry), D(rz), ptr(dens), ptr(en),
                                  *[ptr(want[k]) for k in ("u", "p", "r", "w", "kx", "ky", "kz")])
    rro = h._acc("run_cg_init", rx, ry, rz)
    for k, v in want.items():
        assert np.array_equal(h.download(k), v), k
    assert rro == pytest.approx(rro_o, rel=RTOL_DOT)
    # halo(u, p), copy_u, three CG iterations through the deferred/fused path
    u, p = want["u"], want["p"]
    kx, ky, kz, w, r = want["kx"], want["ky"], want["kz"], want["w"], want["r"]
    for f in (u, p):
        oracle_lib.o3_halo_field(x, y, z, hd, 1, nb, ptr(f))
    h.reset_fields_to_exchange()
    h.flags[3] = h.flags[4] = True
    h.halo_update(1)
    u0 = h.download("u0")
    oracle_lib.o3_copy_u(x, y, z, hd, ptr(u0), ptr(u))
    h._call("run_copy_u")
    assert np.array_equal(h.download("u0"), u0)
    oracle_lib.o3_cg_calc_w.restype = D
    oracle_lib.o3_cg_calc_ur.restype = D
    for it in range(3):
        pw_o = oracle_lib.o3_cg_calc_w(x, y, z, hd, ptr(p), ptr(w), ptr(kx), ptr(ky), ptr(kz))
        pw = h._acc("run_cg_calc_w")
        assert np.array_equal(h.download("w"), w) and np.array_equal(h.download("p"), p)
        assert pw == pytest.approx(pw_o, rel=RTOL_DOT)
        a = 0.3 + 0.1 * it
        rrn_o = oracle_lib.o3_cg_calc_ur(x, y, z, hd, D(a), ptr(u), ptr(p), ptr(r), ptr(w))
        rrn = h._acc("run_cg_calc_ur", a)
        assert np.array_equal(h.download("u"), u) and np.array_equal(h.download("r"), r)
        assert rrn == pytest.approx(rrn_o, rel=RTOL_DOT)
        b = 0.55 - 0.1 * it
        oracle_lib.o3_cg_calc_p(x, y, z, hd, D(b), ptr(p), ptr(r))
        h._call("run_cg_calc_p", b)
        for f in (u, p):
            oracle_lib.o3_halo_field(x, y, z, hd, 1, nb, ptr(f))
        h.halo_update(1)
    # Chebyshev, PPCG and shared kernels
    theta = 1.3
    h.chunk.theta = theta
    h.reset_fields_to_exchange()
    oracle_lib.o3_cheby_init(x, y, z, hd, D(theta), ptr(u), ptr(u0), ptr(p), ptr(r), ptr(w), ptr(kx), ptr(ky), ptr(kz))
    h._call("run_cheby_init")
    for k, v in (("u", u), ("p", p), ("r", r), ("w", w)):
        assert np.array_equal(h.download(k), v), k
    oracle_lib.o3_halo_field(x, y, z, hd, 1, nb, ptr(u))
    h.flags[3] = True
    h.halo_update(1)
    oracle_lib.o3_cheby_iterate(x, y, z, hd, D(0.8), D(0.35), ptr(u), ptr(u0), ptr(p), ptr(r), ptr(w), ptr(kx),
                                ptr(ky), ptr(kz))
    h._call("run_cheby_iterate", 0.8, 0.35)
    for k, v in (("u", u), ("p", p), ("r", r), ("w", w)):
        assert np.array_equal(h.download(k), v), k
    sd = h.download("sd")
    oracle_lib.o3_ppcg_init(x, y, z, hd, D(theta), ptr(r), ptr(sd))
    h._call("run_ppcg_init")
    assert np.array_equal(h.download("sd"), sd)
    h.reset_fields_to_exchange()
    h.flags[5] = True
    for it in range(2):
        oracle_lib.o3_halo_field(x, y, z, hd, 1, nb, ptr(sd))
        h.halo_update(1)
        oracle_lib.o3_ppcg_inner(x, y, z, hd, D(0.7), D(0.2 + it), ptr(u), ptr(r), ptr(kx), ptr(ky), ptr(kz), ptr(sd))
        h._call("run_ppcg_inner_iteration", 0.7, 0.2 + it)
        for k, v in (("u", u), ("r", r), ("sd", sd)):
            assert np.array_equal(h.download(k), v), (k, it)
    oracle_lib.o3_calculate_residual(x, y, z, hd, ptr(u), ptr(u0), ptr(r), ptr(kx), ptr(ky), ptr(kz))
    h._call("run_calculate_residual")
    assert np.array_equal(h.download("r"), r)
    oracle_lib.o3_calculate_2norm.restype = D
    assert h.norm("r") == pytest.approx(oracle_lib.o3_calculate_2norm(x, y, z, hd, ptr(r)), rel=RTOL_DOT)
    oracle_lib.o3_finalise(x, y, z, hd, ptr(en), ptr(dens), ptr(u))
    h._call("run_finalise")
    assert np.array_equal(h.download("energy"), en)
    out = (D * 4)()
    oracle_lib.o3_field_summary(x, y, z, hd, ptr(h.download("volume")), ptr(dens), ptr(h.download("energy0")),
                                ptr(u), out)
    for g_, o_ in zip(h.field_summary(), out):
        assert g_ == pytest.approx(o_, rel=RTOL_DOT)
    # Jacobi
    rxj, ryj, rzj = 0.2, 0.3, 0.4
    kx, ky, kz, u0, u, r = (h.download(k) for k in ("kx", "ky", "kz", "u0", "u", "r"))
    oracle_lib.o3_jacobi_init(x, y, z, hd, c.coefficient, D(rxj), D(ryj), D(rzj), ptr(dens), ptr(en), ptr(u0),
                              ptr(u), ptr(kx), ptr(ky), ptr(kz))
    h._call("run_jacobi_init", rxj, ryj, rzj)
    for k, v in (("u0", u0), ("u", u), ("kx", kx), ("ky", ky), ("kz", kz)):
        assert np.array_equal(h.download(k), v), k
    oracle_lib.o3_jacobi_iterate.restype = D
    err_o = oracle_lib.o3_jacobi_iterate(x, y, z, hd, ptr(kx), ptr(ky), ptr(kz), ptr(u0), ptr(u), ptr(r))
    v = C.c_double(5.0)
    h._call("run_jacobi_iterate", C.byref(v))
    assert v.value == pytest.approx(err_o, rel=RTOL_DOT)
    assert np.array_equal(h.download("u"), u) and np.array_equal(h.download("r"), r)


@pytest.mark.parametrize("face", range(6))
def test_3d_pack_unpack(host3, face):
    h = host3
    x, y, z, hd, depth = h.chunk.x, h.chunk.y, h.chunk.z, h.cfg.halo_depth, 2
    u = h.download("u")
    nx, ny, nz = x - 2 * hd, y - 2 * hd, z - 2 * hd
    inner = u[hd:z - hd, hd:y - hd, hd:x - hd]
    n = depth * {0: nz * ny, 1: nz * ny, 2: nz * nx, 3: nz * nx, 4: ny * nx, 5: ny * nx}[face]
    buf = np.zeros(n)
    h._call("run_pack_or_unpack", depth, face, True, h.chunk.vec_u, ptr(buf))
    sel = {0: inner[:, :, :depth], 1: inner[:, :, nx - depth:], 2: inner[:, :depth, :], 3: inner[:, ny - depth:, :],
           4: inner[:depth], 5: inner[nz - depth:]}[face]
    assert np.array_equal(buf, np.ascontiguousarray(sel).ravel())


CASES_3D = ["shipped_3d_25_20", "odd_3d_40x36x28_cg", "odd_3d_40x36x28_cheby", "odd_3d_40x36x28_ppcg",
            "odd_3d_40x36x28_jacobi"]


@pytest.mark.parametrize("name", CASES_3D)
def test_3d_python_host_matches_reference(name, golden_dir):
    g = golden(golden_dir)[name]
    h = Host(g["tea_in"], dims=3)
    try:
        compare(h.run(), g)
    finally:
        h.finalise()


@pytest.mark.parametrize("name", CASES_3D)
def test_3d_device_driver_matches_reference(name, golden_dir):
    g = golden(golden_dir)[name]
    h = Host(g["tea_in"], dims=3)
    try:
        compare(h.run_device(), g)
    finally:
        h.finalise()


@pytest.mark.parametrize("name", ["shipped_3d_25_20", "odd_3d_40x36x28_cg", "odd_3d_40x36x28_ppcg"])
def test_3d_reference_host_binary_dropin(name, golden_dir):
    if not harness_path(3, "b200").exists():
        pytest.skip("oracle/_ref/harness3d_b200 not built")
    g = golden(golden_dir)[name]
    compare(run_reference(g["tea_in"], dims=3, suite="b200"), g)


FIELDS3 = ("u", "u0", "p", "r", "w", "kx", "ky", "kz", "sd", "energy", "density")


@pytest.mark.parametrize("solver", ["cg", "cheby", "ppcg"])
def test_3d_device_driver_memory_state_equals_run_path(solver):
    """The device-resident 3D timestep and the run_* path driven like the
    reference drivers leave every field bit-identical (same sweeps, launch
    shapes and reduction trees), on a mesh with ragged tiles in x, y and z."""
    prob = problems.seeded(3, (37, 19, 23), 29, 3, 1, solver=solver, end_step=2, name="state3")
    text = prob.tea_in()
    a, b = Host(text, 3), Host(text, 3)
    try:
        for tt in range(2):
            ra = a.solve(tt)
            rb = b.solve_device(tt)
            assert ra.iterations == rb.iterations
            assert ra.summary == rb.summary
            for f in FIELDS3:
                assert np.array_equal(a.download(f), b.download(f)), (solver, tt, f)
    finally:
        a.finalise()
        b.finalise()


def test_3d_adjoint_rejects_bad_arguments():
    h = Host(problems.seeded(3, (12, 10, 8), 3, 2, 0, solver="cheby", end_step=1, name="adjbad").tea_in(), 3)
    try:
        with pytest.raises(Exception):          # the adjoint differentiates the CG timestep only
            h.adjoint_gradient(1, 1, [0, 10, 0, 10, 0, 10], 1e-10)
    finally:
        h.finalise()
    h = Host(problems.seeded(3, (12, 10, 8), 3, 2, 0, solver="cg", end_step=1, name="adjbad2").tea_in(), 3)
    try:
        with pytest.raises(Exception):          # at least one step
            h.adjoint_gradient(0, 1, [0, 10, 0, 10, 0, 10], 1e-10)
    finally:
        h.finalise()


@pytest.mark.parametrize("solver,path", [("cg", "device"), ("cg", "run"), ("cheby", "device"), ("ppcg", "device")])
def test_3d_tma_sweep_matches_async_copies(solver, path):
    """The stencil sweeps fed by TMA tile loads (even row length: 38 + 4) and
    the ones fed by per-thread asynchronous copies give bit-identical fields
    and iteration counts, through the device driver (CG, Chebyshev, PPCG)
    and through run_*, on a mesh with ragged tiles in x (32 + 6), y and z."""
    prob = problems.seeded(3, (38, 19, 23), 29, 3, 1, solver=solver, end_step=2, name="tma3")
    text = prob.tea_in()
    a, b = Host(text, 3), Host(text, 3)
    try:
        a.lib.tl3d_set_temporal_blocking(a.chunk, 0)   # the one-step sweeps, fed both ways
        b.lib.tl3d_set_temporal_blocking(b.chunk, 0)
        b.lib.tl3d_set_tma(b.chunk, 0)
        for tt in range(2):
            ra = a.solve_device(tt) if path == "device" else a.solve(tt)
            rb = b.solve_device(tt) if path == "device" else b.solve(tt)
            assert ra.iterations == rb.iterations
            assert ra.summary == rb.summary
            for f in FIELDS3:
                assert np.array_equal(a.download(f), b.download(f)), (path, tt, f)
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("solver,dims,inner", [
    ("cheby", (37, 19, 23), 10),
    ("ppcg", (37, 19, 23), 10),
    ("ppcg", (37, 19, 23), 7),
    ("ppcg", (37, 19, 23), 1),
    ("cheby", (38, 19, 23), 10),
    ("ppcg", (38, 19, 23), 5),
    ("cheby", (30, 24, 150), 10),
    ("ppcg", (30, 24, 150), 4),
])
def test_3d_blocked_trips_match_one_step(solver, dims, inner):
    """The device driver's temporally blocked Chebyshev trips and PPCG inner
    steps (k3_blocked / k3_blocked_tma: up to two per launch, x-y tiles with
    a margin, z segments of 64 planes) leave every field and the iteration
    counts bit-identical to one launch per trip / step, on meshes with
    ragged tiles in x and y, odd rows (per-thread loads) and even rows (region
    planes by TMA), one or three z segments, and inner-step counts that fill,
    split and underfill the blocks."""
    prob = problems.seeded(3, dims, 31, 3, 1, solver=solver, end_step=2, name="blk3").with_(
        ppcg_inner_steps=inner)
    text = prob.tea_in()
    a, b = Host(text, 3), Host(text, 3)
    try:
        b.lib.tl3d_set_temporal_blocking(b.chunk, 0)
        for tt in range(2):
            ra = a.solve_device(tt)
            rb = b.solve_device(tt)
            assert ra.iterations == rb.iterations
            assert ra.iterations.get("Cheby" if solver == "cheby" else "PPCG", 0) > 0
            assert ra.summary == rb.summary
            for f in FIELDS3:
                assert np.array_equal(a.download(f), b.download(f)), (solver, dims, tt, f)
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("solver,dims,inner,cap", [
    ("cheby", (37, 19, 23), 10, None),
    ("cheby", (38, 19, 23), 10, None),
    ("cheby", (38, 19, 23), 10, 183),
    ("ppcg", (37, 19, 23), 10, None),
    ("ppcg", (38, 19, 23), 7, None),
    ("ppcg", (38, 19, 23), 2, None),
    ("ppcg", (38, 19, 23), 1, None),
])
def test_3d_run_path_queues_are_bit_identical(solver, dims, inner, cap):
    """Through run_* (the reference drivers' call sequence), the Chebyshev
    trips and PPCG inner steps deferred and run temporally blocked (each trip
    ending with its u += p; sd = r / theta with the first step, the last sd
    update after the blocks) give the same iteration counts, summaries and
    memory state, bit for bit, as one launch per call; per-thread loads (odd
    rows) and TMA-staged regions (even rows), an iteration cap that stops
    the queue between norm checks, and inner-step counts that split, fill
    and underfill the two-step blocks."""
    prob = problems.seeded(3, dims, 37, 3, 1, solver=solver, end_step=2, name="q3").with_(ppcg_inner_steps=inner)
    if cap:
        prob = prob.with_(max_iters=cap)
    text = prob.tea_in()
    a, b = Host(text, 3), Host(text, 3)
    try:
        b.lib.tl3d_set_temporal_blocking(b.chunk, 0)
        for tt in range(2):
            ra = a.solve(tt)
            rb = b.solve(tt)
            assert ra.iterations == rb.iterations
            assert ra.iterations.get("Cheby" if solver == "cheby" else "PPCG", 0) > 0
            assert ra.summary == rb.summary
            assert ra.exact_error == rb.exact_error
            for f in FIELDS3:
                assert np.array_equal(a.download(f), b.download(f)), (solver, dims, tt, f)
    finally:
        a.finalise()
        b.finalise()


@pytest.mark.parametrize("dims,trips", [((37, 19, 23), 1), ((38, 19, 23), 4), ((38, 19, 23), 5)])
def test_3d_cg_sweeps_run_the_deferred_trips_first(dims, trips, cheby_then_cg_sweeps):
    """Chebyshev trips still queued when run_cg_solver_calc_w, _calc_ur and
    _calc_p are called run before them: the sweeps' dot products and the
    memory state match, bit for bit, a chunk that ran every trip at once."""
    text = problems.seeded(3, dims, 41, 3, 1, solver="cheby", end_step=1, name="qcg3").tea_in()
    a, b = Host(text, 3), Host(text, 3)
    try:
        b.lib.tl3d_set_temporal_blocking(b.chunk, 0)
        ra = cheby_then_cg_sweeps(a, trips)
        rb = cheby_then_cg_sweeps(b, trips)
        assert ra == rb
        for f in FIELDS3:
            assert np.array_equal(a.download(f), b.download(f)), (dims, trips, f)
    finally:
        a.finalise()
        b.finalise()
