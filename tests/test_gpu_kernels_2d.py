"""Element-wise parity of every 2D run_* kernel with the oracle (B200 only).

Each kernel is called through the C ABI on a small odd-sized grid and its
output fields are compared with the oracle's restatement of the same
reference kernel on the same inputs. Element-wise kernels must match BIT FOR
BIT (the suite is built with -fmad=false and evaluates the reference's
expressions in the reference's order); dot products may differ only by
summation order (relative 1e-13).
"""
import ctypes as C

import numpy as np
import pytest

from tealeaf_b200 import problems
from tealeaf_b200.host import Host

pytestmark = pytest.mark.gpu

RTOL_DOT = 1e-13
D = C.c_double
P = C.POINTER(C.c_double)


def ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P)


@pytest.fixture(scope="module")
def host():
    prob = problems.seeded(2, (37, 29), 21, 3, 2, solver="cg", end_step=1, name="kernels")
    # add a point state so every geometry branch is exercised (the parser moves
    # its coordinates by dx/100, 2d/parse_config.c:254-260, so it never lands
    # exactly on a vertex and paints nothing -- in the reference as here)
    prob.states.append("density=0.5 energy=3.0 geometry=point xmin=5.0 ymin=5.0 xmax=5.0 ymax=5.0")
    h = Host(prob.tea_in(), dims=2)
    yield h
    h.finalise()


def geo(h):
    return h.chunk.x, h.chunk.y, h.cfg.halo_depth


def test_initial_state(host, oracle_lib):
    h = host
    x, y, hd = geo(h)
    c = h.cfg
    vx, vy, cx, cy = np.zeros(x + 1), np.zeros(y + 1), np.zeros(x), np.zeros(y)
    vol, xa, ya = np.zeros(x * y), np.zeros((x + 1) * y), np.zeros(x * (y + 1))
    oracle_lib.o2_set_chunk_data(x, y, hd, D(c.grid_x_min), D(c.grid_y_min), D(c.dx), D(c.dy),
                                 ptr(vx), ptr(vy), ptr(cx), ptr(cy), ptr(vol), ptr(xa), ptr(ya))
    from oracle.oracle import OState
    sts = (OState * len(h.states))()
    for n, s in enumerate(h.states):
        sts[n] = OState(s.density, s.energy, s.x_min, s.y_min, 0.0, s.x_max, s.y_max, 0.0, s.radius, s.geometry)
    dens, e0, u = np.zeros((y, x)), np.zeros((y, x)), np.zeros((y, x))
    oracle_lib.o2_set_chunk_state(x, y, ptr(vx), ptr(vy), ptr(cx), ptr(cy), ptr(dens), ptr(e0), ptr(u),
                                  len(h.states), sts)
    nb = (C.c_int * 4)(-1, -1, -1, -1)
    for f in (dens, e0):
        oracle_lib.o2_halo_field(x, y, hd, 2, nb, ptr(f))
    assert np.array_equal(h.download("density"), dens)
    assert np.array_equal(h.download("energy0"), e0)
    assert np.array_equal(h.download("energy"), e0)      # store_energy after the halo update
    assert np.array_equal(h.download("u"), u)
    assert np.array_equal(h.download("volume").ravel(), vol)
    assert len(np.unique(dens)) >= 2                     # the boxes and circles really painted


def _cg_init(h, oracle_lib, rx, ry):
    x, y, hd = geo(h)
    dens, en = h.download("density"), h.download("energy")
    want = {k: np.zeros((y, x)) for k in ("u", "p", "r", "w", "kx", "ky")}
    for k in ("w", "kx", "ky"):
        want[k] = h.download(k)  # untouched cells keep their previous values
    oracle_lib.o2_cg_init.restype = D
    rro_o = oracle_lib.o2_cg_init(x, y, hd, h.cfg.coefficient, D(rx), D(ry), ptr(dens), ptr(en),
                                  *[ptr(want[k]) for k in ("u", "p", "r", "w", "kx", "ky")])
    rro = h._acc("run_cg_init", rx, ry)
    for k, v in want.items():
        assert np.array_equal(h.download(k), v), k
    assert rro == pytest.approx(rro_o, rel=RTOL_DOT)


def test_cg_kernels(host, oracle_lib):
    h = host
    x, y, hd = geo(h)
    rx, ry = 0.004 / h.cfg.dx ** 2, 0.004 / h.cfg.dy ** 2
    h.reset_fields_to_exchange()
    h.flags[1] = h.flags[2] = h.flags[0] = True
    h.halo_update(2)
    _cg_init(h, oracle_lib, rx, ry)
    nb = (C.c_int * 4)(-1, -1, -1, -1)
    # halo on u, p then copy_u
    u, p = h.download("u"), h.download("p")
    oracle_lib.o2_halo_field(x, y, hd, 1, nb, ptr(u))
    oracle_lib.o2_halo_field(x, y, hd, 1, nb, ptr(p))
    h.reset_fields_to_exchange()
    h.flags[3] = h.flags[4] = True
    h.halo_update(1)
    assert np.array_equal(h.download("u"), u)
    assert np.array_equal(h.download("p"), p)
    u0 = h.download("u0")
    oracle_lib.o2_copy_u(x, y, hd, ptr(u0), ptr(u))
    h._call("run_copy_u")
    assert np.array_equal(h.download("u0"), u0)

    kx, ky, w, r = h.download("kx"), h.download("ky"), h.download("w"), h.download("r")
    for it in range(3):
        oracle_lib.o2_cg_calc_w.restype = D
        pw_o = oracle_lib.o2_cg_calc_w(x, y, hd, ptr(p), ptr(w), ptr(kx), ptr(ky))
        pw = h._acc("run_cg_calc_w")
        assert np.array_equal(h.download("w"), w)
        assert pw == pytest.approx(pw_o, rel=RTOL_DOT)
        alpha = 0.37 + 0.1 * it
        oracle_lib.o2_cg_calc_ur.restype = D
        rrn_o = oracle_lib.o2_cg_calc_ur(x, y, hd, D(alpha), ptr(u), ptr(p), ptr(r), ptr(w))
        rrn = h._acc("run_cg_calc_ur", alpha)
        assert np.array_equal(h.download("u"), u)
        assert np.array_equal(h.download("r"), r)
        assert rrn == pytest.approx(rrn_o, rel=RTOL_DOT)
        beta = 0.61 - 0.05 * it
        oracle_lib.o2_cg_calc_p(x, y, hd, D(beta), ptr(p), ptr(r))
        h._call("run_cg_calc_p", beta)
        oracle_lib.o2_halo_field(x, y, hd, 1, nb, ptr(u))
        oracle_lib.o2_halo_field(x, y, hd, 1, nb, ptr(p))
        h.halo_update(1)
        assert np.array_equal(h.download("p"), p)
        assert np.array_equal(h.download("u"), u)


def test_cheby_ppcg_and_shared_kernels(host, oracle_lib):
    h = host
    x, y, hd = geo(h)
    nb = (C.c_int * 4)(-1, -1, -1, -1)
    u, u0, p, r, w = (h.download(k) for k in ("u", "u0", "p", "r", "w"))
    kx, ky, sd, dens, en = (h.download(k) for k in ("kx", "ky", "sd", "density", "energy"))
    theta = 1.7
    h.chunk.theta = theta
    oracle_lib.o2_cheby_init(x, y, hd, D(theta), ptr(u), ptr(u0), ptr(p), ptr(r), ptr(w), ptr(kx), ptr(ky))
    h._call("run_cheby_init")
    for k, v in (("u", u), ("p", p), ("r", r), ("w", w)):
        assert np.array_equal(h.download(k), v), k
    for it in range(2):
        oracle_lib.o2_halo_field(x, y, hd, 1, nb, ptr(u))
        h.reset_fields_to_exchange()
        h.flags[3] = True
        h.halo_update(1)
        a, b = 0.9 - 0.1 * it, 0.3 + 0.05 * it
        oracle_lib.o2_cheby_iterate(x, y, hd, D(a), D(b), ptr(u), ptr(u0), ptr(p), ptr(r), ptr(w), ptr(kx), ptr(ky))
        h._call("run_cheby_iterate", a, b)
        for k, v in (("u", u), ("p", p), ("r", r), ("w", w)):
            assert np.array_equal(h.download(k), v), (k, it)

    oracle_lib.o2_ppcg_init(x, y, hd, D(theta), ptr(r), ptr(sd))
    h._call("run_ppcg_init")
    assert np.array_equal(h.download("sd"), sd)
    for it in range(3):
        oracle_lib.o2_halo_field(x, y, hd, 1, nb, ptr(sd))
        h.reset_fields_to_exchange()
        h.flags[5] = True
        h.halo_update(1)
        a, b = 0.8, 0.15 * (it + 1)
        oracle_lib.o2_ppcg_inner(x, y, hd, D(a), D(b), ptr(u), ptr(r), ptr(kx), ptr(ky), ptr(sd))
        h._call("run_ppcg_inner_iteration", a, b)
        for k, v in (("u", u), ("r", r), ("sd", sd)):
            assert np.array_equal(h.download(k), v), (k, it)

    oracle_lib.o2_calculate_residual(x, y, hd, ptr(u), ptr(u0), ptr(r), ptr(kx), ptr(ky))
    h._call("run_calculate_residual")
    assert np.array_equal(h.download("r"), r)
    oracle_lib.o2_calculate_2norm.restype = D
    for name, arr in (("r", r), ("u0", u0)):
        assert h.norm(name) == pytest.approx(oracle_lib.o2_calculate_2norm(x, y, hd, ptr(arr)), rel=RTOL_DOT)
    oracle_lib.o2_finalise(x, y, hd, ptr(en), ptr(dens), ptr(u))
    h._call("run_finalise")
    assert np.array_equal(h.download("energy"), en)
    vol, e0 = h.download("volume"), h.download("energy0")
    out = (D * 4)()
    oracle_lib.o2_field_summary(x, y, hd, ptr(vol), ptr(dens), ptr(e0), ptr(u), out)
    got = h.field_summary()
    for g_, o_ in zip(got, out):
        assert g_ == pytest.approx(o_, rel=RTOL_DOT)


def test_jacobi_kernels(host, oracle_lib):
    h = host
    x, y, hd = geo(h)
    dens, en = h.download("density"), h.download("energy")
    u0, u, kx, ky, r = (h.download(k) for k in ("u0", "u", "kx", "ky", "r"))
    rx, ry = 0.3, 0.2
    oracle_lib.o2_jacobi_init(x, y, hd, h.cfg.coefficient, D(rx), D(ry), ptr(dens), ptr(en), ptr(u0), ptr(u),
                              ptr(kx), ptr(ky))
    h._call("run_jacobi_init", rx, ry)
    for k, v in (("u0", u0), ("u", u), ("kx", kx), ("ky", ky)):
        assert np.array_equal(h.download(k), v), k
    oracle_lib.o2_jacobi_iterate.restype = D
    for it in range(2):
        err_o = oracle_lib.o2_jacobi_iterate(x, y, hd, ptr(kx), ptr(ky), ptr(u0), ptr(u), ptr(r))
        v = C.c_double(123.0)   # assigned, not accumulated
        h._call("run_jacobi_iterate", C.byref(v))
        assert v.value == pytest.approx(err_o, rel=RTOL_DOT)
        assert np.array_equal(h.download("u"), u)
        assert np.array_equal(h.download("r"), r)


@pytest.mark.parametrize("face", [0, 1, 2, 3])
@pytest.mark.parametrize("depth", [1, 2])
def test_pack_unpack(host, face, depth):
    h = host
    x, y, hd = geo(h)
    u = h.download("u")
    nxi, nyi = x - 2 * hd, y - 2 * hd
    n = depth * (nyi if face in (0, 1) else nxi)
    buf = np.zeros(n)
    h._call("run_pack_or_unpack", depth, face, True, h.chunk.u, ptr(buf))
    inner = u[hd:y - hd, hd:x - hd]
    want = {0: inner[:, :depth], 1: inner[:, nxi - depth:], 2: inner[:depth, :], 3: inner[nyi - depth:, :]}[face]
    assert np.array_equal(buf, np.ascontiguousarray(want).ravel())
    # unpack a recognisable buffer into the halo and check the placement
    src = np.arange(n, dtype=np.float64) + 1000.0
    h._call("run_pack_or_unpack", depth, face, False, h.chunk.sd, ptr(src))
    sd = h.download("sd")
    if face == 0:
        got = sd[hd:y - hd, hd - depth:hd]
    elif face == 1:
        got = sd[hd:y - hd, x - hd:x - hd + depth]
    elif face == 2:
        got = sd[hd - depth:hd, hd:x - hd]
    else:
        got = sd[y - hd:y - hd + depth, hd:x - hd]
    assert np.array_equal(np.ascontiguousarray(got).ravel(), src)
