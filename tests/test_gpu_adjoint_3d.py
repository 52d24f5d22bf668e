"""The 3D adjoint (tl3d_adjoint_gradient / tl3d_solve_step_backward) on the B200.

* Against the FP64 CPU adjoint of the oracle (pinned to central differences
  of the reference's own forward timestep in tests/test_adjoint_oracle.py):
  J within 1e-12 relative, the gradient within 1e-9 of its norm.
* Against central differences (h = 1e-6 on log density) of the B200 forward
  timestep at the most sensitive cells and at seeded random cells: 1e-6
  relative plus the rounding floor of J (eps * |J| / h).
* Checkpoint interval and recomputation do not change the result, and the
  chunk ends in its state after the forward timesteps.
"""
import numpy as np
import pytest

from tealeaf_b200 import problems
from tealeaf_b200.config import read_config
from tealeaf_b200.host import Host

pytestmark = pytest.mark.gpu

BOX = [6.0, 9.0, 6.0, 9.0, 6.0, 9.0]
H = 1e-6
ADJ_TOL = 1e-13


def _problem(steps=4, n=(20, 18, 16)):
    return problems.seeded(3, n, 33, 6, 0, solver="cg", eps=1e-14, end_step=steps, name="adj_gpu")


def _objective(host, hd=2):
    u, v, rho = host.download("u"), host.download("volume"), host.download("density")
    c = host.cfg
    nz, ny, nx = c.grid_z_cells, c.grid_y_cells, c.grid_x_cells
    sl = (slice(hd, hd + nz), slice(hd, hd + ny), slice(hd, hd + nx))
    xs = c.grid_x_min + c.dx * (np.arange(nx) + 0.5)
    ys = c.grid_y_min + c.dy * (np.arange(ny) + 0.5)
    zs = c.grid_z_min + c.dz * (np.arange(nz) + 0.5)
    m = ((zs >= BOX[4]) & (zs <= BOX[5]))[:, None, None] & ((ys >= BOX[2]) & (ys <= BOX[3]))[None, :, None] & \
        ((xs >= BOX[0]) & (xs <= BOX[1]))[None, None, :]
    return float(np.sum((v[sl] * rho[sl] * u[sl])[m]))


def _forward_J(text, steps, cell=None, log_scale=0.0, hd=2):
    h = Host(text, 3)
    try:
        if cell is not None:
            rho = h.download("density")
            c = h.cfg
            nx, ny = c.grid_x_cells, c.grid_y_cells
            k, j, i = cell % nx, (cell // nx) % ny, cell // (nx * ny)
            rho[i + hd, j + hd, k + hd] *= np.exp(log_scale)
            h.upload("density", rho)
        for tt in range(steps):
            h.solve_device(tt, summary=False)
        return _objective(h)
    finally:
        h.finalise()


@pytest.fixture(scope="module")
def gpu_adjoint():
    text = _problem().tea_in()
    h = Host(text, 3)
    try:
        J, g, st = h.adjoint_gradient(4, 2, BOX, ADJ_TOL)
        energy = h.download("energy")
    finally:
        h.finalise()
    return text, J, g, st, energy


def test_gpu_adjoint_matches_cpu_adjoint(gpu_adjoint, oracle_lib):
    text, J, g, st, _ = gpu_adjoint
    cfg, states = read_config(text, 3)
    Jc, gc = oracle_lib.adjoint3d(cfg, states, BOX, ADJ_TOL)
    assert J == pytest.approx(Jc, rel=1e-12)
    assert np.linalg.norm(g - gc) <= 1e-9 * np.linalg.norm(gc)
    assert st.checkpoints == 2 and st.forward_steps == 4 + 2   # one segment recomputed
    assert st.adjoint_iters > 0


def test_gpu_adjoint_matches_central_differences(gpu_adjoint):
    text, J, g, _, _ = gpu_adjoint
    gf = g.ravel()
    rng = np.random.default_rng(5)
    cells = list(np.argsort(-np.abs(gf))[:3]) + list(rng.integers(0, gf.size, 3))
    noise = 8.0 * np.finfo(float).eps * abs(J) / (2 * H)
    for c in cells:
        fd = (_forward_J(text, 4, int(c), H) - _forward_J(text, 4, int(c), -H)) / (2 * H)
        assert abs(fd - gf[c]) <= 1e-6 * abs(gf[c]) + noise, (c, gf[c], fd)


def test_checkpoint_interval_and_final_state(gpu_adjoint):
    text, J, g, _, energy = gpu_adjoint
    h = Host(text, 3)
    try:
        J1, g1, st1 = h.adjoint_gradient(4, 1, BOX, ADJ_TOL)
    finally:
        h.finalise()
    assert J1 == J and np.array_equal(g1, g)
    assert st1.checkpoints == 4 and st1.forward_steps == 4 + 3
    f = Host(text, 3)
    try:
        for tt in range(4):
            f.solve_device(tt, summary=False)
        assert np.array_equal(f.download("energy"), energy)
        assert _objective(f) == pytest.approx(J, rel=1e-14)
    finally:
        f.finalise()
