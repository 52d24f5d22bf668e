"""tea.in parsing (host side) and the seeded problem generator."""
import numpy as np
import pytest

from tealeaf_b200 import problems
from tealeaf_b200.config import CIRCULAR, RECIP_CONDUCTIVITY, RECTANGULAR, read_config

SHIPPED_2D = """*tea
state 1 density=100.0 energy=0.0001
state 2 density=0.1 energy=25.0 geometry=rectangle xmin=0.0 xmax=1.0 ymin=1.0 ymax=2.0
state 3 density=0.1 energy=0.1 geometry=circular xmin=5.0 ymin=5.0 xmax=1.0 ymax=1.0 radius=2.0

xmin                = 0.0
ymin                = 0.0
xmax                = 10.0
ymax                = 10.0
x_cells             = 4096
y_cells             = 4096
x_cells             = 7

use_ppcg
use_c_kernels
check_result
coefficient_inverse_density
eps                 = 1.0e-15
epslim              = 0.0001
max_iters           = 5000
initial_timestep    = 0.004
end_step            = 3
*endtea
"""


def test_reference_parser_rules():
    c, st = read_config(SHIPPED_2D, 2)
    # x_cells is only read while it holds the default (2d/parse_config.c:102-107)
    assert (c.grid_x_cells, c.grid_y_cells) == (4096, 4096)
    assert c.eps == 1e-15 and c.eps_lim == 1e-4          # "epslim" is matched before "eps"
    assert c.solver == 3 and c.solver_name == "PPCG"
    assert c.coefficient == RECIP_CONDUCTIVITY and c.kernel_language == 0
    assert c.max_iters == 5000 and c.end_step == 3 and c.dt_init == 0.004
    dx = 10.0 / 4096
    assert c.dx == dx
    assert st[1].geometry == RECTANGULAR
    assert st[1].x_min == 0.0 + dx / 100.0 and st[1].x_max == 1.0 - dx / 100.0
    assert st[2].geometry == CIRCULAR and st[2].radius == 2.0
    assert st[2].x_min == 5.0 + dx / 100.0                 # circle centres move too


def test_3d_reads_cells_unconditionally():
    text = "x_cells = 8\nx_cells = 9\ny_cells = 5\nz_cells = 4\nstate 1 density=1 energy=2\n"
    c, _ = read_config(text, 3)
    assert (c.grid_x_cells, c.grid_y_cells, c.grid_z_cells) == (9, 5, 4)


def test_generator_is_seeded_and_round_trips():
    a = problems.dropin_2d(4096, seed=2, steps=10, solver="cheby")
    b = problems.dropin_2d(4096, seed=2, steps=10, solver="cheby")
    assert a.tea_in() == b.tea_in()
    assert problems.dropin_2d(4096, seed=3).tea_in() != a.tea_in()
    c, st = read_config(a.tea_in(), 2)
    assert len(st) == 1 + 8 + 4
    assert sum(s.geometry == CIRCULAR for s in st[1:]) == 4
    assert c.presteps == 30 and c.solver == 2 and c.grid_x_cells == 4096
    for s in st[1:]:
        assert s.density == 0.1 and 0.1 <= s.energy <= 25.0


def test_batched_sizes_log_uniform():
    ps = problems.batched_2d(64, seed=5)
    sizes = np.array([p.cells for p in ps]).ravel()
    assert len(ps) == 64 and sizes.min() >= 128 and sizes.max() <= 2048
    assert all(p.eps == 1e-12 for p in ps)
