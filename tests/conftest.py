"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs on any machine (oracle pins, ABI/layout checks, host
logic, multi-process CPU tests); `-m gpu` needs a B200 and calls the suite
through its C ABI.
"""
import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built suite libraries")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle.oracle import OracleLib
    return OracleLib()


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


def _cheby_then_cg_sweeps(h, trips):
    """One timestep's opening through run_* on a tealeaf_b200.host.Host
    (2D or 3D): 15 CG steps, the eigenvalue bounds, Chebyshev trips in the
    reference drivers' pattern (a depth-1 halo of u before each), then CG
    sweeps called with no other run_* call between them, as a host leaving
    the Chebyshev phase straight for CG would. Returns (pw, rrn)."""
    from tealeaf_b200.host import FIELD_DENSITY, FIELD_ENERGY1, FIELD_P, FIELD_U
    c, ch = h.cfg, h.chunk
    rx, ry = c.dt_init / (c.dx * c.dx), c.dt_init / (c.dy * c.dy)
    rz = c.dt_init / (c.dz * c.dz) if h.dims == 3 else 0.0
    h.reset_fields_to_exchange()
    h.flags[FIELD_ENERGY1] = h.flags[FIELD_DENSITY] = True
    h.halo_update(2)
    rro = h.cg_init_driver(rx, ry, rz)
    n_cg = 15
    for tt in range(n_cg):
        rro, _ = h.cg_main_step(tt, rro)
        h.halo_update(1)
    h._eigenvalues(n_cg)
    h._cheby_coefs(trips + 1)
    h._call("run_cheby_init")
    h.reset_fields_to_exchange()
    h.flags[FIELD_U] = True
    h.halo_update(1)
    for n in range(1, trips + 1):
        h._call("run_cheby_iterate", ch.cheby_alphas[n], ch.cheby_betas[n])
        h.halo_update(1)
    h.reset_fields_to_exchange()
    h.flags[FIELD_P] = True
    h.halo_update(1)
    pw = h._acc("run_cg_calc_w")
    rrn = h._acc("run_cg_calc_ur", rro / pw)
    h._call("run_cg_calc_p", rrn / rro)
    return pw, rrn


@pytest.fixture(scope="session")
def cheby_then_cg_sweeps():
    return _cheby_then_cg_sweeps
