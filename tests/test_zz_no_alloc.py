"""The allocation-free 2-norm entry point (tl2d_calculate_2norm_noalloc).

It exists for callers that cannot allocate device memory, or cannot afford
the synchronisation an allocation implies, while a solve is running: its
reduction scratch is a static device array of fixed size instead of memory
from cudaMalloc. These tests call it through the C ABI and compare it with the
regular run_calculate_2norm on the same field (equal up to rounding: the two
add their block partials in different trees), twice in a row per field: the
static array keeps the previous call's contents, and the repeated calls show
that leftover contents do not change the result. The file is named so pytest
collects it last.
"""
import ctypes as C

import pytest

from tealeaf_b200 import abi, problems

RTOL_DOT = 1e-13


def test_noalloc_rejects_grids_beyond_its_scratch():
    """Oversized grids fail with an error before anything is launched (no GPU needed)."""
    lib = abi.load(2)
    abi.check(lib, 2)  # start clean
    rc = lib.tl2d_calculate_2norm_noalloc(C.c_void_p(0x1000), 20004, 20004, 2, C.c_void_p(0x2000), None)
    assert rc == 22
    with pytest.raises(abi.SuiteError, match="static scratch"):
        abi.check(lib, 2)


@pytest.mark.gpu
def test_noalloc_matches_run_calculate_2norm_twice():
    import torch

    from tealeaf_b200.host import Host

    prob = problems.plain_2d(300, seed=9, steps=1, solver="cg")
    h = Host(prob.tea_in(), dims=2)
    try:
        h.run(1)
        stream = h.lib.tl2d_stream(C.byref(h.chunk))
        x, y, hd = h.chunk.x, h.chunk.y, h.cfg.halo_depth
        for field in ("u0", "r", "u0", "r"):       # two calls in a row per field
            want = h.norm(field)                    # existing entry point (host result)
            out = torch.zeros(1, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            ptr = getattr(h.chunk, field)
            rc = h.lib.tl2d_calculate_2norm_noalloc(C.c_void_p(ptr), x, y, hd, C.c_void_p(out.data_ptr()),
                                                     C.c_void_p(stream))
            abi.check(h.lib, 2)
            assert rc == 0
            torch.cuda.synchronize()
            got = out.item()
            assert got == pytest.approx(want, rel=RTOL_DOT), field
            assert want > 0.0
    finally:
        h.finalise()
