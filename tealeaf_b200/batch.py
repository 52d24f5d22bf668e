"""Batched 2D timesteps: many independent problems of different sizes solved
in one persistent, graph-captured launch (tl2d_batch_* in batch2d.cu).

Each problem is an ordinary chunk initialised through the reference kernel
interface by its own Host (tea.in settings, state painting, halos); the batch
then runs one solve() of every problem per step. The Host objects stay alive
as long as the batch.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .host import DriverError, Host


class Batch:
    def __init__(self, tea_ins: Sequence[str], tile_rows: int = 0, grid_blocks: int = 0):
        self.hosts: List[Host] = [Host(t, dims=2) for t in tea_ins]
        self.lib = self.hosts[0].lib
        n = len(self.hosts)
        chunks = (C.POINTER(abi.Chunk2D) * n)(*[C.pointer(h.chunk) for h in self.hosts])
        settings = (C.POINTER(abi.Settings2D) * n)(*[C.pointer(h.settings) for h in self.hosts])
        self._keep = (chunks, settings)
        self.handle = self.lib.tl2d_batch_create(chunks, settings, n, tile_rows, grid_blocks)
        abi.check(self.lib, 2)
        if not self.handle:
            raise DriverError("tl2d_batch_create failed")

    @property
    def count(self) -> int:
        return len(self.hosts)

    def tune(self, trial_iters: int = 50) -> dict:
        best = C.c_double()
        rc = self.lib.tl2d_batch_tune(self.handle, trial_iters, C.byref(best))
        abi.check(self.lib, 2)
        if rc:
            raise DriverError("tl2d_batch_tune returned %d" % rc)
        return dict(self.config(), trial_ms=best.value)

    def config(self) -> dict:
        rows, grid = C.c_int(), C.c_int()
        self.lib.tl2d_batch_config(self.handle, C.byref(rows), C.byref(grid))
        return {"tile_rows": rows.value, "grid_blocks": grid.value}

    def step(self) -> abi.BatchStats:
        st = abi.BatchStats()
        rc = self.lib.tl2d_batch_step(self.handle, C.byref(st))
        abi.check(self.lib, 2)
        if rc:
            raise DriverError("tl2d_batch_step returned %d" % rc)
        return st

    def set_wait_limit(self, cycles: int) -> None:
        """SM clocks a phase wait of the batch kernel may take before it gives up (<= 0: the default)."""
        rc = self.lib.tl2d_batch_set_wait_limit(self.handle, cycles)
        abi.check(self.lib, 2)
        if rc:
            raise DriverError("tl2d_batch_set_wait_limit returned %d" % rc)

    def results(self):
        n = self.count
        it = np.zeros(n, dtype=np.int32)
        rr = np.zeros(n)
        conv = np.zeros(n, dtype=np.int32)
        self.lib.tl2d_batch_results(self.handle, it.ctypes.data_as(C.c_void_p), rr.ctypes.data_as(C.c_void_p),
                                    conv.ctypes.data_as(C.c_void_p))
        abi.check(self.lib, 2)
        return it, rr, conv

    def summaries(self) -> List[List[float]]:
        return [h.field_summary() for h in self.hosts]

    def close(self):
        if getattr(self, "handle", None):
            self.lib.tl2d_batch_destroy(self.handle)
            self.handle = None
        for h in getattr(self, "hosts", []):
            h.finalise()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
