"""One mesh decomposed over ranks, one chunk per rank, solved through run_*.

The reference splits the mesh into num_ranks x num_chunks_per_rank chunks
with the least halo surface per cell (decompose_field,
2d/initialise.c:34-134, 3d/initialise.c:34-174), exchanges the faces of the
fields being updated between neighbouring chunks before the local halos
(halo_update_driver.c:6-25, remote_halo_driver.c:11-128 in 2d/drivers and
3d/drivers) and sums every dot product over the ranks (sum_over_ranks,
2d/comms.c:55-61). Here each rank (one process per GPU) owns one chunk:

* `decompose` restates decompose_field: chunk counts along each axis by the
  same search and metric, the remainder cells given to the first chunks of
  each axis, neighbours by chunk index (-1 on the mesh boundary).
* `FaceExchange` moves the faces: per axis in the order x, y(, z), every face
  with a neighbour packs the requested fields, `depth` layers deep, into one
  message (the suite's own run_pack_or_unpack, which takes host or device
  memory), the messages of the axis cross in both directions as
  torch.distributed point-to-point operations (NCCL between GPUs, gloo
  between host processes), and each received message is unpacked on the face
  it came through; the next axis starts once the previous one is unpacked.
* `DistHost` is tealeaf_b200.host.Host over that chunk: the reference
  drivers' call sequence, the remote faces before the local halos, and,
  wherever the drivers call sum_over_ranks, the ranks' values gathered and
  added in rank order.

The device-resident entry points (tl2d_solve_step, tl3d_solve_step, the
refinement and adjoint forms) hold no exchange and refuse a chunk with an
internal face; a decomposed mesh runs through run_*.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist

from . import abi
from .host import DriverError, Host

EXTERNAL_FACE = -1

# Chunk members of the exchangeable fields, in the reference's field order
# (FIELD_DENSITY, FIELD_ENERGY0, FIELD_ENERGY1, FIELD_U, FIELD_P, FIELD_SD;
# remote_halo_driver.c invoke_pack_or_unpack).
_FIELD_MEMBERS = {
    2: ("density", "energy0", "energy", "u", "p", "sd"),
    3: ("density", "energy0", "energy", "vec_u", "vec_p", "vec_sd"),
}


@dataclass(frozen=True)
class ChunkBox:
    """One chunk of the decomposed mesh."""

    index: int
    cells: Tuple[int, ...]       # interior cells along x, y(, z)
    lo: Tuple[int, ...]          # first global cell along x, y(, z): left, bottom(, back)
    neighbours: Tuple[int, ...]  # chunk per face (left, right, bottom, top(, back, front)), -1 external

    @property
    def hi(self) -> Tuple[int, ...]:
        return tuple(l + n for l, n in zip(self.lo, self.cells))


def chunk_counts(cells: Sequence[int], num_chunks: int) -> Tuple[int, ...]:
    """Chunks along x, y(, z): the first factorisation of num_chunks, in the
    reference's search order, with the least squared-extent sum per chunk
    volume (2d/initialise.c:43-71, 3d/initialise.c:43-85)."""
    if num_chunks < 1:
        raise ValueError("num_chunks must be at least 1 (got %d)" % num_chunks)
    ext = [float(c) for c in cells]
    best, found = math.inf, None
    if len(cells) == 2:
        for xx in range(1, num_chunks + 1):
            if num_chunks % xx:
                continue
            yy = num_chunks // xx
            a, b = ext[0] / xx, ext[1] / yy
            metric = ((a * a + b * b) * 2) / (a * b)
            if metric < best:
                best, found = metric, (xx, yy)
    elif len(cells) == 3:
        for xx in range(1, num_chunks + 1):
            if num_chunks % xx:
                continue
            wedge = num_chunks // xx
            for yy in range(1, wedge + 1):
                if wedge % yy:
                    continue
                zz = num_chunks // (xx * yy)
                a, b, c = ext[0] / xx, ext[1] / yy, ext[2] / zz
                metric = ((a * a + b * b + c * c) * 2) / (a * b * c)
                if metric < best:
                    best, found = metric, (xx, yy, zz)
    else:
        raise ValueError("cells must give 2 or 3 extents")
    if found is None:
        raise ValueError("failed to decompose the field with given parameters")
    return found


def decompose(cells: Sequence[int], num_chunks: int) -> List[ChunkBox]:
    """Every chunk of the mesh (decompose_field): chunk index
    xx + yy*X (+ zz*X*Y); along each axis the first (cells % count) chunks
    take one cell more, and each chunk starts where the previous ended."""
    counts = chunk_counts(cells, num_chunks)
    dims = len(cells)
    strides = [1, counts[0], counts[0] * (counts[1] if dims > 1 else 1)][:dims]
    per_axis = []
    for n, cnt in zip(cells, counts):
        base, extra = divmod(n, cnt)
        per_axis.append([(k * base + min(k, extra), base + (1 if k < extra else 0)) for k in range(cnt)])
        if base < 1:
            raise ValueError("%d cells cannot be split into %d chunks" % (n, cnt))
    boxes = []
    for index in range(num_chunks):
        pos = [(index // strides[a]) % counts[a] for a in range(dims)]
        nb = []
        for a in range(dims):
            nb.append(index - strides[a] if pos[a] > 0 else EXTERNAL_FACE)
            nb.append(index + strides[a] if pos[a] < counts[a] - 1 else EXTERNAL_FACE)
        boxes.append(ChunkBox(index=index,
                              cells=tuple(per_axis[a][pos[a]][1] for a in range(dims)),
                              lo=tuple(per_axis[a][pos[a]][0] for a in range(dims)),
                              neighbours=tuple(nb)))
    return boxes


Packer = Callable[[int, int, object, int, bool], None]


class FaceExchange:
    """The remote halo exchange of one chunk (remote_halo_driver.c:11-128).

    `pack(face, depth, field, address, is_pack)` packs the face of `field`
    into (or unpacks it from) face_len(face, depth) doubles at `address`;
    messages live on `device` (cuda under NCCL, cpu under gloo)."""

    def __init__(self, box: ChunkBox, group=None, device: Optional[torch.device] = None):
        self.box = box
        self.group = group
        self.device = device if device is not None else torch.device("cpu")
        self._buffers = {}   # (face, doubles) -> (send, recv); free again once run() returns

    def _pair(self, face: int, count: int):
        key = (face, count)
        if key not in self._buffers:
            send = torch.empty(count, dtype=torch.float64, device=self.device)
            self._buffers[key] = (send, torch.empty_like(send))
        return self._buffers[key]

    def face_len(self, face: int, depth: int) -> int:
        n = depth
        for a, c in enumerate(self.box.cells):
            if a != face // 2:
                n *= c
        return n

    def _peer(self, chunk: int) -> int:
        return chunk if self.group is None else dist.get_global_rank(self.group, chunk)

    def run(self, depth: int, fields: Sequence[object], pack: Packer) -> None:
        if not fields:
            return
        for axis in range(len(self.box.cells)):
            ops, received = [], []
            for face in (2 * axis, 2 * axis + 1):
                nb = self.box.neighbours[face]
                if nb == EXTERNAL_FACE:
                    continue
                n = self.face_len(face, depth)
                send, recv = self._pair(face, n * len(fields))
                for k, f in enumerate(fields):
                    pack(face, depth, f, send.data_ptr() + 8 * k * n, True)
                peer = self._peer(nb)
                ops.append(dist.P2POp(dist.isend, send, peer, self.group))
                ops.append(dist.P2POp(dist.irecv, recv, peer, self.group))
                received.append((face, n, recv))
            if ops:
                for work in dist.batch_isend_irecv(ops):
                    work.wait()
                if self.device.type == "cuda":
                    torch.cuda.current_stream(self.device).synchronize()
            for face, n, recv in received:
                for k, f in enumerate(fields):
                    pack(face, depth, f, recv.data_ptr() + 8 * k * n, False)


class DistHost(Host):
    """tealeaf_b200.host.Host on this rank's chunk of the decomposed mesh.

    Needs an initialised torch.distributed process group (`group`, default
    the world); rank r owns chunk r. Messages and the rank sums use `device`:
    by default the current CUDA device under NCCL, the host otherwise. The
    suite library (its own statically linked CUDA runtime) is pointed at
    `gpu`: by default the message device's index under NCCL, else the
    library's default device."""

    def __init__(self, tea_in: str, dims: int = 2, group=None, device: Optional[torch.device] = None,
                 gpu: Optional[int] = None, lib=None):
        if not dist.is_available() or not dist.is_initialized():
            raise DriverError("DistHost needs an initialised torch.distributed process group")
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if device is None:
            device = (torch.device("cuda", torch.cuda.current_device())
                      if dist.get_backend(group) == "nccl" else torch.device("cpu"))
        self.device = device
        self.gpu = gpu if gpu is not None else (device.index if device.type == "cuda" else None)
        self._lib_override = lib
        # every rank takes part in the group's first operation (NCCL creates its
        # communicator there; a first point-to-point batch must involve all ranks)
        dist.all_reduce(torch.zeros(1, dtype=torch.float64, device=device), group=group)
        super().__init__(tea_in, dims)

    # -- chunk and settings (2d/initialise.c:34-134 for this rank) -------------------
    def _load_lib(self):
        if self._lib_override is not None:
            return self._lib_override
        lib = super()._load_lib()
        if self.gpu is not None:
            getattr(lib, "tl%dd_set_device" % self.dims)(self.gpu)
        return lib

    def _fill_settings(self):
        super()._fill_settings()
        s = self.settings
        s.rank = self.rank
        s.num_ranks = s.num_chunks = self.world
        s.num_chunks_per_rank = 1

    def _initialise_chunk(self):
        c, hd = self.cfg, self.cfg.halo_depth
        cells = (c.grid_x_cells, c.grid_y_cells) + ((c.grid_z_cells,) if self.dims == 3 else ())
        try:
            box = decompose(cells, self.world)[self.rank]
        except ValueError as e:
            raise DriverError(str(e)) from None
        if min(box.cells) < hd:
            raise DriverError("chunk %d has %s cells, fewer than the halo depth %d" % (box.index, box.cells, hd))
        self.box = box
        self.exchange = FaceExchange(box, self.group, self.device)
        ch = self.chunk
        ch.x = box.cells[0] + 2 * hd
        ch.y = box.cells[1] + 2 * hd
        ch.left, ch.right = box.lo[0], box.hi[0]
        ch.bottom, ch.top = box.lo[1], box.hi[1]
        if self.dims == 3:
            ch.z = box.cells[2] + 2 * hd
            ch.back, ch.front = box.lo[2], box.hi[2]
        ch.dt_init = c.dt_init
        nb = (C.c_int * 6)(*(list(box.neighbours) + [EXTERNAL_FACE] * (6 - len(box.neighbours))))
        ext = abi.ChunkExtension()
        self._keep += [nb, ext]
        ch.neighbours = C.cast(nb, C.POINTER(C.c_int))
        ch.ext = C.pointer(ext)

    # -- halo_update_driver: remote faces, then the local halos -----------------------
    def halo_update(self, depth):
        fields = [f for f in range(6) if self.flags[f]]
        if not fields:
            return
        members = _FIELD_MEMBERS[self.dims]
        self.exchange.run(depth, [getattr(self.chunk, members[f]) for f in fields], self._pack)
        self._call("run_local_halos", depth)

    def _pack(self, face, depth, field, address, is_pack):
        self._call("run_pack_or_unpack", depth, face, is_pack, field,
                   C.cast(C.c_void_p(address), C.POINTER(C.c_double)))

    # -- sum_over_ranks (2d/comms.c:55-61) ----------------------------------------------
    def _sum(self, value: float) -> float:
        """The ranks' values added in rank order, ((v0 + v1) + v2) + ..., on
        every rank: the same rounding whatever the backend's reduction
        algorithm, and the order of the MPI stand-in the reference's own
        multi-rank runs are checked with."""
        t = torch.tensor([value], dtype=torch.float64, device=self.device)
        parts = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(parts, t, group=self.group)
        vals = torch.cat(parts).tolist()
        acc = vals[0]
        for v in vals[1:]:
            acc += v
        return acc

    # -- the device-resident forms hold no exchange -------------------------------------
    def _one_chunk_only(self, what):
        if self.world > 1:
            raise DriverError("%s solves one undivided chunk; a decomposed mesh runs through run_*" % what)

    def solve_device(self, tt: int, summary: bool = True):
        self._one_chunk_only("the device-resident timestep")
        return super().solve_device(tt, summary)

    def refine_step(self, tt: int, rel_tol: float, precision: int, summary: bool = True):
        self._one_chunk_only("the refinement form")
        return super().refine_step(tt, rel_tol, precision, summary)

    def adjoint_gradient(self, steps: int, every: int, box, rel_tol: float):
        self._one_chunk_only("the adjoint form")
        return super().adjoint_gradient(steps, every, box, rel_tol)

    # -- the whole mesh from every rank's chunk -------------------------------------------
    def gather_interior(self, name: str) -> np.ndarray:
        """The interior of field `name` over the whole mesh, on every rank
        (array order z, y, x as download)."""
        hd = self.cfg.halo_depth
        inner = np.ascontiguousarray(self.download(name)[(slice(hd, -hd),) * self.dims])
        parts: List[object] = [None] * self.world
        dist.all_gather_object(parts, (self.box, inner), group=self.group)
        c = self.cfg
        shape = (c.grid_x_cells, c.grid_y_cells) + ((c.grid_z_cells,) if self.dims == 3 else ())
        out = np.empty(shape[::-1], dtype=np.float64)
        for box, arr in parts:
            out[tuple(slice(l, h) for l, h in zip(box.lo[::-1], box.hi[::-1]))] = arr
        return out
