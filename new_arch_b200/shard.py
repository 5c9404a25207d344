"""Chain shards: one SCMF system spread over several GPUs (scmf_shard_* in
include/scmf.h).

The reference's multi-GPU scheme splits a system's chains over GPUs
(init_config.cu:220-222), sums the per-GPU integer density counts
(mesh.cu:10-81 P2P, mesh_mpi.cpp:16 MPI_Allreduce) and hands every GPU the
summed field (mesh.cu:191-215).  Here each rank (one process per GPU) holds a
`Shard`; the sum of the counts is one NCCL all-reduce of n_types * n_cells
int32 words per sweep over NVLink (`ShardedSystem`), and every rank computes
the same field from the sum.  Positions and summed counts are bit-identical to
the whole system run on one GPU.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib
from .spec import SystemSpec


def shard_chains(spec: SystemSpec, shard: int, n_shards: int) -> Tuple[List[int], List[int]]:
    """(first chain, chain count) per architecture of shard `shard` of `n_shards`."""
    h = spec.to_c()
    try:
        n = len(spec.archs)
        first, count = (C.c_int32 * n)(), (C.c_int32 * n)()
        check(lib().scmf_shard_chains(h, int(shard), int(n_shards), first, count, n))
    finally:
        lib().scmf_spec_destroy(h)
    return list(first), list(count)


class Shard:
    """Chain shard `shard` of `n_shards` of the system `spec` describes, on the
    current CUDA device, its kernels enqueued on `stream` (a CUDA stream handle)."""

    def __init__(self, spec: SystemSpec, shard: int, n_shards: int, stream: Optional[int] = None):
        L = lib()
        self.spec = spec
        self.shard, self.n_shards = shard, n_shards
        h = spec.to_c()
        try:
            self._h = C.c_void_p()
            check(L.scmf_system_create_shard(h, int(shard), int(n_shards), C.c_void_p(stream) if stream else None,
                                             C.byref(self._h)))
        finally:
            L.scmf_spec_destroy(h)
        info = _lib.SpecInfo()
        check(L.scmf_system_get_info(self._h, C.byref(info)))
        self.n_beads, self.n_cells, self.n_types = info.n_beads, info.n_cells, info.n_types
        self.count_words = self.n_types * self.n_cells

    def init_coords(self, d_partial: int) -> None:
        check(lib().scmf_shard_init_coords(self._h, C.c_void_p(d_partial)))

    def move(self, d_partial: int) -> None:
        check(lib().scmf_shard_move(self._h, C.c_void_p(d_partial)))

    def field(self, d_total: int, close_sweep: bool = True) -> None:
        check(lib().scmf_shard_field(self._h, C.c_void_p(d_total), int(bool(close_sweep))))

    def coords(self) -> np.ndarray:
        out = np.empty(3 * self.n_beads, dtype=np.float32)
        check(lib().scmf_get_coords(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out.reshape(-1, 3)

    def counts(self) -> np.ndarray:
        """The shard's own counts (the grid of its beads)."""
        out = np.empty(self.count_words, dtype=np.uint32)
        check(lib().scmf_get_counts(self._h, out.ctypes.data_as(C.POINTER(C.c_uint32)), out.size))
        return out

    def omega(self) -> np.ndarray:
        out = np.empty(self.count_words, dtype=np.float32)
        check(lib().scmf_get_omega(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    def stats(self) -> dict:
        st = _lib.Stats()
        check(lib().scmf_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.Stats._fields_ if k != "reserved"}

    def synchronize(self) -> None:
        check(lib().scmf_synchronize(self._h))

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().scmf_system_destroy(h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ShardedSystem:
    """This rank's shard of one system spread over the ranks of a
    torch.distributed process group (backend "nccl", one GPU per rank); the
    per-sweep sum of the counts is an in-place all-reduce on the shard's stream
    (`stream`; time it with events recorded there)."""

    def __init__(self, spec: SystemSpec, group=None):
        import torch
        import torch.distributed as dist
        self._dist, self._group = dist, group
        if dist.is_available() and dist.is_initialized():
            rank, world = dist.get_rank(group), dist.get_world_size(group)
        else:                       # one process, one shard: the sum is the shard's own counts
            rank, world = 0, 1
        self.world = world
        # a stream of its own (never the legacy default stream, whose handle is 0,
        # which the C ABI reads as "make a private stream"): the shard's kernels and
        # the all-reduce are ordered on it
        self._torch = torch
        self.stream = torch.cuda.Stream()
        self.shard = Shard(spec, rank, world, self.stream.cuda_stream)
        with torch.cuda.stream(self.stream):
            self.buf = torch.zeros(self.shard.count_words, dtype=torch.int32, device="cuda")

    def _sum(self) -> None:
        if self.world > 1:
            with self._torch.cuda.stream(self.stream):
                self._dist.all_reduce(self.buf, op=self._dist.ReduceOp.SUM, group=self._group)

    def init_coords(self) -> None:
        self.shard.init_coords(self.buf.data_ptr())
        self._sum()
        self.shard.field(self.buf.data_ptr(), close_sweep=False)

    def step(self, n_sweeps: int = 1) -> None:
        for _ in range(n_sweeps):
            self.shard.move(self.buf.data_ptr())
            self._sum()
            self.shard.field(self.buf.data_ptr(), close_sweep=True)

    def counts(self) -> np.ndarray:
        """The summed counts of the last sweep (the whole system's)."""
        self.stream.synchronize()
        return self.buf.cpu().numpy().view(np.uint32)

    def close(self) -> None:
        self.shard.close()
