"""Row-sharded evaluation of one mesh over several GPUs (one process per GPU).

The reference evaluates the rows of the Near() and Far() lists on host threads, splits
them by nonzero count and adds the per-thread derivative slices before the chain rule
(src/FMM/FMM_Traversor.hpp:56-147, src/ClusterTree.hpp:1115-1208). Here every process
holds the same mesh at the same coordinates, evaluates a contiguous range of row tiles
(`rpb_tpe0_pairs_shard`), the partial buffers are summed with one all-reduce over the
process group (NCCL between GPUs), and every process applies the chain rule and the
vertex gather to the sum (`rpb_tpe0_collect_shards`). The buffer holds the centred moment
derivatives of the primitives (10 N) and clusters (10 N_C) and the energy part (1).
"""
from __future__ import annotations

import ctypes

from . import _capi
from ._capi import check


def shard_range(count: int, shards: int, shard: int) -> tuple[int, int]:
    """The items [first, last) of `shard` when `count` items are split into `shards`
    contiguous ranges of sizes differing by at most one (the tiles of a pattern)."""
    if shards < 1 or not 0 <= shard < shards:
        raise ValueError("shard out of range")
    return count * shard // shards, count * (shard + 1) // shards


class ShardedDifferential:
    """Differential of `energy` (a TangentPointEnergy0) on mesh `M`, row-sharded over the
    ranks of `group` (torch.distributed, default group). Every rank constructs it for its
    own copy of the mesh; calls are collective (every rank calls in the same order)."""

    def __init__(self, M, energy, group=None):
        import torch
        import torch.distributed as dist

        self.M, self.energy, self.group = M, energy, group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        lib = _capi.load()
        check(lib.rpb_mesh_set_shards(M._h, self.world), "rpb_mesh_set_shards")
        n = ctypes.c_int64()
        check(lib.rpb_mesh_shard_buffer_doubles(M._h, ctypes.byref(n)), "rpb_mesh_shard_buffer_doubles")
        self.buf = torch.zeros(n.value, dtype=torch.float64, device=torch.device("cuda", torch.cuda.current_device()))
        self.stream = torch.cuda.ExternalStream(M.stream())

    def rows(self):
        """(near rows, far rows) of this rank, each [first, last) in tree order."""
        nr = (ctypes.c_int64 * 2)()
        fr = (ctypes.c_int64 * 2)()
        check(_capi.load().rpb_mesh_shard_rows(self.M._h, self.rank, nr, fr), "rpb_mesh_shard_rows")
        return (nr[0], nr[1]), (fr[0], fr[1])

    def __call__(self, Y_dev_ptr: int, ldY: int = 3, alpha: float = 1.0, beta: float = 0.0, want_energy=True):
        """Y = alpha dE + beta Y (device pointer, n_v x ldY float64, the mesh stream).
        Returns the energy (synchronizing) or None."""
        import torch
        import torch.distributed as dist

        lib = _capi.load()
        check(lib.rpb_tpe0_pairs_shard(self.M._h, self.energy.q, self.energy.p, self.rank,
                                       ctypes.c_void_p(self.buf.data_ptr())), "rpb_tpe0_pairs_shard")
        if self.world > 1:
            done = torch.cuda.Event()
            done.record(self.stream)
            cur = torch.cuda.current_stream()
            cur.wait_event(done)
            dist.all_reduce(self.buf, op=dist.ReduceOp.SUM, group=self.group)
            reduced = torch.cuda.Event()
            reduced.record(cur)
            self.stream.wait_event(reduced)
        check(lib.rpb_tpe0_collect_shards(self.M._h, ctypes.c_void_p(self.buf.data_ptr()), float(alpha), float(beta),
                                          ctypes.c_void_p(Y_dev_ptr), ldY), "rpb_tpe0_collect_shards")
        if not want_energy:
            return None
        self.stream.synchronize()
        return float(self.buf[-1].item())
