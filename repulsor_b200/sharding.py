"""Row-sharded evaluation of one mesh over several GPUs (one process per GPU).

The reference evaluates the rows of the Near() and Far() lists on host threads, splits
them by nonzero count and adds the per-thread derivative slices before the chain rule
(src/FMM/FMM_Traversor.hpp:56-147, src/ClusterTree.hpp:1115-1208). Here every process
holds the same mesh at the same coordinates and evaluates a contiguous range of row tiles
of the *full* symmetric patterns (`rpb_tpe0_pairs_shard`). A row accumulates only its own
derivative, so the shards' rows are disjoint: each process sends only the rows it owns
(one all-gather over the process group, NCCL between GPUs), every process places the
other shards' rows into its buffer and adds the shards' energy parts in shard order, and
then applies the chain rule and the vertex gather (`rpb_tpe0_collect_shards`). The buffer
holds the moment derivatives of the primitives (10 N) and clusters (10 N_C) and
the energy part (1); an all-gather moves each row once, half the bytes of a ring
all-reduce of the whole buffer, and adds nothing but the energy parts.
"""
from __future__ import annotations

import ctypes

from . import _capi
from ._capi import check

FAR_DIM = 10    # doubles per row of a shard buffer (moment derivatives)


def shard_range(count: int, shards: int, shard: int) -> tuple[int, int]:
    """The items [first, last) of `shard` when `count` items are split into `shards`
    contiguous ranges of sizes differing by at most one (the tiles of a pattern)."""
    if shards < 1 or not 0 <= shard < shards:
        raise ValueError("shard out of range")
    return count * shard // shards, count * (shard + 1) // shards


def exchange_layout(near_rows, far_rows, n_simplices: int, near_dim: int = FAR_DIM, far_dim: int = FAR_DIM):
    """Pieces of the shard buffer each shard owns and the length of one all-gather chunk.

    near_rows / far_rows: per shard, [first, last) rows of Near() and Far() (tree order).
    The buffer holds near_dim doubles per primitive, then far_dim per cluster, then the
    energy part (the device's buffers: 10 and 10).
    Returns (pieces, chunk): pieces[s] = [(offset, length), (offset, length)] in doubles of
    the buffer (the near rows, then the far rows, which start at near_dim N); chunk = the
    longest shard's row doubles + 1 (the last double of a chunk carries that shard's energy)."""
    if len(near_rows) != len(far_rows) or not near_rows:
        raise ValueError("one near and one far row range per shard")
    pieces = []
    for (a, b), (c, d) in zip(near_rows, far_rows):
        if not (0 <= a <= b and 0 <= c <= d):
            raise ValueError("row ranges must be [first, last) with first <= last")
        pieces.append([(near_dim * a, near_dim * (b - a)), (near_dim * n_simplices + far_dim * c, far_dim * (d - c))])
    chunk = max(sum(n for _, n in p) for p in pieces) + 1
    return pieces, chunk


def pack_owned(buf, pieces, chunk, out):
    """Copies this shard's rows and its energy part (buf[-1]) into `out` (chunk doubles)."""
    at = 0
    for off, n in pieces:
        out[at:at + n].copy_(buf[off:off + n])
        at += n
    out[chunk - 1] = buf[-1]


def unpack_gathered(buf, gathered, pieces_all, chunk, own):
    """Places the other shards' rows from `gathered` (shards x chunk) into `buf` and sets
    buf[-1] to the sum of all shards' energy parts, added in shard order."""
    for s, pieces in enumerate(pieces_all):
        if s == own:
            continue
        at = 0
        for off, n in pieces:
            buf[off:off + n].copy_(gathered[s, at:at + n])
            at += n
    energy = gathered[0, chunk - 1].clone()
    for s in range(1, len(pieces_all)):
        energy += gathered[s, chunk - 1]
    buf[-1] = energy


def exchange_rows(buf, pieces_all, chunk, rank, group=None, send=None, gathered=None):
    """The data-path exchange of a sharded evaluation: one all-gather of every shard's
    owned rows, after which `buf` on every rank holds the sum of all shards' buffers.
    Returns the number of doubles this rank received."""
    import torch
    import torch.distributed as dist

    world = len(pieces_all)
    if send is None:
        send = torch.empty(chunk, dtype=buf.dtype, device=buf.device)
    if gathered is None:
        gathered = torch.empty((world, chunk), dtype=buf.dtype, device=buf.device)
    pack_owned(buf, pieces_all[rank], chunk, send)
    dist.all_gather_into_tensor(gathered.view(-1), send, group=group)
    unpack_gathered(buf, gathered, pieces_all, chunk, rank)
    return (world - 1) * chunk


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
        dev = torch.device("cuda", torch.cuda.current_device())
        self.buf = torch.zeros(n.value, dtype=torch.float64, device=dev)
        self.stream = torch.cuda.ExternalStream(M.stream())
        near, far = zip(*(self.rows(s) for s in range(self.world)))
        self.pieces, self.chunk = exchange_layout(list(near), list(far), int(M.stats()["simplex_count"]))
        self.send = torch.empty(self.chunk, dtype=torch.float64, device=dev)
        self.gathered = torch.empty((self.world, self.chunk), dtype=torch.float64, device=dev)
        self.received_doubles = 0

    def rows(self, shard=None):
        """(near rows, far rows) of `shard` (default: this rank), each [first, last) in tree order."""
        nr = (ctypes.c_int64 * 2)()
        fr = (ctypes.c_int64 * 2)()
        s = self.rank if shard is None else shard
        check(_capi.load().rpb_mesh_shard_rows(self.M._h, s, nr, fr), "rpb_mesh_shard_rows")
        return (nr[0], nr[1]), (fr[0], fr[1])

    def __call__(self, Y_dev_ptr: int, ldY: int = 3, alpha: float = 1.0, beta: float = 0.0, want_energy=True):
        """Y = alpha dE + beta Y (device pointer, n_v x ldY float64, the mesh stream).
        Returns the energy (synchronizing) or None."""
        import torch

        lib = _capi.load()
        check(lib.rpb_tpe0_pairs_shard(self.M._h, self.energy.q, self.energy.p, self.rank,
                                       ctypes.c_void_p(self.buf.data_ptr())), "rpb_tpe0_pairs_shard")
        if self.world > 1:
            done = torch.cuda.Event()
            done.record(self.stream)
            cur = torch.cuda.current_stream()
            cur.wait_event(done)
            self.received_doubles = exchange_rows(self.buf, self.pieces, self.chunk, self.rank, self.group,
                                                  self.send, self.gathered)
            exchanged = torch.cuda.Event()
            exchanged.record(cur)
            self.stream.wait_event(exchanged)
        check(lib.rpb_tpe0_collect_shards(self.M._h, ctypes.c_void_p(self.buf.data_ptr()), float(alpha), float(beta),
                                          ctypes.c_void_p(Y_dev_ptr), ldY), "rpb_tpe0_collect_shards")
        if not want_energy:
            return None
        self.stream.synchronize()
        return float(self.buf[-1].item())
