"""Row-sharded evaluation of one mesh over several processes (repulsor_b200/sharding.py,
rpb_tpe0_pairs_shard / rpb_tpe0_collect_shards). CPU: the partition; two gloo ranks that
each evaluate one shard with the oracle (upper-triangle rows split like the reference's
threads), all-reduce the derivative slices and collect; and the exchange the GPU path
uses -- ranks that own disjoint rows of the full patterns all-gather only those rows (the
oracle's row-owned slices, and synthetic buffers on 2 and 3 ranks whose assembly must
equal the all-reduced sum and whose received bytes are about half a ring all-reduce's).
GPU: the shards of one mesh evaluated in turn on one GPU
and summed equal the unsharded Differential, and the torch.distributed driver with a
one-rank NCCL group equals it too (every GPU call of this build has one GPU)."""
import ctypes
import os
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from repulsor_b200 import meshes  # noqa: E402
from repulsor_b200.sharding import exchange_layout, exchange_rows, shard_range  # noqa: E402

Q, P = 6.0, 12.0


def test_shard_range_covers_contiguously_and_balanced():
    for count in (0, 1, 7, 296, 591, 1000):
        for shards in (1, 2, 3, 8):
            ranges = [shard_range(count, shards, s) for s in range(shards)]
            assert ranges[0][0] == 0 and ranges[-1][1] == count
            for (a, b), (c, d) in zip(ranges, ranges[1:]):
                assert b == c and a <= b
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _oracle_rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dom, (V, S) = meshes.config_mesh(2, small=True)
        O = oracle.OracleMesh(dom, V, S)
        Dn, Df, e = O.partial_derivatives(rank, world, Q, P)
        buf = torch.from_numpy(np.concatenate([Dn.ravel(), Df.ravel(), [e]]))
        dist.all_reduce(buf, op=dist.ReduceOp.SUM)
        b = buf.numpy()
        nd = Dn.size
        Y = O.collect(b[:nd].reshape(Dn.shape), b[nd:nd + Df.size].reshape(Df.shape))
        E_full, Y_full = O.differential(Q, P)
        out[rank] = (float(b[-1]), E_full, float(np.abs(Y - Y_full).max() / np.abs(Y_full).max()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_all_reduce_shard_slices_to_the_full_differential():
    world = 2
    port = 29600 + os.getpid() % 1000
    with mp.get_context("spawn").Manager() as manager:
        out = manager.dict()
        mp.spawn(_oracle_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        e, E_full, dy = res[r]
        assert abs(e - E_full) <= 1e-13 * abs(E_full)
        assert dy <= 1e-13


def _gather_rows_rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # the oracle's row-owned slices, exchanged by the all-gather of owned rows
        dom, (V, S) = meshes.config_mesh(2, small=True)
        O = oracle.OracleMesh(dom, V, S)
        N, NC = O.nS, O.counts()["clusters"]
        near = [shard_range(N, world, s) for s in range(world)]
        far = [shard_range(NC, world, s) for s in range(world)]
        Dn, Df, e = O.row_derivatives(near[rank], far[rank], Q, P)
        nd = Dn.shape[1]
        buf = torch.from_numpy(np.concatenate([Dn.ravel(), Df.ravel(), [e]]))
        pieces, chunk = exchange_layout(near, far, N, near_dim=nd, far_dim=10)
        received = exchange_rows(buf, pieces, chunk, rank)
        b = buf.numpy()
        Y = O.collect(b[:Dn.size].reshape(Dn.shape), b[Dn.size:Dn.size + Df.size].reshape(Df.shape))
        E_full, Y_full = O.differential(Q, P)
        res = [float(b[-1]), E_full, float(np.abs(Y - Y_full).max() / np.abs(Y_full).max()), received, buf.numel()]
        # synthetic buffers: random rows owned by this rank, zero elsewhere; the assembly
        # must equal the sum over ranks (bit for bit: each row has one owner)
        n_near, n_far = 1001 + 7 * world, 2003
        near = [shard_range(n_near, world, s) for s in range(world)]
        far = [shard_range(n_far, world, s) for s in range(world)]
        pieces, chunk = exchange_layout(near, far, n_near)

        def shard_buffer(s):
            g = np.random.default_rng(100 + s)
            x = np.zeros(10 * (n_near + n_far) + 1)
            for off, n in pieces[s]:
                x[off:off + n] = g.standard_normal(n)
            x[-1] = g.standard_normal()
            return x

        mine = torch.from_numpy(shard_buffer(rank))
        got = exchange_rows(mine, pieces, chunk, rank)
        want = np.sum([shard_buffer(s) for s in range(world)], axis=0)
        e_sum = 0.0
        for s in range(world):
            e_sum += shard_buffer(s)[-1]
        want[-1] = e_sum
        res += [bool(np.array_equal(mine.numpy(), want)), got, mine.numel()]
        out[rank] = res
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_all_gather_of_owned_rows_composes_the_full_differential(world):
    port = 29650 + world + os.getpid() % 900
    with mp.get_context("spawn").Manager() as manager:
        out = manager.dict()
        mp.spawn(_gather_rows_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        e, E_full, dy, received, total, exact, got, total2 = res[r]
        assert abs(e - E_full) <= 1e-13 * abs(E_full)
        assert dy <= 1e-12
        assert exact
        # received doubles: each other shard's rows once (+ its energy); a ring all-reduce
        # of the whole buffer moves 2 (W-1)/W of it through every rank
        for rec, n in ((received, total), (got, total2)):
            assert rec <= (world - 1) / world * n * 1.01 + world
            assert rec <= 0.51 * 2 * (world - 1) / world * n + world


@pytest.mark.gpu
@pytest.mark.parametrize("shards", [2, 3])
def test_shards_on_one_gpu_sum_to_the_differential(shards):
    import repulsor_b200 as rpb
    from repulsor_b200 import _capi

    lib = _capi.load()
    dom, (V, S) = meshes.config_mesh(2)
    M = rpb.SimplicialMesh(V, S)
    tpe = rpb.TangentPointEnergy0(Q, P)
    D_ref = np.zeros_like(V)
    E_ref = tpe.Differential(M, 1.0, 0.0, D_ref)
    _capi.check(lib.rpb_mesh_set_shards(M._h, shards), "set_shards")
    # the regrouped tiles give rows other lane groups, hence other FP32 partial sums: the
    # unsharded evaluation with the same tiles is the bit-level reference
    D_same = np.zeros_like(V)
    E_same = tpe.Differential(M, 1.0, 0.0, D_same)
    assert abs(E_same - E_ref) <= 1e-8 * abs(E_ref)
    assert np.abs(D_same - D_ref).max() <= 1e-6 * np.abs(D_ref).max()
    n = ctypes.c_int64()
    _capi.check(lib.rpb_mesh_shard_buffer_doubles(M._h, ctypes.byref(n)), "buffer")
    st = M.stats()
    assert n.value == 10 * st["simplex_count"] + 10 * st["cluster_count"] + 1
    total = torch.zeros(n.value, dtype=torch.float64, device="cuda")
    ext = torch.cuda.ExternalStream(M.stream())
    rows_near, rows_far = [], []
    for s in range(shards):
        buf = torch.full((n.value,), 7.0, dtype=torch.float64, device="cuda")   # the call must overwrite it
        torch.cuda.synchronize()
        _capi.check(lib.rpb_tpe0_pairs_shard(M._h, Q, P, s, ctypes.c_void_p(buf.data_ptr())), "pairs_shard")
        ext.synchronize()
        total += buf
        nr = (ctypes.c_int64 * 2)()
        fr = (ctypes.c_int64 * 2)()
        _capi.check(lib.rpb_mesh_shard_rows(M._h, s, nr, fr), "shard_rows")
        rows_near.append((nr[0], nr[1]))
        rows_far.append((fr[0], fr[1]))
    for rows, count in ((rows_near, st["simplex_count"]), (rows_far, st["cluster_count"])):
        assert rows[0][0] == 0 and rows[-1][1] == count
        assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
    Y = torch.zeros((V.shape[0], 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _capi.check(lib.rpb_tpe0_collect_shards(M._h, ctypes.c_void_p(total.data_ptr()), 1.0, 0.0,
                                            ctypes.c_void_p(Y.data_ptr()), 3), "collect")
    ext.synchronize()
    E = float(total[-1].item())
    D = Y.cpu().numpy()
    assert abs(E - E_same) <= 1e-12 * abs(E_same)
    assert np.abs(D - D_same).max() <= 1e-12 * np.abs(D_same).max()
    _capi.check(lib.rpb_mesh_set_shards(M._h, 1), "set_shards")
    D1 = np.zeros_like(V)
    assert tpe.Differential(M, 1.0, 0.0, D1) == pytest.approx(E_ref, rel=1e-13)


def _nccl_rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import repulsor_b200 as rpb
    from repulsor_b200.sharding import ShardedDifferential

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(rank)
    dist.init_process_group("nccl", rank=rank, world_size=world)
    try:
        dom, (V, S) = meshes.config_mesh(2)
        M = rpb.SimplicialMesh(V, S)
        tpe = rpb.TangentPointEnergy0(Q, P)
        D_ref = np.zeros_like(V)
        E_ref = tpe.Differential(M, 1.0, 0.0, D_ref)
        sd = ShardedDifferential(M, tpe)
        Y = torch.zeros((V.shape[0], 3), dtype=torch.float64, device="cuda")
        E = sd(Y.data_ptr())
        E2 = sd(Y.data_ptr(), alpha=1.0, beta=1.0)
        torch.cuda.synchronize()
        out[rank] = (E, E2, E_ref, float(np.abs(Y.cpu().numpy() - 2 * D_ref).max() / np.abs(D_ref).max()),
                     sd.rows())
        del sd
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_driver_with_one_nccl_rank_equals_the_differential():
    port = 29700 + os.getpid() % 1000
    with mp.get_context("spawn").Manager() as manager:
        out = manager.dict()
        mp.spawn(_nccl_rank, args=(1, port, out), nprocs=1, join=True)
        E, E2, E_ref, dy, rows = out[0]
    assert E == pytest.approx(E_ref, rel=1e-12) and E2 == pytest.approx(E_ref, rel=1e-12)
    assert dy <= 1e-12
    assert rows[0][0] == 0 and rows[1][0] == 0
