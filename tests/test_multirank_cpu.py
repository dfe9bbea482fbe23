"""Multi-rank paths on CPU with the gloo backend, world size 2 (no GPU):
the column sharding of one assembly (each rank assembles its shard with the
oracle, rank 0 merges the column blocks and compares them with the full
assembly) and the max-over-ranks timing reduction used by the benchmark."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    import datetime
    import sys

    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))


def _sharded_rank(rank, world, port):
    _init(rank, world, port)
    try:
        from emerge_b200 import workloads as W
        from emerge_b200.partition import extract_block, merge_blocks, shard_of
        from oracle import oracle as O

        wl = W.wr90_dielectric(n=(8, 5, 12), seed=4)
        f, m = wl.field, wl.field.mesh
        cond = np.arange(3, f.ntets, 41)
        k0 = wl.k0
        sh = shard_of(m, rank, world, cond)
        e, b, c = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, sh.excluded_tets(), nthreads=1)
        blk = extract_block(sh, c.indptr, c.indices, c.values_lincomb(e, b, 1.0, -k0 ** 2, 1))
        got = [None] * world
        dist.all_gather_object(got, (blk, sh.tetids.size, sh.est_nnz))
        if rank == 0:
            blocks = [g[0] for g in got]
            ip, ix, vv = merge_blocks(blocks, f.n_field)
            dE, dB, cm = O.tet_mass_stiffness_matrices(f, wl.er, wl.ur, cond, nthreads=1)
            ref = cm.values_lincomb(dE, dB, 1.0, -k0 ** 2, 1)
            assert np.array_equal(ip, cm.indptr) and np.array_equal(ix, cm.indices)
            assert np.array_equal(vv, ref)  # same tets, same order: bitwise
            nnz = [sum(x.size for x in g[0].indices) for g in got]
            assert max(nnz) <= 1.1 * min(nnz), nnz
            assert sum(g[1] for g in got) < 1.25 * (f.ntets - cond.size)  # halo overhead bounded
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _maxreduce_rank(rank, world, port):
    _init(rank, world, port)
    try:
        from emerge_b200.ranks import max_over_ranks, sum_over_ranks

        mx = max_over_ranks([1.0 + rank, 10.0 - rank])
        sm = sum_over_ranks([float(rank)])
        assert mx == [float(world), 10.0], mx
        assert sm == [float(sum(range(world)))]
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("fn", [_sharded_rank, _maxreduce_rank])
def test_world2_gloo(fn):
    mp.start_processes(fn, args=(2, _free_port()), nprocs=2, join=True, start_method="spawn")


def test_partition_single_process_covers_everything():
    from emerge_b200 import workloads as W
    from emerge_b200.partition import partition

    wl = W.wr90_air(n=(6, 4, 10))
    m = wl.field.mesh
    for world in (1, 2, 3, 7):
        sh = partition(m, world)
        assert sh[0].edge_lo == 0 and sh[-1].edge_hi == m.n_edges
        assert sh[0].face_lo == 0 and sh[-1].face_hi == m.n_tris
        for a, b in zip(sh, sh[1:]):
            assert a.edge_hi == b.edge_lo and a.face_hi == b.face_lo and a.node_hi == b.node_lo
        covered = np.zeros(m.n_tets, bool)
        for s in sh:
            covered[s.tetids] = True
        assert covered.all()
