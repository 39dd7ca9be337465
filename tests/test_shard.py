"""Sharding of the batched workloads over ranks (blood_network_b200/shard.py):
the partitions, and the gather over a world_size-2 gloo process group on the
CPU with a direct sparse solve standing in for the GPU solver."""
import os
import socket
import tempfile

import numpy as np
import pytest

from blood_network_b200.shard import partition_columns, partition_networks


def test_partition_networks_balanced_and_complete():
    rng = np.random.default_rng(0)
    nnz = rng.integers(10_000, 1_000_000, 257)
    for ws in (1, 2, 3, 8):
        parts = partition_networks(nnz, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(nnz)))
        loads = [int(nnz[p].sum()) if p else 0 for p in parts]
        assert max(loads) <= nnz.sum() / ws + nnz.max()
        assert parts == partition_networks(nnz, ws)  # deterministic
    assert partition_networks([5], 4) == [[0], [], [], []]


def test_partition_columns():
    for k, ws in ((64, 8), (64, 3), (5, 8), (0, 2)):
        cols = partition_columns(k, ws)
        sizes = [len(c) for c in cols]
        assert sum(sizes) == k and max(sizes) - min(sizes) <= 1
        assert [c.start for c in cols] == sorted(c.start for c in cols)


def _spsolve_nets(nets):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    out = []
    for nt in nets:
        A = sp.csr_matrix((nt.data, nt.indices, nt.indptr), shape=(nt.n, nt.n)).tocsc()
        out.append((spla.spsolve(A, nt.rhs), 1))
    return out


def _nets():
    from blood_network_b200.network import vascular_network
    return [vascular_network(depth=5, n_nodes=200 + 150 * k, seed=k, keep_segments=False)
            for k in range(7)]


def _worker(rank, ws, port, outdir):
    import torch.distributed as dist
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    from blood_network_b200.shard import solve_columns_distributed, solve_networks_distributed
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=ws)
    try:
        nets = _nets()
        res = solve_networks_distributed(nets, _spsolve_nets)
        ref = _spsolve_nets(nets)
        ok1 = all(np.array_equal(a[0], b[0]) for a, b in zip(res, ref))
        nt = nets[3]
        A = sp.csr_matrix((nt.data, nt.indices, nt.indptr), shape=(nt.n, nt.n)).tocsc()
        B = np.asfortranarray(np.random.default_rng(1).standard_normal((nt.n, 5)))

        def solve_block(Bb):
            return spla.spsolve(A, Bb).reshape(nt.n, -1), np.ones(Bb.shape[1], np.int32)

        X, its = solve_columns_distributed(B, solve_block)
        ok2 = X.shape == B.shape and np.allclose(A @ X, B) and its.shape == (5,)
        with open(os.path.join(outdir, f"rank{rank}"), "w") as f:
            f.write(f"{int(ok1)}{int(ok2)}")
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gather_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(2, _free_port(), d), nprocs=2, join=True)
        for r in range(2):
            assert open(os.path.join(d, f"rank{r}")).read() == "11"


def _bench_worker(rank, ws, port, outdir):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=ws)
    try:
        bench.barrier(ws)
        m = bench.max_over_ranks(0.5 + rank, ws)  # the bench's max-over-ranks timing
        with open(os.path.join(outdir, f"rank{rank}"), "w") as f:
            f.write(repr(m))
    finally:
        dist.destroy_process_group()


def test_bench_max_over_ranks_on_two_gloo_ranks():
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_bench_worker, args=(2, _free_port(), d), nprocs=2, join=True)
        assert [float(open(os.path.join(d, f"rank{r}")).read()) for r in range(2)] == [1.5, 1.5]
