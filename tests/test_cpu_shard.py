"""Sharding of the batched workload across ranks (host logic, CPU only).

Two gloo ranks on 127.0.0.1 each take their size-balanced shard of a batch
of small pencils, solve it with the LAPACK oracle standing in for the
device kernel, and gather eigenvalues on rank 0, which checks that every
pencil was solved exactly once and that the result equals a single-process
solve of the whole batch."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_balance_partition_properties(pkg):
    sh = pkg.shard
    sizes = pkg.pencils.batch_sizes(2048, 4)
    for world in (1, 2, 4, 8):
        parts, load = sh.balance(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        assert sh.imbalance(load) < 1.01
        assert parts == sh.balance(sizes, world)[0]  # deterministic


def _worker(rank, world, port, sizes, out_path):
    import importlib.util
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    spec = importlib.util.spec_from_file_location("gevp_pdhgeqz_b200", os.path.join(root, "gevp-pdhgeqz_b200",
                                                                                      "__init__.py"))
    pkg = importlib.util.module_from_spec(spec)
    sys.modules["gevp_pdhgeqz_b200"] = pkg
    spec.loader.exec_module(pkg)
    from oracle import lapack as L
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    mine = pkg.shard.shard(sizes, rank, world)
    res = {}
    for i in mine:
        H, T = pkg.pencils.batched_pencil(i, sizes[i], seed=9)
        _, _, ar, ai, be, _, _, info = L.dhgeqz(H, T, "E", "N", "N")
        assert info == 0
        res[i] = (ar, ai, be)
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    if rank == 0:
        import pickle
        with open(out_path, "wb") as f:
            pickle.dump(gathered, f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_batch(pkg, lapack, tmp_path):
    import pickle
    import torch.multiprocessing as mp
    sizes = [int(v) for v in pkg.pencils.batch_sizes(24, 9, 4, 40)]
    out = str(tmp_path / "gathered.pkl")
    mp.start_processes(_worker, args=(2, _free_port(), sizes, out), nprocs=2, join=True, start_method="spawn")
    with open(out, "rb") as f:
        gathered = pickle.load(f)
    seen = {}
    for part in gathered:
        for i, v in part.items():
            assert i not in seen
            seen[i] = v
    assert sorted(seen) == list(range(len(sizes)))
    for i, n in enumerate(sizes):
        H, T = pkg.pencils.batched_pencil(i, n, seed=9)
        _, _, ar, ai, be, _, _, _ = lapack.dhgeqz(H, T, "E", "N", "N")
        for a, b in zip(seen[i], (ar, ai, be)):
            assert np.array_equal(a, b)
