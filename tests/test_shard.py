"""The multi-process paths on CPU: the batch sharding of waltz_b200.shard
(partition by bytes, archive-size exchange) and the benchmark's max-over-ranks
timing, with world_size-2 gloo process groups (no GPU). The chunk archives of
the sharded run come from the oracle, so the shared result can be checked
against one process compressing the whole list."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from waltz_b200 import shard


def test_partition_covers_and_balances():
    rng = np.random.default_rng(4)
    sides = np.array([32, 48, 64, 96, 128])
    sizes = [int(np.prod(rng.choice(sides, 3))) * 4 for _ in range(512)]
    for world in (1, 2, 3, 4, 8):
        shares = shard.partition(sizes, world)
        assert len(shares) == world
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(sizes)))
        assert all(s == sorted(s) for s in shares)
        loads = [sum(sizes[i] for i in s) for s in shares]
        assert max(loads) - sum(loads) / world <= max(sizes)
        assert shares == shard.partition(sizes, world)  # deterministic: every rank agrees


def test_partition_edge_cases():
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5], 2) == [[0], []]
    assert shard.partition([7, 7, 7, 7], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.partition([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _chunks():
    rng = np.random.default_rng(11)
    out = []
    for k in range(12):
        shape = tuple(int(v) for v in rng.choice([8, 12, 16, 24], 3))
        out.append((rng.standard_normal(shape).cumsum(axis=2) * 0.1).astype(np.float32))
    return out


def _worker(rank, world, port, result_dir):
    import torch.distributed as dist
    from oracle import oracle as O
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        chunks = _chunks()
        mine = shard.my_share([c.nbytes for c in chunks], rank, world)
        local = {i: O.compress(chunks[i], 1e-3) for i in mine}
        sizes, offsets = shard.exchange_sizes({i: len(a) for i, a in local.items()})
        # the archives of all ranks, laid out in chunk order, gathered on rank 0
        parts = [None] * world
        dist.all_gather_object(parts, local)
        worst = bench.dist_max(float(rank + 1), world)
        if rank == 0:
            merged = {}
            for p in parts:
                merged.update(p)
            blob = b"".join(merged[i] for i in sorted(merged))
            np.save(os.path.join(result_dir, "sizes.npy"), np.array([sizes[i] for i in sorted(sizes)]))
            np.save(os.path.join(result_dir, "offsets.npy"), np.array([offsets[i] for i in sorted(offsets)]))
            with open(os.path.join(result_dir, "blob.bin"), "wb") as fh:
                fh.write(blob)
            with open(os.path.join(result_dir, "max.txt"), "w") as fh:
                fh.write(repr(worst))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_batch_over_gloo(tmp_path):
    """Two gloo ranks compress their shares of a 12-chunk list; the exchanged
    sizes and offsets describe a container equal to one process compressing
    every chunk, and the max-over-ranks timing helper returns the larger
    rank's value."""
    import torch.multiprocessing as mp
    from oracle import oracle as O
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    chunks = _chunks()
    expect = [O.compress(c, 1e-3) for c in chunks]
    sizes = np.load(tmp_path / "sizes.npy")
    offsets = np.load(tmp_path / "offsets.npy")
    assert list(sizes) == [len(a) for a in expect]
    assert list(offsets) == list(np.concatenate([[0], np.cumsum(sizes)[:-1]]))
    assert (tmp_path / "blob.bin").read_bytes() == b"".join(expect)
    assert float((tmp_path / "max.txt").read_text()) == 2.0
