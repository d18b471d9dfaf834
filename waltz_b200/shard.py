"""Sharding of the batched form across GPUs (one process per GPU).

Chunks of a batch are independent archives, so a batch shards without any
data-path collective: every rank takes a share of the chunk list, balanced
by bytes, and compresses or decodes it on its own GPU. The only exchange is
of metadata, each chunk's archive size, when the ranks' archives are to be
laid out in one container (a prefix over the sizes in chunk order).

`partition` is deterministic (every rank computes the same shares from the
same size list); `exchange_sizes` runs over any torch.distributed process
group (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations


def partition(sizes, world):
    """Chunk indices per rank, balanced by bytes: chunks in decreasing size
    (ties by index) each go to the rank with the fewest bytes so far (ties by
    rank). Every index appears in exactly one share; a share's bytes exceed
    the mean by at most the largest chunk. Shares list their indices in
    increasing order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0] * world
    shares = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        shares[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(s) for s in shares]


def my_share(sizes, rank, world):
    return partition(sizes, world)[rank]


def exchange_sizes(local, group=None):
    """Every rank's {chunk index: archive bytes} merged on every rank (one
    all-gather of small objects), with the archive offsets of a container
    that stores the archives in chunk order: returns (sizes, offsets) as
    dicts over all chunk indices."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, {int(k): int(v) for k, v in local.items()}, group=group)
    sizes = {}
    for p in parts:
        for k, v in p.items():
            if k in sizes:
                raise ValueError(f"chunk {k} compressed on two ranks")
            sizes[k] = v
    offsets, at = {}, 0
    for k in sorted(sizes):
        offsets[k] = at
        at += sizes[k]
    return sizes, offsets
