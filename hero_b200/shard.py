"""One correction split across devices by subject reads (the multi-GPU form).

Every subject read is independent given the read-only query table, and the
votes are integer sums, so a correction of N reads on W devices is: every rank
holds the whole query set and its k-mer table, aligns the subject reads of its
own contiguous range (``shard_range``) against it, and the ranks add their vote
states in one all-reduce (``allreduce_votes``: NCCL over NVLink for CUDA
buffers, gloo for host buffers); the consensus over the summed votes is then
the consensus of the whole run, on every rank.  This is HERO's own chunking
(SubjectReadAligner::start streams subject chunks into one vote matrix,
SubjectReadAligner.cpp:493-645) spread over devices.

    torchrun --nproc-per-node 8 prog.py   # each rank:
    res = correct_sharded(reads, aligner="affine")
"""
from __future__ import annotations


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous range [a, b) of n subject reads for rank of world (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    q, r = divmod(n, world)
    a = rank * q + min(rank, r)
    return a, a + q + (1 if rank < r else 0)


def _dist():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist
    return None


def world_rank() -> tuple[int, int]:
    d = _dist()
    return (d.get_world_size(), d.get_rank()) if d else (1, 0)


def allreduce_votes(buf) -> None:
    """Adds the ranks' vote states in place (int32 tensor; addition mod 2^32).

    The state's mismatch votes are unsigned and its match-run differences are
    signed; both are added as int32, whose wrap-around sum has the same bits as
    the unsigned and the signed sums."""
    import torch
    d = _dist()
    if d is None:
        return
    if buf.dtype != torch.int32:
        raise TypeError("vote states are int32 words")
    d.all_reduce(buf, op=d.ReduceOp.SUM)


def owner_slices(q_off, world: int, words_per_base: int = 4, tail_words: int = 1) -> list:
    """Each rank owns a contiguous range of query reads (shard_range) and the
    vote-state words of their bases: [(first_read, count, nbases, [(lo, hi), ...])]
    per rank.  The state is [bases][words_per_base] followed, when tail_words,
    by [bases][tail_words] (the device layout: 4 mismatch-vote words, then one
    match-run difference word per base)."""
    n = len(q_off) - 1
    nqb = int(q_off[-1]) if n else 0
    out = []
    for r in range(world):
        a, b = shard_range(n, r, world)
        b0, b1 = int(q_off[a]), int(q_off[b])
        sl = [(words_per_base * b0, words_per_base * b1)]
        if tail_words:
            base = words_per_base * nqb
            sl.append((base + tail_words * b0, base + tail_words * b1))
        out.append((a, b - a, b1 - b0, sl))
    return out


def reduce_votes_to_owners(buf, owners) -> None:
    """Adds the ranks' vote states slice by slice into each slice's owner, in
    place (one reduce per owned slice, NCCL over NVLink for CUDA buffers, gloo
    for host buffers): afterwards rank r's buffer holds the whole run's votes
    for its own reads; other slices are left as they were.  Half the bytes of
    an all-reduce of the whole state cross the links, and no copies are made."""
    import torch
    d = _dist()
    if d is None:
        return
    if buf.dtype != torch.int32:
        raise TypeError("vote states are int32 words")
    for r, (_, _, _, slices) in enumerate(owners):
        for lo, hi in slices:
            if hi > lo:
                d.reduce(buf[lo:hi], dst=r, op=d.ReduceOp.SUM)


def max_over_ranks(x: float, device=None) -> float:
    """The largest value of x over the ranks (device times: max, never wall clock)."""
    import torch
    d = _dist()
    if d is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


def exchange_votes(h, device: int) -> None:
    """Sums the vote states of every rank's context h in place (one all-reduce)."""
    import torch
    words = h.votes_words()
    buf = torch.empty(max(1, words), dtype=torch.int32, device=torch.device("cuda", device))
    h.votes_save(buf.data_ptr())  # returns once the copy is done
    allreduce_votes(buf)
    torch.cuda.current_stream(device).synchronize()
    h.votes_load(buf.data_ptr())


def correct_sharded(reads, device: int | None = None, **kw) -> dict:
    """Corrects reads against themselves with the subject reads split over the
    ranks of the default process group (one rank per GPU).  Each rank votes
    into its own device buffer (hero_set_vote_buffer), the states are reduced
    to the owners of query-read ranges in place, each rank calls the consensus
    of its own reads (hero_consensus_range), and the ranges are gathered, so
    every rank returns the whole result (hero_b200.correct's outputs)."""
    import numpy as np
    import torch

    from hero_b200 import Hero
    world, rank = world_rank()
    dev = torch.cuda.current_device() if device is None else device
    a, b = shard_range(reads.n, rank, world)
    owners = owner_slices(reads.off, world)
    nqb = int(reads.off[-1]) if reads.n else 0
    state = torch.zeros(max(1, 5 * nqb) + 64, dtype=torch.int32, device=torch.device("cuda", dev))
    with Hero(device=dev, **kw) as h:
        h.set_vote_buffer(state.data_ptr(), state.numel() * 4)
        h.set_queries(reads.seq, reads.off, reads.names)
        h.build_index()
        h.align_self_range(a, b - a)
        torch.cuda.synchronize(dev)
        reduce_votes_to_owners(state, owners)
        torch.cuda.synchronize(dev)
        first, count, nb, _ = owners[rank]
        own = h.consensus_range(first, count, nb)
        stats = h.stats()
    parts = [own]
    d = _dist()
    if d is not None:
        parts = [None] * world
        d.all_gather_object(parts, own)
    res = {k: np.concatenate([p[k] for p in parts]) for k in own}
    res["stats"] = stats
    return res
