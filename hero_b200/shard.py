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
    ranks of the default process group (one rank per GPU); every rank returns
    the whole result (hero_b200.correct's outputs)."""
    import torch

    from hero_b200 import Hero
    world, rank = world_rank()
    dev = torch.cuda.current_device() if device is None else device
    a, b = shard_range(reads.n, rank, world)
    with Hero(device=dev, **kw) as h:
        h.set_queries(reads.seq, reads.off, reads.names)
        h.build_index()
        h.align_self_range(a, b - a)
        exchange_votes(h, dev)
        res = h.consensus()
        res["stats"] = h.stats()
    return res
