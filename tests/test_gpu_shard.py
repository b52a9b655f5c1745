"""The sharded form on one GPU: subject-read shards aligned by separate
contexts, their vote states added on the device and loaded back, give the
whole run's votes and consensus; the single-rank correct_sharded equals
correct; bad ranges are refused."""
import numpy as np
import pytest
from fixtures import FIXTURES, params, upper

from hero_b200 import Hero, HeroError, correct
from hero_b200.shard import correct_sharded, shard_range

pytestmark = pytest.mark.gpu


def _same(a, b):
    for f in ("seq", "imin", "imed", "imax", "good"):
        assert np.array_equal(a[f], b[f]), f
    for f in ("mismatch_rate", "gc"):
        assert np.array_equal(a[f].view(np.uint64), b[f].view(np.uint64)), f


@pytest.mark.parametrize("name,world", [("mix_affine", 2), ("c2_30k", 3)])
def test_shards_sum_to_the_whole_run(name, world):
    import torch
    gen, flags = FIXTURES[name]
    rs = upper(gen())
    kw = params(flags)
    with Hero(**kw) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        h.align_self()
        whole_votes = h.votes()
        whole = h.consensus()
    ctxs = [Hero(**kw) for _ in range(world)]
    try:
        total = None
        for r, h in enumerate(ctxs):
            h.set_queries(rs.seq, rs.off, rs.names)
            h.build_index()
            a, b = shard_range(rs.n, r, world)
            h.align_self_range(a, b - a)
            buf = torch.empty(h.votes_words(), dtype=torch.int32, device="cuda")
            h.votes_save(buf.data_ptr())
            total = buf if total is None else total + buf
        torch.cuda.synchronize()
        ctxs[0].votes_load(total.data_ptr())
        assert np.array_equal(ctxs[0].votes(), whole_votes)
        _same(ctxs[0].consensus(), whole)
    finally:
        for h in ctxs:
            h.close()


@pytest.mark.parametrize("name,world", [("mix_affine", 2), ("c2_30k", 3)])
def test_owners_of_query_ranges_reproduce_the_whole_run(name, world):
    """The in-place form: every shard votes into its own caller-owned buffer,
    each owner's slice of the summed state goes to the owner's buffer, and the
    owners' range consensuses together are the whole run's."""
    import torch

    from hero_b200.shard import owner_slices
    gen, flags = FIXTURES[name]
    rs = upper(gen())
    kw = params(flags)
    whole = correct(rs, **kw)
    owners = owner_slices(rs.off, world)
    nqb = int(rs.off[-1])
    bufs = [torch.zeros(5 * nqb + 64, dtype=torch.int32, device="cuda") for _ in range(world)]
    ctxs = [Hero(**kw) for _ in range(world)]
    try:
        for r, h in enumerate(ctxs):
            h.set_vote_buffer(bufs[r].data_ptr(), bufs[r].numel() * 4)
            h.set_queries(rs.seq, rs.off, rs.names)
            h.build_index()
            a, b = shard_range(rs.n, r, world)
            h.align_self_range(a, b - a)
        torch.cuda.synchronize()
        for r in range(world):  # the reduce each owner receives
            for lo, hi in owners[r][3]:
                bufs[r][lo:hi] = sum(buf[lo:hi] for buf in bufs)
        torch.cuda.synchronize()
        parts = [ctxs[r].consensus_range(*owners[r][:3]) for r in range(world)]
        got = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
        _same(got, whole)
    finally:
        for h in ctxs:
            h.close()


def test_single_rank_sharded_correction_equals_correct():
    gen, flags = FIXTURES["c1_20k"]
    rs = upper(gen())
    kw = params(flags)
    _same(correct_sharded(rs, **kw), correct(rs, **kw))


def test_ranges_outside_the_query_set_are_refused():
    gen, flags = FIXTURES["c1_20k"]
    rs = upper(gen())
    with Hero() as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        with pytest.raises(HeroError):
            h.align_self_range(rs.n - 1, 2)
        h.align_self_range(rs.n, 0)  # empty range at the end: nothing to do
