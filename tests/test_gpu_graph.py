"""The batched form: a correction round captured as one CUDA graph and replayed
gives the same bytes as the plain form, and re-plans when the reads change."""
import pytest
from fixtures import FIXTURES, params, upper
from hero_testlib import assert_same_consensus

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1_20k", "c2_30k", "mix_i0"])
def test_graph_rounds_match_plain(gpu_lib, oracle, name):
    from hero_b200 import Hero
    gen, flags = FIXTURES[name]
    rs = upper(gen())
    kw = params(flags)
    want = oracle.correct(rs, **kw)
    with Hero(subject_batch=1500, **kw) as h:  # several batches inside one graph
        h.set_queries(rs.seq, rs.off, rs.names)
        for rnd in range(4):                      # eager+capture, then 3 replays
            h.round(graph=True)
            got = h.fetch()
            assert_same_consensus(want, got, f"{name} round {rnd}")
        assert h.stats()["graph_rounds"] == 3
        h.round(graph=False)                      # plain form on the same context
        assert_same_consensus(want, h.fetch(), f"{name} plain")


def test_graph_replans_when_reads_change(gpu_lib, oracle):
    from hero_b200 import Hero
    a = upper(FIXTURES["c1_20k"][0]())
    b = upper(FIXTURES["mix"][0]())
    with Hero() as h:
        for rs in (a, b, a):
            h.set_queries(rs.seq, rs.off, rs.names)
            h.round(graph=True)
            h.round(graph=True)
            assert_same_consensus(oracle.correct(rs), h.fetch(), "replan")
