"""GPU path (through the C ABI) against the oracle and the reference's outputs."""
import hashlib
import json
import os

import numpy as np
import pytest
from fixtures import FIXTURES, params, upper
from hero_testlib import assert_same_consensus, format_outputs

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(HERE, "manifest.json")))


def md5(b):
    return hashlib.md5(b).hexdigest()


def run_gpu(rs, subject_batch=0, separate_subjects=False, **kw):
    from hero_b200 import Hero
    with Hero(subject_batch=subject_batch, **kw) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        if separate_subjects:
            h.align_subjects(rs.seq, rs.off, rs.names)
        else:
            h.align_self()
        res = h.consensus()
        res["votes"] = h.votes()
        res["stats"] = h.stats()
    return res


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_gpu_matches_reference(gpu_lib, oracle, name):
    gen, flags = FIXTURES[name]
    raw = gen()
    rs = upper(raw)
    kw = params(flags)
    got = run_gpu(rs, **kw)
    want = oracle.correct(rs, **kw)
    assert np.array_equal(got["votes"], want["votes"]), "vote matrix differs"
    assert_same_consensus(want, got, name)
    fa, info = format_outputs(rs.names, got["seq"], rs.off, got["imin"], got["imed"],
                              got["imax"], got["mismatch_rate"], got["gc"])
    assert md5(fa) == MANIFEST[name]["fasta_md5"]
    assert md5(info) == MANIFEST[name]["info_md5"]
    st, ost = got["stats"], want["stats"]
    assert st["hits"] == ost["hits"]
    assert st["chains"] == ost["chains"]
    assert st["chains_kept"] == ost["chains_kept"]
    assert st["records_built"] == ost["records_built"]
    assert st["records_accepted"] == ost["records_accepted"]
    assert st["records_kept"] == ost["records_kept"]
    assert st["dp_segments_ref"] == ost["dp_segments"]
    assert st["dp_cells"] == ost["dp_cells"]
    assert st["vote_anomalies"] == 0
    assert st["dp_stage_timeouts"] == 0


def test_pair_rows_staged_by_bulk_copies(gpu_lib, oracle):
    """The pair wavefront stages its row bases in shared memory with the bulk
    copy engine (cp.async.bulk on an mbarrier): on a workload of 16-bit pairs
    most tasks are staged, no wait runs out, and the output is the oracle's."""
    gen, flags = FIXTURES["c2_30k"]
    rs = upper(gen())
    kw = params(flags)
    got = run_gpu(rs, **kw)
    st = got["stats"]
    assert st["dp_cells_pairs"] > 0
    assert st["dp_tasks_staged"] > 0
    assert st["dp_stage_timeouts"] == 0
    assert_same_consensus(oracle.correct(rs, **kw), got, "c2_30k staged")


@pytest.mark.parametrize("batch", [1, 7, 1000])
def test_gpu_batching_is_invisible(gpu_lib, oracle, batch):
    gen, flags = FIXTURES["mix_affine"]
    rs = upper(gen())
    kw = params(flags)
    want = run_gpu(rs, **kw)
    got = run_gpu(rs, subject_batch=batch, separate_subjects=True, **kw)
    assert_same_consensus(want, got, f"batch {batch}")
    assert np.array_equal(want["votes"], got["votes"])


def test_gpu_chunks_accumulate(gpu_lib, oracle):
    """Subjects streamed in two calls give the same votes as one call."""
    from hero_b200 import Hero
    gen, flags = FIXTURES["c1_20k"]
    rs = upper(gen())
    kw = params(flags)
    h1 = rs.n // 3
    with Hero(**kw) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        a = slice(0, h1 + 1)
        h.align_subjects(rs.seq[:int(rs.off[h1])], rs.off[a], rs.names[:h1])
        off2 = rs.off[h1:] - rs.off[h1]
        h.align_subjects(rs.seq[int(rs.off[h1]):], off2, rs.names[h1:])
        got = h.consensus()
        got_votes = h.votes()
    want = oracle.correct(rs, **kw)
    assert np.array_equal(got_votes, want["votes"])
    assert_same_consensus(want, got, "chunks")


def test_gpu_empty_and_tiny_inputs(gpu_lib):
    from hero_b200 import Hero
    with Hero() as h:
        seq = np.frombuffer(b"ACGT", np.uint8)
        h.set_queries(seq, np.array([0, 4], np.uint64), np.array([1], np.int64))
        h.build_index()
        h.align_self()
        r = h.consensus()
        assert bytes(r["seq"]) == b"ACGT"
        assert r["good"][0] == 0
    with Hero() as h:
        h.set_queries(np.zeros(0, np.uint8), np.zeros(1, np.uint64), np.zeros(0, np.int64))
        h.build_index()
        h.align_self()
        r = h.consensus()
        assert len(r["seq"]) == 0


def test_gpu_rejects_bad_input(gpu_lib):
    from hero_b200 import Hero, HeroError
    with Hero() as h:
        with pytest.raises(HeroError):
            h.build_index()                          # called out of order
        with pytest.raises(HeroError):
            h.align_self()                           # no index yet
        with pytest.raises(HeroError):               # offsets must not decrease
            h.set_queries(np.zeros(8, np.uint8), np.array([0, 5, 4], np.uint64),
                          np.array([1, 2], np.int64))
        with pytest.raises(HeroError):               # offsets must start at 0
            h.set_queries(np.zeros(8, np.uint8), np.array([1, 8], np.uint64),
                          np.array([1], np.int64))
        with pytest.raises(HeroError):               # read longer than 32767 bases
            h.set_queries(np.zeros(40000, np.uint8), np.array([0, 40000], np.uint64),
                          np.array([1], np.int64))
