"""DP kernel shapes (the autotuner's choices) never change results.

Every candidate shape of hero_b200.autotune -- warps per block, 16-bit pairs of
segments, row-chunk or one-lane tracebacks -- corrects the same reads to the
same bytes, votes and statistics as the default shape; the tuner's record
names the fastest candidate per class."""
import json

import numpy as np
import pytest
from fixtures import FIXTURES, params, upper

from hero_b200 import autotune

pytestmark = pytest.mark.gpu


def _run(rs, kw, classes):
    from hero_b200 import Hero
    with Hero(tuning=classes, **kw) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        h.align_self()
        r = h.consensus()
        r["votes"] = h.votes()
        r["stats"] = h.stats()
    return r


@pytest.mark.parametrize("name", ["c2_30k", "mix_affine", "c1_20k", "mix"])
def test_every_candidate_shape_gives_the_same_result(name):
    gen, flags = FIXTURES[name]
    rs = upper(gen())
    kw = params(flags)
    base = _run(rs, kw, [])
    for shape in autotune.candidates():
        got = _run(rs, kw, [dict(shape, rows_max=100000)])
        for f in ("seq", "imin", "imed", "imax", "good", "votes"):
            assert np.array_equal(base[f], got[f]), (shape, f)
        for f in ("mismatch_rate", "gc"):
            assert np.array_equal(base[f].view(np.uint64), got[f].view(np.uint64)), (shape, f)
        assert base["stats"]["dp_cells"] == got["stats"]["dp_cells"]


def test_tuner_records_the_fastest_candidate(tmp_path):
    rec = autotune.tune(genome_bp=20_000, read_lengths=[150], log=lambda *a: None)
    (cls,) = rec["classes"]
    # the class key is the longest DP side of the sample, as the oracle's segments give it
    from hero_testlib import Oracle
    seg = Oracle().correct(upper(autotune.sample(150, 20_000)), aligner="affine",
                           keep_segments=True)["segments"]
    rows = int(np.maximum(seg["s1"] - seg["s0"], seg["q1"] - seg["q0"]).max())
    assert cls["rows_seen"] == rows and cls["rows_max"] == autotune.ROWS_LAST
    assert len(cls["candidates"]) == len(list(autotune.candidates()))
    assert cls["ms"] == min(c["ms"] for c in cls["candidates"])
    p = tmp_path / "tuning.json"
    p.write_text(json.dumps(rec))
    from hero_b200._lib import load_tuning
    assert load_tuning(str(p))[0]["warps_per_block"] in (1, 2, 4)
