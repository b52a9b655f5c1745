"""The CPU oracle against the reference's own outputs (golden manifest)."""
import gzip
import hashlib
import json
import os

import pytest
from fixtures import FIXTURES, MAPPING_FIXTURES, MERGE_FIXTURES, STORED, aln_flags, params, upper
from hero_testlib import format_outputs

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(HERE, "manifest.json")))


def md5(b):
    return hashlib.md5(b).hexdigest()


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_oracle_matches_reference(oracle, name):
    gen, flags = FIXTURES[name]
    rs = gen()
    m = MANIFEST[name]
    assert m["flags"] == flags
    assert md5(rs.to_fastq()) == m["fastq_md5"], "synthetic generator drifted"
    r = oracle.correct(upper(rs), **params(flags))
    fa, info = format_outputs(rs.names, r["seq"], rs.off, r["imin"], r["imed"], r["imax"],
                              r["mismatch_rate"], r["gc"])
    if name in STORED:
        assert fa == gzip.open(os.path.join(HERE, name + ".fasta.gz")).read()
        assert info == gzip.open(os.path.join(HERE, name + ".info.gz")).read()
    assert md5(fa) == m["fasta_md5"]
    assert md5(info) == m["info_md5"]


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_oracle_alignment_output_matches_reference(oracle, name):
    """Alignment-output mode (no -c): the .aln bytes of the reference."""
    gen, flags = FIXTURES[name]
    m = MANIFEST[name]
    kw = params(aln_flags(flags))
    kw.pop("consensus_threshold")
    r = oracle.correct(upper(gen()), aln=True, **kw)
    assert len(r["aln"]) == m["aln_bytes"]
    assert md5(r["aln"]) == m["aln_md5"]


@pytest.mark.parametrize("name", sorted(MERGE_FIXTURES))
def test_oracle_merge_matches_reference(oracle, name):
    """--merge on paired input: the reference's _merged.fasta, _unmerged.fasta, .info."""
    from hero_testlib import format_merged
    gen, flags = MERGE_FIXTURES[name]
    rs = gen()
    m = MANIFEST[name]
    assert md5(rs.to_fastq()) == m["fastq_md5"], "synthetic generator drifted"
    r = oracle.correct(upper(rs), merge=True, **params(flags))
    merged, unmerged = format_merged(rs.names, r["merged_seq"], rs.off, r["merged_len"])
    _, info = format_outputs(rs.names, r["seq"], rs.off, r["imin"], r["imed"], r["imax"],
                             r["mismatch_rate"], r["gc"])
    assert md5(merged) == m["merged_fasta_md5"]
    assert md5(unmerged) == m["unmerged_fasta_md5"]
    assert md5(info) == m["info_md5"]


@pytest.mark.parametrize("name", MAPPING_FIXTURES)
def test_oracle_mapping_matches_reference(oracle, name):
    """-c --mapping: the reference's coverage histogram."""
    gen, flags = FIXTURES[name]
    kw = params(aln_flags(flags))
    r = oracle.correct(upper(gen()), mapping=True, **kw)
    assert md5(r["histogram"]) == MANIFEST[name]["mapping_md5"]


def test_quality_filter(oracle):
    import numpy as np
    qf = oracle.lib.hero_oracle_quality_filter
    def f(s):
        a = np.frombuffer(s, np.uint8).copy()
        return qf(a.ctypes.data, len(a))
    assert f(b"ACGTACGTAC") == 1
    assert f(b"ACGTNCGTAC") == 0           # non-ACGT
    assert f(b"AAAAAAAACG") == 0           # 8 of 10 the same base: 8 >= (10*.8)
    assert f(b"AAAAAAACGT") == 1
    assert f(b"A") == 0                    # threshold 0
