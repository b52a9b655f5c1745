"""--merge on the GPU (paired input): the overhang votes equal the oracle's, and
the merged / unmerged reads and the .info equal the reference's own files (md5
in the golden manifest), through the library -- plain and graph-replayed
rounds -- and through the drop-in CLI; misuse is refused."""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest
from fixtures import MERGE_FIXTURES, params, upper
from hero_testlib import format_merged, format_outputs

from hero_b200 import Hero, HeroError, build

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(HERE, "manifest.json")))


def md5(b):
    return hashlib.md5(b).hexdigest()


@pytest.mark.parametrize("name", sorted(MERGE_FIXTURES))
def test_merge_matches_reference(oracle, name):
    gen, flags = MERGE_FIXTURES[name]
    rs = gen()
    m = MANIFEST[name]
    kw = params(flags)
    with Hero(merge_pairs=True, **kw) as h:
        h.set_queries(upper(rs).seq, rs.off, rs.names)
        h.build_index()
        h.align_self()
        res = h.consensus()
        ext = h.overhang()
        mg = h.merge_pairs()
    want = oracle.correct(upper(rs), merge=True, **kw)
    assert np.array_equal(ext, want["overhang"])
    merged, unmerged = format_merged(rs.names, mg["merged_seq"], rs.off, mg["merged_len"])
    assert md5(merged) == m["merged_fasta_md5"]
    assert md5(unmerged) == m["unmerged_fasta_md5"]
    _, info = format_outputs(rs.names, res["seq"], rs.off, res["imin"], res["imed"], res["imax"],
                             res["mismatch_rate"], res["gc"])
    assert md5(info) == m["info_md5"]


def test_merge_after_graph_rounds():
    gen, flags = MERGE_FIXTURES["merge_pairs_affine"]
    rs = upper(gen())
    m = MANIFEST["merge_pairs_affine"]
    with Hero(merge_pairs=True, **params(flags)) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        for _ in range(3):  # eager + capture, then replays (overhang votes cleared per round)
            h.round(graph=True)
            mg = h.merge_pairs()
            merged, unmerged = format_merged(rs.names, mg["merged_seq"], rs.off, mg["merged_len"])
            assert md5(merged) == m["merged_fasta_md5"]
            assert md5(unmerged) == m["unmerged_fasta_md5"]


def test_merge_misuse_is_refused():
    gen, _ = MERGE_FIXTURES["merge_c1_20k"]
    rs = upper(gen())
    with Hero(merge_pairs=True) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        h.align_self()
        with pytest.raises(HeroError):  # no consensus of these votes yet
            h.merge_pairs()
    with Hero() as h:  # a context without the flag
        h.set_queries(rs.seq, rs.off, rs.names)
        with pytest.raises(HeroError):
            h.merge_pairs()
    with Hero(merge_pairs=True) as h:  # an odd number of reads cannot be paired
        o = rs.off[:rs.n]
        h.set_queries(rs.seq[:o[-1]], o, rs.names[:rs.n - 1])
        h.build_index()
        h.align_self()
        h.consensus()
        with pytest.raises(HeroError):
            h.merge_pairs()
    with pytest.raises(HeroError):  # --merge belongs to the consensus mode
        Hero(merge_pairs=True, alignment_output=True)


def test_cli_merge_matches_reference(tmp_path):
    build.build_library()
    cli = build.build_cli()
    gen, flags = MERGE_FIXTURES["merge_pairs"]
    rs = gen()
    fq = tmp_path / "in.fq"
    fq.write_bytes(rs.to_fastq())
    out = tmp_path / "out"
    r = subprocess.run([cli, "-q", str(fq), "-s", str(fq), "-c", "--covinfo", "--merge", "-t", "8",
                        "-o", str(out)] + flags, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    m = MANIFEST["merge_pairs"]
    assert not os.path.exists(str(out) + ".fasta")
    assert md5(open(str(out) + "_merged.fasta", "rb").read()) == m["merged_fasta_md5"]
    assert md5(open(str(out) + "_unmerged.fasta", "rb").read()) == m["unmerged_fasta_md5"]
    assert md5(open(str(out) + ".info", "rb").read()) == m["info_md5"]
