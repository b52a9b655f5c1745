"""Alignment-output mode (HERO without -c) on the GPU: the .aln bytes of the
reference itself (md5 and size in the golden manifest) for every fixture,
through the library and through the drop-in CLI, with subjects streamed in
small batches and in chunks from a separate file."""
import hashlib
import json
import os
import subprocess

import pytest
from fixtures import FIXTURES, aln_flags, params, upper

from hero_b200 import Hero, build

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(HERE, "manifest.json")))


def md5(b):
    return hashlib.md5(b).hexdigest()


def kwargs(flags):
    kw = params(aln_flags(flags))
    kw.pop("consensus_threshold")
    return kw


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_alignment_output_matches_reference(name):
    gen, flags = FIXTURES[name]
    rs = upper(gen())
    with Hero(alignment_output=True, **kwargs(flags)) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        h.align_self()
        aln = h.alignments()
        assert h.alignments() == b""  # taken
        st = h.stats()
    assert len(aln) == MANIFEST[name]["aln_bytes"]
    assert md5(aln) == MANIFEST[name]["aln_md5"]
    assert st["records_kept"] > 0


def test_alignment_output_in_small_batches_and_chunks():
    gen, flags = FIXTURES["mix_affine"]
    rs = upper(gen())
    kw = kwargs(flags)
    with Hero(alignment_output=True, subject_batch=97, **kw) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        parts = []
        for a, b in ((0, 1000), (1000, 1001), (1001, rs.n)):  # chunks, one of a single read
            o = rs.off[a:b + 1]
            h.align_subjects(rs.seq[o[0]:o[-1]], o - o[0], rs.names[a:b])
            parts.append(h.alignments())
    aln = b"".join(parts)
    assert md5(aln) == MANIFEST["mix_affine"]["aln_md5"]


def test_consensus_calls_are_refused_in_alignment_output_mode():
    from hero_b200 import HeroError
    gen, flags = FIXTURES["c1_20k"]
    rs = upper(gen())
    with Hero(alignment_output=True) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        with pytest.raises(HeroError):
            h.round(graph=False)
        with pytest.raises(HeroError):
            h.consensus()
    with Hero() as h:  # a consensus context has no alignment text
        h.set_queries(rs.seq, rs.off, rs.names)
        with pytest.raises(HeroError):
            h.alignments()


@pytest.mark.parametrize("name", ["c1_20k", "c2_30k_narrow", "mix_k21_l60"])
def test_cli_alignment_output_matches_reference(tmp_path, name):
    build.build_library()
    cli = build.build_cli()
    gen, flags = FIXTURES[name]
    rs = gen()
    fq = tmp_path / "in.fq"
    fq.write_bytes(rs.to_fastq())
    out = tmp_path / "out"
    r = subprocess.run([cli, "-q", str(fq), "-s", str(fq), "--singleReads", "-t", "8",
                        "-o", str(out)] + aln_flags(flags), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert not os.path.exists(str(out) + ".fasta")
    data = open(str(out) + ".aln", "rb").read()
    assert md5(data) == MANIFEST[name]["aln_md5"]
