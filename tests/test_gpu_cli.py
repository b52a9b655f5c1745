"""The drop-in CLI end to end: reads files, corrects on the GPU, writes the
reference's .fasta/.info (md5 of the reference's own outputs)."""
import hashlib
import json
import os
import subprocess

import pytest
from fixtures import FIXTURES

from hero_b200 import build

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(HERE, "manifest.json")))


def md5f(p):
    return hashlib.md5(open(p, "rb").read()).hexdigest()


@pytest.fixture(scope="module")
def cli():
    build.build_library()
    return build.build_cli()


def to_fasta(rs):
    out = []
    for i in range(rs.n):
        s = rs.read(i)
        # wrapped at 60 columns: the reader joins the lines
        lines = [s[j:j + 60] for j in range(0, len(s), 60)] or [b""]
        out.append(b">%d\n%s\n" % (int(rs.names[i]), b"\n".join(lines)))
    return b"".join(out)


@pytest.mark.parametrize("name", ["c1_20k", "c2_30k_narrow", "mix", "mix_k21_l60"])
def test_cli_matches_reference(cli, tmp_path, name):
    gen, flags = FIXTURES[name]
    rs = gen()
    fq = tmp_path / "in.fq"
    fq.write_bytes(rs.to_fastq())
    out = tmp_path / "out"
    r = subprocess.run([cli, "-q", str(fq), "-s", str(fq), "-c", "--covinfo", "--singleReads",
                        "-t", "8", "-o", str(out)] + flags, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert md5f(str(out) + ".fasta") == MANIFEST[name]["fasta_md5"]
    assert md5f(str(out) + ".info") == MANIFEST[name]["info_md5"]


def test_cli_fasta_input_and_separate_subject_file(cli, tmp_path):
    gen, flags = FIXTURES["c1_20k"]
    rs = gen()
    fa = tmp_path / "in.fa"
    fa.write_bytes(to_fasta(rs))
    subj = tmp_path / "subj.fa"  # same reads under another name: streamed as subjects
    subj.write_bytes(to_fasta(rs))
    out = tmp_path / "out"
    r = subprocess.run([cli, "-q", str(fa), "-s", str(subj), "-c", "--covinfo",
                        "-o", str(out)] + flags, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # even read count: the paired writer prints the same bytes as --singleReads
    assert md5f(str(out) + ".fasta") == MANIFEST["c1_20k"]["fasta_md5"]
    assert md5f(str(out) + ".info") == MANIFEST["c1_20k"]["info_md5"]


def test_cli_appends_like_the_reference(cli, tmp_path):
    gen, flags = FIXTURES["mix"]
    rs = gen()
    fq = tmp_path / "in.fq"
    fq.write_bytes(rs.to_fastq())
    out = tmp_path / "out"
    args = [cli, "-q", str(fq), "-s", str(fq), "-c", "--singleReads", "-o", str(out)] + flags
    for _ in range(2):
        assert subprocess.run(args, capture_output=True).returncode == 0
    data = open(str(out) + ".fasta", "rb").read()
    half = len(data) // 2
    assert data[:half] == data[half:]
    assert hashlib.md5(data[:half]).hexdigest() == MANIFEST["mix"]["fasta_md5"]
