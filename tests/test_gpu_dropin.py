"""HERO itself with the library in place of its aligner (oracle/_ref/hero_ref_gpu,
built by oracle/dropin/make_dropin.py from the reference's sources with three
lines of main.cpp changed): run with the reference's flags, its .fasta/.info
files are byte-identical to the unmodified reference's (the manifest's md5s)."""
import hashlib
import json
import os
import subprocess

import pytest
from fixtures import FIXTURES

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "hero_ref_gpu")
MANIFEST = json.load(open(os.path.join(ROOT, "tests", "golden", "manifest.json")))


@pytest.mark.skipif(not os.path.exists(BIN), reason="HERO with the drop-in binding not built")
@pytest.mark.parametrize("name", ["c1_20k", "c2_30k", "mix_affine"])
def test_hero_with_the_library_matches_the_reference(tmp_path, name):
    gen, flags = FIXTURES[name]
    rs = gen()
    fq = tmp_path / "in.fq"
    fq.write_bytes(rs.to_fastq())
    out = tmp_path / "out"
    r = subprocess.run([BIN, "-q", str(fq), "-s", str(fq), "-c", "--covinfo", "--singleReads",
                        "-t", "4", "-o", str(out)] + flags, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    want = MANIFEST[name]
    fa = hashlib.md5((tmp_path / "out.fasta").read_bytes()).hexdigest()
    info = hashlib.md5((tmp_path / "out.info").read_bytes()).hexdigest()
    assert fa == want["fasta_md5"] and info == want["info_md5"], (name, r.stdout[-1000:])
