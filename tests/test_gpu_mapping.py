"""--mapping on the device (HERO_FLAG_MAPPING): per subject only the records
SubjectRead::chooseQueryWithBestAlignment keeps vote, and the coverage
histogram (QueryDataset::getCoverageAndWriteResults) is byte-identical to the
reference's file (the manifest's md5); the vote matrix equals the oracle's."""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest
from fixtures import FIXTURES, MAPPING_FIXTURES, aln_flags, params, upper

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MANIFEST = json.load(open(os.path.join(ROOT, "tests", "golden", "manifest.json")))


@pytest.mark.parametrize("name", MAPPING_FIXTURES)
def test_mapping_histogram_matches_reference(gpu_lib, oracle, name):
    from hero_b200 import Hero
    gen, flags = FIXTURES[name]
    rs = upper(gen())
    kw = params(aln_flags(flags))
    with Hero(mapping=True, **kw) as h:
        h.set_queries(rs.seq, rs.off, rs.names)
        h.build_index()
        h.align_self()
        hist = h.mapping_histogram()
        votes = h.votes()
    text = Hero.mapping_text(hist)
    assert hashlib.md5(text).hexdigest() == MANIFEST[name]["mapping_md5"], name
    want = oracle.correct(rs, mapping=True, **kw)
    assert np.array_equal(votes, want["votes"]), name


def test_mapping_cli_matches_reference(tmp_path):
    from hero_b200 import build
    cli = build.build_cli()
    gen, flags = FIXTURES["c2_30k"]
    fq = tmp_path / "in.fq"
    fq.write_bytes(gen().to_fastq())
    out = tmp_path / "hist"
    r = subprocess.run([cli, "-q", str(fq), "-s", str(fq), "-c", "--mapping", "--singleReads",
                        "-o", str(out)] + aln_flags(flags), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert hashlib.md5(out.read_bytes()).hexdigest() == MANIFEST["c2_30k"]["mapping_md5"]
