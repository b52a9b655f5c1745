"""Regenerates the golden manifest from the reference itself.

Runs the unmodified reference (oracle/_ref/hero_ref, built from the reference
sources by oracle/Makefile) on every fixture input and records md5 sums of the
input FASTQ and of the reference .fasta/.info; the outputs of the fixtures in
STORED are kept gzipped.  Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from fixtures import FIXTURES, STORED  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "hero_ref")


def md5(b: bytes) -> str:
    return hashlib.md5(b).hexdigest()


def run_reference(fq: str, flags: list[str], workdir: str) -> tuple[bytes, bytes]:
    out = os.path.join(workdir, "out")
    for ext in (".fasta", ".info"):  # outputs are opened in append mode
        if os.path.exists(out + ext):
            os.remove(out + ext)
    subprocess.run([REF, "-q", fq, "-s", fq, "-c", "--covinfo", "--singleReads", "-t",
                    str(os.cpu_count() or 1), "-o", out] + flags,
                   stdout=subprocess.DEVNULL, check=True)
    with open(out + ".fasta", "rb") as f:
        fa = f.read()
    with open(out + ".info", "rb") as f:
        info = f.read()
    return fa, info


def main():
    manifest = {}
    with tempfile.TemporaryDirectory() as d:
        for name, (gen, flags) in FIXTURES.items():
            rs = gen()
            fqb = rs.to_fastq()
            fq = os.path.join(d, "in.fq")
            with open(fq, "wb") as f:
                f.write(fqb)
            fa, info = run_reference(fq, flags, d)
            manifest[name] = dict(flags=flags, reads=rs.n, fastq_md5=md5(fqb),
                                  fasta_md5=md5(fa), info_md5=md5(info))
            if name in STORED:
                for ext, data in ((".fasta.gz", fa), (".info.gz", info)):
                    with gzip.GzipFile(os.path.join(HERE, name + ext), "wb", mtime=0) as g:
                        g.write(data)
            print(name, manifest[name], flush=True)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
