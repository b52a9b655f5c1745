"""The drop-in's read parser (hero_b200/host/hero_host.cpp, load_reads) on the
CPU against a plain restatement of the reference's reading rules
(QueryDataset.cpp:246-391: a FASTQ record is four lines, read with getline;
FASTA records run from '>' to '>'; names through atoi; bases uppercased):
edge cases of blank, truncated and unterminated input, and files large enough
that the parser's threads split them at arbitrary bytes."""
import os
import subprocess

import numpy as np
import pytest

from hero_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def parse_bin(tmp_path_factory):
    lib = build.build_library()
    out = str(tmp_path_factory.mktemp("bin") / "host_parse")
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "include"),
                    "-o", out, os.path.join(ROOT, "tests", "emu", "host_parse.cpp"),
                    os.path.join(ROOT, "hero_b200", "host", "hero_host.cpp"),
                    "-L", os.path.dirname(lib), "-lhero_b200",
                    "-Wl,-rpath," + os.path.dirname(lib)], check=True)
    return out


def _atoi(b: bytes) -> int:
    s = b.lstrip(b" \t\n\r\v\f")
    sign, i = 1, 0
    if s[:1] in (b"+", b"-"):
        sign = -1 if s[:1] == b"-" else 1
        i = 1
    j = i
    while j < len(s) and 48 <= s[j] <= 57:
        j += 1
    return sign * int(s[i:j]) if j > i else 0


def _model(data: bytes):
    """The reading rules, restated plainly: [(id, bases)] or the error kind."""
    if not data:
        return []
    fasta = data[:1] == b">"
    if not fasta and data[:1] != b"@":
        return "format"
    n, p, recs = len(data), 0, []

    def line():
        nonlocal p
        if p >= n:
            return None
        e = data.find(b"\n", p)
        e = n if e < 0 else e
        b = p
        p = e + 1 if e < n else n
        return data[b:e]

    if not fasta:
        while True:
            l0 = line()
            if l0 is None:
                break
            l1 = line()
            if l1 is None:
                if l0:
                    return "truncated"
                break
            line()
            line()
            if not l0 and not l1:
                continue
            recs.append((l0, l1))
    else:
        while p < n:
            l0 = line()
            e = data.find(b">", p)
            e = n if e < 0 else e
            b = p
            p = e + 1 if e < n else n
            if not l0 and e == b:
                continue
            recs.append((l0, data[b:e].replace(b"\n", b"")))
    out = []
    for name, seq in recs:
        if name[:1] in (b">", b"@"):
            name = name[1:]
        out.append((_atoi(name), seq.upper()))
    return out


def _run(parse_bin, tmp_path, *blobs):
    paths = []
    for i, b in enumerate(blobs):
        f = tmp_path / f"in{i}"
        f.write_bytes(b)
        paths.append(str(f))
    r = subprocess.run([parse_bin, *paths], capture_output=True, check=True)
    text = r.stdout
    if text.startswith(b"ERR "):
        return "truncated" if b"truncated" in text else "format" if b"format" in text else text
    out = []
    for ln in text.split(b"\n")[:-1]:
        i, s = ln.split(b" ", 1)
        out.append((int(i), s))
    return out


CASES = [
    b"@1\nACGT\n+\nIIII\n@2\nacgtn\n+\nIIIII\n",
    b"@1\nACGT\n+\nIIII\n@2\nACGT\n+\nIIII",            # no final newline
    b"@1\nACGT\n+\nIIII\n\n\n\n\n",                      # blank lines at the end
    b"@1\nACGT\n+\nIIII\n\n\n+\n\n@3\nGG\n+\nII\n",       # a blank record in the middle
    b"@1\nACGT\n+\nIIII\n@7\n",                          # a lone header at the end
    b"@1\nACGT\n+\nIIII\n@7",                            # the same without its newline
    b"@1\nACGT\n+\nIIII\n\n",                            # one blank line after the record
    b"@-12 lane:3\nAC\n+\nII\n@  42x\nGT\n+\nII\n@abc\nT\n+\nI\n",  # atoi rules
    b"@" + b"9" * 5 + b"x" * 200 + b"\nACGT\n+\nIIII\n",   # a long name
    b"@1\n\n+\n\n@2\nA\n+\nI\n",                         # an empty sequence with a name
    b">1\nACGT\nacgt\n>2\n\n>3\nGG",                     # FASTA: wrapped, empty, unterminated
    b">1\nACGT\n>\n",                                    # FASTA: an empty trailing record
    b"#1\nACGT\n",                                       # neither FASTA nor FASTQ
    b"",
]


@pytest.mark.parametrize("i", range(len(CASES)))
def test_edge_cases(parse_bin, tmp_path, i):
    assert _run(parse_bin, tmp_path, CASES[i]) == _model(CASES[i])


def test_large_files_split_across_threads(parse_bin, tmp_path):
    rng = np.random.default_rng(5)
    recs = []
    for r in range(30000):
        L = int(rng.integers(0, 120))
        s = bytes(rng.choice(list(b"ACGTacgtN"), L))
        name = b"%d" % int(rng.integers(-5, 10 ** 6))
        if rng.random() < 0.01:
            recs.append(b"\n\n\n\n")  # a blank record
        recs.append(b"@" + name + b" x\n" + s + b"\n+\n" + b"I" * L + b"\n")
    a = b"".join(recs)
    fa = b"".join(b">%d\n%s\n" % (i, b"ACGTAC" * int(rng.integers(0, 30))) for i in range(20000))
    for blobs in ((a,), (a[:-1],), (a, fa), (fa, a)):  # several files append
        want = []
        for b in blobs:
            m = _model(b)
            assert isinstance(m, list)
            want += m
        assert _run(parse_bin, tmp_path, *blobs) == want
