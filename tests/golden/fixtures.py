"""Golden fixtures: seeded inputs and the reference flags they were run with.

Each fixture's input is regenerated from its seed (hero_b200.synth); the
reference outputs recorded by make_golden.py are stored beside this file
(manifest.json: md5 of the FASTQ and of the reference .fasta/.info; the
smallest outputs are also kept gzipped).  Read names are 1..N, except in
c2_20k_names (shuffled, duplicated and negative names).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from hero_b200 import synth  # noqa: E402


def _mix(seed: int = 11) -> synth.ReadSet:
    """Mixed lengths 35..160 with N bases and lowercase reads injected (5 % each)."""
    rs = synth.config3(seed=seed, genome_bp=15000, coverage=25, lmin=35, lmax=160)
    rng = np.random.default_rng(seed + 1000)
    seq = rs.seq.copy()
    for i in range(rs.n):
        a, b = int(rs.off[i]), int(rs.off[i + 1])
        if rng.random() < 0.05 and b > a:
            seq[a + int(rng.integers(b - a))] = ord("N")
        if rng.random() < 0.05:
            seq[a:b] = np.frombuffer(bytes(seq[a:b]).lower(), np.uint8)
    rs.seq = seq
    return rs


def _names(seed: int = 23) -> synth.ReadSet:
    """Affine workload reads under shuffled names, 3 % of them repeating another
    read's name (such reads never align to each other: the self-hit test compares
    names) and 1 % negative (atoi keeps the sign; the .aln prints a query's id as
    UINT64)."""
    rs = synth.config2(seed=seed, genome_bp=20000, n_repeats=4)
    rng = np.random.default_rng(seed + 2000)
    names = rng.permutation(np.arange(1, rs.n + 1, dtype=np.int64))
    dup = rng.random(rs.n) < 0.03
    names[dup] = names[rng.integers(0, rs.n, int(dup.sum()))]
    neg = rng.random(rs.n) < 0.01
    names[neg] = -names[neg]
    rs.names = names
    return rs


def _pairs(seed: int = 31) -> synth.ReadSet:
    """Read pairs for --merge: per fragment of 160-290 bases (either strand of a
    20 kbp genome) the first 150 bases and the reverse complement of the last
    150, stored as reads 2i and 2i+1, with 0.5 % substitutions."""
    rng = np.random.default_rng(seed)
    g = synth.random_genome(rng, 20000)
    reads = []
    for _ in range(2700):
        flen = int(rng.integers(160, 291))
        a = int(rng.integers(0, len(g) - flen))
        frag = g[a:a + flen]
        if rng.random() < 0.5:
            frag = synth.revcomp(frag)
        reads.append(synth.substitute(rng, frag[:150], 0.005))
        reads.append(synth.substitute(rng, synth.revcomp(frag[flen - 150:]), 0.005))
    off = np.zeros(len(reads) + 1, np.uint64)
    off[1:] = np.cumsum([len(r) for r in reads])
    return synth.ReadSet(np.concatenate(reads).astype(np.uint8), off,
                         np.arange(1, len(reads) + 1, dtype=np.int64))


# name -> (input generator, reference flags)
FIXTURES = {
    "c1_20k": (lambda: synth.config1(genome_bp=20000), []),
    "c1_20k_affine": (lambda: synth.config1(genome_bp=20000), ["-a", "a"]),
    "c1_20k_narrow": (lambda: synth.config1(genome_bp=20000), ["-m", "2", "-i", "1"]),
    "c2_30k": (lambda: synth.config2(genome_bp=30000, n_repeats=4), ["-a", "a"]),
    "c2_30k_narrow": (lambda: synth.config2(genome_bp=30000, n_repeats=4),
                      ["-a", "a", "-m", "3", "-i", "2"]),
    "c2_30k_k31": (lambda: synth.config2(genome_bp=30000, n_repeats=4),
                   ["-k", "31", "-a", "a", "-c", "0.7"]),
    "mix": (_mix, []),
    "mix_affine": (_mix, ["-a", "a"]),
    "mix_k21_l60": (_mix, ["-k", "21", "-l", "60"]),
    "mix_i0": (_mix, ["-i", "0", "-m", "4"]),
    "c2_20k_names": (_names, ["-a", "a"]),
}

# --merge fixtures: name -> (input generator, reference flags besides
# -c --covinfo --merge; paired input, no --singleReads)
MERGE_FIXTURES = {
    "merge_pairs": (_pairs, []),
    "merge_pairs_affine": (_pairs, ["-a", "a"]),
    "merge_c1_20k": (lambda: synth.config1(genome_bp=20000), []),
}

# -c --mapping (--singleReads, one query file): the coverage histogram of the
# best record covering each subject; name -> the FIXTURES entry it runs on
MAPPING_FIXTURES = ("c1_20k", "c2_30k", "mix_affine", "c2_20k_names")

# fixtures whose reference outputs are stored in full (gzipped)
STORED = ("c1_20k", "mix_affine")


def upper(rs: synth.ReadSet) -> synth.ReadSet:
    """The reads as HERO holds them after parsing (toupper, QueryDataset.cpp:208-209)."""
    seq = np.frombuffer(bytes(rs.seq).upper(), np.uint8).copy()
    return synth.ReadSet(seq, rs.off, rs.names, rs.qual, dict(rs.meta))


def aln_flags(flags: list[str]) -> list[str]:
    """The flags of the alignment-output mode: the consensus threshold (-c x) dropped."""
    out, i = [], 0
    while i < len(flags):
        if flags[i] == "-c":
            i += 2
            continue
        out += flags[i:i + 2]
        i += 2
    return out


def params(flags: list[str]) -> dict:
    """Reference flags -> keyword arguments of hero_b200.Hero (Config::setConfig)."""
    p = dict(k=39, min_overlap=40, aligner="global", max_mismatch_rate=1.0,
             max_indel_rate=1.0, consensus_threshold=0.6)
    i = 0
    while i < len(flags):
        f = flags[i]
        v = flags[i + 1] if i + 1 < len(flags) else None
        if f == "-k":
            p["k"] = int(v)
        elif f == "-l":
            p["min_overlap"] = int(v)
        elif f == "-a":
            p["aligner"] = "affine" if v == "a" else "global"
        elif f == "-m":
            p["max_mismatch_rate"] = float(v) / 100.0
        elif f == "-i":
            p["max_indel_rate"] = float(v) / 100.0
        elif f == "-c":
            p["consensus_threshold"] = float(v)
        else:
            raise ValueError(f)
        i += 2
    return p
