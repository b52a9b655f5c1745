"""Seeded synthetic sequencing reads for the HERO read-correction workloads.

No public dataset is involved: every workload is generated from a seed, so the
same seed gives byte-identical FASTQ on any machine with the same numpy.

Read names are the integers 1..N.  HERO parses names with ``atoi``
(QueryDataset.cpp:269, SubjectDataset.cpp:195) and drops hits whose query and
subject ids are equal (SubjectReadAligner.cpp:463-465), so names must be
distinct positive integers or every hit is discarded as a self hit.

Bases are stored as uppercase ASCII ``uint8``.  A read set is a ``ReadSet``:
one flat byte buffer plus offsets, which is also the layout the C ABI takes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
# complement table over ASCII (A<->T, C<->G); other bytes map to themselves
_COMP = np.arange(256, dtype=np.uint8)
_COMP[ord("A")], _COMP[ord("T")] = ord("T"), ord("A")
_COMP[ord("C")], _COMP[ord("G")] = ord("G"), ord("C")


@dataclass
class ReadSet:
    """Reads as one flat ASCII buffer: read i is ``seq[off[i]:off[i+1]]``."""

    seq: np.ndarray                 # uint8, concatenated bases
    off: np.ndarray                 # uint64, n+1 offsets
    names: np.ndarray               # int64, read names (integers)
    qual: list | None = None        # per-read quality strings (bytes) or None
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.off) - 1

    @property
    def lengths(self) -> np.ndarray:
        return np.diff(self.off).astype(np.uint32)

    @property
    def total_bases(self) -> int:
        return int(self.off[-1])

    def read(self, i: int) -> bytes:
        return self.seq[int(self.off[i]):int(self.off[i + 1])].tobytes()

    def to_fastq(self) -> bytes:
        out = []
        for i in range(self.n):
            s = self.read(i)
            q = self.qual[i] if self.qual is not None else b"?" * len(s)
            out.append(b"@%d\n%s\n+\n%s\n" % (int(self.names[i]), s, q))
        return b"".join(out)

    def write_fastq(self, path) -> None:
        with open(path, "wb") as f:
            # chunked to bound memory on large sets
            step = 200_000
            for a in range(0, self.n, step):
                b = min(self.n, a + step)
                lens = self.lengths[a:b]
                buf = []
                for i in range(a, b):
                    s = self.seq[int(self.off[i]):int(self.off[i + 1])].tobytes()
                    q = self.qual[i] if self.qual is not None else b"?" * int(lens[i - a])
                    buf.append(b"@%d\n%s\n+\n%s\n" % (int(self.names[i]), s, q))
                f.write(b"".join(buf))


def revcomp(a: np.ndarray) -> np.ndarray:
    return _COMP[a[::-1]]


def random_genome(rng: np.random.Generator, g: int, gc: float = 0.5) -> np.ndarray:
    """iid genome of ``g`` bases with GC fraction ``gc`` (uniform A/C/G/T at 0.5)."""
    p_at = (1.0 - gc) / 2.0
    p_cg = gc / 2.0
    codes = rng.choice(4, size=g, p=[p_at, p_cg, p_cg, p_at])  # A C G T
    return _ACGT[codes]


def substitute(rng: np.random.Generator, a: np.ndarray, rate) -> np.ndarray:
    """Replace each base with prob ``rate`` (scalar or per-position) by one of the other three."""
    a = a.copy()
    hit = rng.random(a.shape) < rate
    if hit.any():
        code = np.searchsorted(_ACGT, a[hit])
        code = (code + rng.integers(1, 4, size=code.shape)) & 3
        a[hit] = _ACGT[code]
    return a


def add_repeats(rng, genome: np.ndarray, n: int = 40, lmin: int = 1000, lmax: int = 5000,
                divergence: float = 0.005) -> np.ndarray:
    """Copy ``n`` random segments (length U{lmin..lmax}) to random places, at ``divergence``."""
    g = genome.copy()
    G = len(g)
    for _ in range(n):
        ln = int(rng.integers(lmin, lmax + 1))
        src = int(rng.integers(0, G - ln))
        dst = int(rng.integers(0, G - ln))
        g[dst:dst + ln] = substitute(rng, g[src:src + ln], divergence)
    return g


def _geom_capped(rng, size, p=0.6, cap=3):
    return np.minimum(rng.geometric(p, size=size), cap)


@dataclass
class ErrorModel:
    """Per-read error model.

    ``sub_lo``/``sub_hi``: substitution rate rising linearly from the first to
    the last base of a read (equal for a constant rate).  ``ins``/``dele``:
    per-base insertion / deletion event rates; event lengths are
    geometric(``p_len``) capped at ``cap``.
    """

    sub_lo: float
    sub_hi: float
    ins: float = 0.0
    dele: float = 0.0
    p_len: float = 0.6
    cap: int = 3
    const_q: int | None = None     # constant Phred quality, else Phred of the rate

    def rate(self, L: int) -> np.ndarray:
        if L == 1:
            return np.array([self.sub_lo])
        return self.sub_lo + (self.sub_hi - self.sub_lo) * np.arange(L) / (L - 1)

    def qual(self, L: int) -> bytes:
        if self.const_q is not None:
            return bytes([33 + self.const_q]) * L
        q = np.clip(np.rint(-10.0 * np.log10(self.rate(L))), 2, 60).astype(np.uint8) + 33
        return q.tobytes()


CONFIG1_ERRORS = ErrorModel(0.01, 0.01, const_q=30)
CONFIG2_ERRORS = ErrorModel(0.001, 0.02, ins=0.0005, dele=0.0005)


def sample_reads(rng, genome: np.ndarray, n: int, lengths, err: ErrorModel,
                 first_name: int = 1) -> ReadSet:
    """Sample ``n`` reads; start uniform, strand 50/50, errors in read coordinates."""
    G = len(genome)
    lengths = np.broadcast_to(np.asarray(lengths, dtype=np.int64), (n,)).copy()
    slack = 48
    starts = rng.integers(0, G - int(lengths.max()) - slack, size=n)
    strand = rng.random(n) < 0.5
    off = np.zeros(n + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lengths)
    out = np.empty(int(off[-1]), dtype=np.uint8)
    has_indel = err.ins > 0 or err.dele > 0
    # per-length caches for rates and qualities
    rate_cache: dict[int, np.ndarray] = {}
    qual_cache: dict[int, bytes] = {}
    quals = []
    for L in np.unique(lengths):
        L = int(L)
        rate_cache[L] = err.rate(L)
        qual_cache[L] = err.qual(L)
    # event draws (per output position) for the indel model
    for L in np.unique(lengths):
        L = int(L)
        idx = np.nonzero(lengths == L)[0]
        m = len(idx)
        tmpl = genome[starts[idx][:, None] + np.arange(L + slack)[None, :]]
        rc = strand[idx]
        if rc.any():
            tmpl[rc] = _COMP[tmpl[rc][:, ::-1]]
        if has_indel:
            ins_ev = rng.random((m, L)) < err.ins
            del_ev = rng.random((m, L)) < err.dele
            ev_rows = np.nonzero(ins_ev.any(1) | del_ev.any(1))[0]
        else:
            ev_rows = np.zeros(0, dtype=np.int64)
        reads = tmpl[:, :L].copy()
        for r in ev_rows:
            t = tmpl[r]
            o = np.empty(L, dtype=np.uint8)
            ti = 0
            oi = 0
            ins_pos = set(np.nonzero(ins_ev[r])[0].tolist())
            del_pos = set(np.nonzero(del_ev[r])[0].tolist())
            events = sorted(ins_pos | del_pos)
            for p in events:
                if p < oi:
                    continue
                # copy template up to output position p
                k = p - oi
                o[oi:p] = t[ti:ti + k]
                ti += k
                oi = p
                if p in del_pos:
                    ti += int(_geom_capped(rng, 1, err.p_len, err.cap)[0])
                if p in ins_pos:
                    li = int(_geom_capped(rng, 1, err.p_len, err.cap)[0])
                    li = min(li, L - oi)
                    o[oi:oi + li] = _ACGT[rng.integers(0, 4, size=li)]
                    oi += li
            if oi < L:
                o[oi:] = t[ti:ti + (L - oi)]
            reads[r] = o
        reads = substitute(rng, reads, rate_cache[L][None, :])
        for j, i in enumerate(idx):
            out[int(off[i]):int(off[i + 1])] = reads[j]
    for i in range(n):
        quals.append(qual_cache[int(lengths[i])])
    names = np.arange(first_name, first_name + n, dtype=np.int64)
    return ReadSet(out, off, names, quals)


def _even(n: int) -> int:
    n = int(round(n))
    return n - (n & 1)


def config1(seed: int = 1, genome_bp: int = 1_000_000, coverage: float = 30.0,
            read_len: int = 100) -> ReadSet:
    """Plain method, small: iid genome, fixed-length reads, 1 % iid substitutions, no indels."""
    rng = np.random.default_rng(seed)
    g = random_genome(rng, genome_bp)
    n = _even(coverage * genome_bp / read_len)
    rs = sample_reads(rng, g, n, read_len, CONFIG1_ERRORS)
    rs.meta.update(config="config1", genome_bp=genome_bp, coverage=coverage,
                   read_len=read_len, seed=seed, aligner="global")
    return rs


def config2(seed: int = 2, genome_bp: int = 5_000_000, coverage: float = 50.0,
            read_len: int = 150, n_repeats: int = 40) -> ReadSet:
    """Affine/indel: genome with repeat copies, substitution ramp 0.1 %->2 %, short indels."""
    rng = np.random.default_rng(seed)
    g = random_genome(rng, genome_bp)
    if n_repeats:
        lmax = min(5000, max(1000, genome_bp // 20))
        lmin = min(1000, lmax)
        g = add_repeats(rng, g, n_repeats, lmin, lmax, 0.005)
    n = _even(coverage * genome_bp / read_len)
    rs = sample_reads(rng, g, n, read_len, CONFIG2_ERRORS)
    rs.meta.update(config="config2", genome_bp=genome_bp, coverage=coverage,
                   read_len=read_len, seed=seed, aligner="affine")
    return rs


def config3(seed: int = 3, genome_bp: int = 20_000_000, coverage: float = 100.0,
            lmin: int = 75, lmax: int = 250) -> ReadSet:
    """Uneven lengths: GC 42 % genome, read lengths U{lmin..lmax}, config-2 error model."""
    rng = np.random.default_rng(seed)
    g = random_genome(rng, genome_bp, gc=0.42)
    n = _even(coverage * genome_bp / ((lmin + lmax) / 2.0))
    lengths = rng.integers(lmin, lmax + 1, size=n)
    rs = sample_reads(rng, g, n, lengths, CONFIG2_ERRORS)
    rs.meta.update(config="config3", genome_bp=genome_bp, coverage=coverage,
                   read_len=(lmin, lmax), seed=seed, aligner="affine")
    return rs


def config5(seed: int = 5, genome_bp: int = 100_000_000, coverage: float = 30.0,
            read_len: int = 150) -> ReadSet:
    """Large diploid job: haplotype B = A with 0.1 % SNPs and 0.01 % 1-3 bp indels."""
    rng = np.random.default_rng(seed)
    a = random_genome(rng, genome_bp)
    b = substitute(rng, a, 0.001)
    ev = np.nonzero(rng.random(genome_bp) < 0.0001)[0]
    pieces = []
    last = 0
    for p in ev:
        p = int(p)
        if p < last:
            continue
        pieces.append(b[last:p])
        ln = int(rng.integers(1, 4))
        if rng.random() < 0.5:          # deletion
            last = p + ln
        else:                           # insertion
            pieces.append(_ACGT[rng.integers(0, 4, size=ln)])
            last = p
    pieces.append(b[last:])
    b = np.concatenate(pieces)
    n = _even(coverage * genome_bp / read_len)
    ra = sample_reads(rng, a, n // 2, read_len, CONFIG2_ERRORS, first_name=1)
    rb = sample_reads(rng, b, n - n // 2, read_len, CONFIG2_ERRORS, first_name=n // 2 + 1)
    seq = np.concatenate([ra.seq, rb.seq])
    off = np.concatenate([ra.off, rb.off[1:] + ra.off[-1]])
    rs = ReadSet(seq, off, np.concatenate([ra.names, rb.names]), ra.qual + rb.qual)
    rs.meta.update(config="config5", genome_bp=genome_bp, coverage=coverage,
                   read_len=read_len, seed=seed, aligner="affine")
    return rs


def paired(seed: int = 6, genome_bp: int = 5_000_000, coverage: float = 50.0,
           read_len: int = 150, frag_min: int = 160, frag_max: int = 290,
           sub_rate: float = 0.005) -> ReadSet:
    """Read pairs for --merge: per fragment (length U{frag_min..frag_max}, either
    strand) its first read_len bases and the reverse complement of its last
    read_len, stored as reads 2i and 2i+1, with iid substitutions."""
    rng = np.random.default_rng(seed)
    g = random_genome(rng, genome_bp)
    npairs = max(1, int(coverage * genome_bp / (2 * read_len)))
    flen = rng.integers(frag_min, frag_max + 1, size=npairs)
    start = rng.integers(0, genome_bp - flen)
    cols = np.arange(read_len)
    head = g[start[:, None] + cols]                           # forward first bases
    tail = _COMP[g[(start + flen)[:, None] - 1 - cols]]       # reverse complement of the end
    flip = rng.random(npairs) < 0.5                          # fragment from the other strand
    left = np.where(flip[:, None], tail, head)
    right = np.where(flip[:, None], head, tail)
    reads = np.empty((2 * npairs, read_len), np.uint8)
    reads[0::2] = left
    reads[1::2] = right
    reads = substitute(rng, reads, sub_rate)
    off = np.arange(2 * npairs + 1, dtype=np.uint64) * np.uint64(read_len)
    rs = ReadSet(reads.reshape(-1), off, np.arange(1, 2 * npairs + 1, dtype=np.int64))
    rs.meta.update(config="paired", genome_bp=genome_bp, coverage=coverage, read_len=read_len,
                   fragments=(frag_min, frag_max), seed=seed)
    return rs


@dataclass
class Job:
    """One correction job of the serving stream."""

    job_id: int
    arrival_s: float
    seed: int
    genome_bp: int
    read_len: int
    coverage: float

    def reads(self) -> ReadSet:
        rng = np.random.default_rng(self.seed)
        g = random_genome(rng, self.genome_bp)
        n = _even(self.coverage * self.genome_bp / self.read_len)
        rs = sample_reads(rng, g, n, self.read_len, CONFIG2_ERRORS)
        rs.meta.update(config="config4-job", job_id=self.job_id, genome_bp=self.genome_bp,
                       read_len=self.read_len, coverage=self.coverage, seed=self.seed,
                       aligner="affine")
        return rs


def config4_jobs(seed: int = 4, n_jobs: int = 200, rate_per_s: float = 1.0,
                 gmin: float = 0.5e6, gmax: float = 20e6, scale: float = 1.0) -> list[Job]:
    """Serving stream: Poisson arrivals, log-uniform genome size, L in {100,150,250}, cov U(20,80).

    ``scale`` multiplies every genome size (tests use a small scale).
    """
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, size=n_jobs)
    arrivals = np.cumsum(gaps) - gaps[0]
    jobs = []
    for j in range(n_jobs):
        gbp = int(math.exp(rng.uniform(math.log(gmin), math.log(gmax))) * scale)
        L = int(rng.choice([100, 150, 250]))
        gbp = max(gbp, 4 * L + 200)
        cov = float(rng.uniform(20, 80))
        jobs.append(Job(j, float(arrivals[j]), int(rng.integers(1, 2**31 - 1)), gbp, L, cov))
    return jobs
