"""The device item logic (hero_core.cuh), compiled for the host, against the oracle.

These run without a GPU: the same source the kernels execute per thread is
driven sequentially and must reproduce the oracle exactly."""
import numpy as np
import pytest
from fixtures import FIXTURES, params, upper

from hero_b200 import synth

ACGT = np.frombuffer(b"ACGT", np.uint8)


def _pairs(rng, n, lmax=70):
    for _ in range(n):
        ls, lq = int(rng.integers(1, lmax)), int(rng.integers(1, lmax))
        s = ACGT[rng.integers(0, 4, ls)]
        if rng.random() < 0.5:
            q = synth.substitute(rng, np.resize(s[rng.integers(0, ls):], lq), 0.1)
        else:
            q = ACGT[rng.integers(0, 4, lq)]
        yield bytes(s), bytes(q.astype(np.uint8))


@pytest.mark.parametrize("affine", [0, 1])
def test_dp_random_segments(oracle, emu, affine):
    rng = np.random.default_rng(100 + affine)
    for s, q in _pairs(rng, 3000):
        band = int(rng.choice([0, 1, 2, 3, 5, 10, 200]))
        right, left = bool(rng.integers(0, 2)), bool(rng.integers(0, 2))
        want, _ = oracle.align(affine, s, q, band, right, left)
        for strip16 in (False, True):
            got = emu.align(affine, s, q, band, right, left, strip16)
            assert np.array_equal(want, got), (affine, s, q, band, right, left, strip16)
        got = emu.align_wave(affine, s, q, band, right, left)
        assert np.array_equal(want, got), (affine, s, q, band, right, left, "wave")


def test_dp_edge_shapes(oracle, emu):
    cases = [(b"A", b"A"), (b"A", b"C"), (b"ACGT", b"A"), (b"A", b"ACGT"), (b"AAAA", b"TTTT"),
             (b"ACGTACGTACGTACGTACGT", b"ACG"), (b"ACGTTTTTTTTT", b"ACGTTTTTTTTT")]
    for affine in (0, 1):
        for s, q in cases:
            for band in (0, 1, 2, 50):
                for right in (False, True):
                    for left in (False, True):
                        want, _ = oracle.align(affine, s, q, band, right, left)
                        got = emu.align(affine, s, q, band, right, left)
                        assert np.array_equal(want, got), (affine, s, q, band, right, left)
                        got = emu.align_wave(affine, s, q, band, right, left)
                        assert np.array_equal(want, got), (affine, s, q, band, right, left, "wave")


@pytest.mark.parametrize("name", ["c1_20k", "c1_20k_narrow", "mix_affine", "mix_k21_l60",
                                  "mix_i0", "c2_20k_names"])
def test_pipeline_matches_oracle(oracle, emu, name):
    gen, flags = FIXTURES[name]
    rs = upper(gen())
    kw = params(flags)
    want = oracle.correct(rs, **kw)
    got = emu.correct(rs, **kw)
    from hero_testlib import assert_same_consensus
    assert_same_consensus(want, got, name)
    assert np.array_equal(want["votes"], got["votes"])


def _indels(rng, x, rate):
    out = []
    for b in x:
        r = rng.random()
        if r < rate:             # deletion
            continue
        out.append(b)
        if r > 1 - rate:         # insertion
            out.append(ACGT[rng.integers(0, 4)])
    return np.array(out, np.uint8)


@pytest.mark.parametrize("affine", [0, 1])
def test_wave_long_segments_with_indels(oracle, emu, affine):
    """Segments of 150-260 bases with substitutions and indels: many strips per
    segment, so the traceback runs in row chunks over many lanes, and paths
    that leave the diagonal make the first guesses wrong."""
    rng = np.random.default_rng(300 + affine)
    for _ in range(150):
        ls = int(rng.integers(150, 261))
        s = ACGT[rng.integers(0, 4, ls)]
        q = _indels(rng, synth.substitute(rng, s.copy(), 0.03), float(rng.choice([0.002, 0.01, 0.05])))
        q = q[:int(rng.integers(max(1, len(q) - 40), len(q) + 1))]
        band = int(rng.choice([300, 1000]))
        right, left = bool(rng.integers(0, 2)), bool(rng.integers(0, 2))
        want, _ = oracle.align(affine, bytes(s), bytes(q), band, right, left)
        got = emu.align_wave(affine, bytes(s), bytes(q), band, right, left)
        assert np.array_equal(want, got), (affine, len(s), len(q), band, right, left)


def test_band_cells_closed_form(emu):
    """band_cells (the reference's loop bounds, BandAligner.cpp:63-66) against the loop."""
    import ctypes as C
    f = emu.lib.emu_band_cells
    f.restype = C.c_uint64
    f.argtypes = [C.c_int32, C.c_int32, C.c_int64]
    rng = np.random.default_rng(5)
    for _ in range(3000):
        c = int(rng.integers(0, 300))
        r = c + int(rng.integers(0, 300))
        m = max(int(rng.choice([0, 1, 3, 10, 80, 300, 70000])), r - c)  # band >= R - C
        want = sum(min(c, i + m) - max(0, i - m) + 1 for i in range(r + 1)
                   if min(c, i + m) >= max(0, i - m))
        assert f(r, c, m) == want, (r, c, m)


def test_rolling_kmers_match_direct(emu):
    """The probe kernel rolls forward and reverse-complement k-mers one base per
    window; every window equals the k-mer built from scratch, for all k."""
    import ctypes as C
    f = emu.lib.emu_kmer_roll_check
    f.restype = C.c_int64
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int32]
    rng = np.random.default_rng(9)
    codes = rng.integers(0, 4, 400).astype(np.uint8)
    for k in (1, 2, 15, 21, 31, 32, 33, 39, 47, 63):
        assert f(codes.ctypes.data, len(codes), k) == -1, k


@pytest.mark.parametrize("affine", [1, 0])
def test_pair_rows_match_oracle(oracle, emu, affine):
    """Two segments of one shape in the tagged 16-bit halves of the pair rows:
    each half's path equals the oracle's path for the aligner (flags may differ
    in align-right, share align-left)."""
    import ctypes as C
    f = emu.lib.emu_align_pair
    f.restype = C.c_int
    f.argtypes = [C.c_int] + [C.c_void_p] * 4 + [C.c_int32, C.c_int32, C.c_int32, C.c_int64,
                                                 C.c_int64, C.c_int, C.c_int, C.c_void_p,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
    rng = np.random.default_rng(77 + affine)
    done = 0

    def query(rng, s, lq):
        if rng.random() < 0.7:
            q = _indels(rng, synth.substitute(rng, np.resize(s, lq).copy(), 0.03), 0.01)
            return np.resize(q, lq).astype(np.uint8)
        return ACGT[rng.integers(0, 4, lq)]

    for _ in range(400):
        ls = int(rng.integers(1, 200))
        left = int(rng.integers(0, 2))
        if rng.random() < 0.3:  # the query side is the longer one (rows), equal in both
            lq = lqb = int(rng.integers(ls, 200))
        else:  # the subject side is the rows; B's columns may differ within the strip count
            lq = int(rng.integers(1, ls + 1))
            lo = max(1, 8 * ((lq - 1) // 8) + 1)
            lqb = lq if left else int(rng.integers(lo, min(ls, lo + 7) + 1))
        seqs = []
        for lqh in (lq, lqb):
            sh = ACGT[rng.integers(0, 4, ls)]
            seqs.append((bytes(sh), bytes(query(rng, sh, lqh))))
        fa = (int(rng.integers(0, 2)) | (left << 1))
        fb = (int(rng.integers(0, 2)) | (left << 1))
        band_a, band_b = int(rng.choice([400, 1000])), int(rng.choice([400, 1000]))
        cap = ls + max(lq, lqb) + 1
        oa, ob = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
        na, nb = C.c_int32(), C.c_int32()
        bufs = [np.frombuffer(x, np.uint8).copy() for x in (seqs[0][0], seqs[0][1], seqs[1][0], seqs[1][1])]
        rc = f(affine, *[b.ctypes.data for b in bufs], ls, lq, lqb, band_a, band_b, fa, fb,
               oa.ctypes.data, C.byref(na), ob.ctypes.data, C.byref(nb), cap)
        assert rc == 0, (ls, lq, lqb, left)
        for (s, q), band, fl, ops, n in ((seqs[0], band_a, fa, oa, na), (seqs[1], band_b, fb, ob, nb)):
            want, _ = oracle.align(affine, s, q, band, bool(fl & 1), bool(fl & 2))
            assert np.array_equal(want, ops[:n.value]), (ls, len(q), band, fl)
        done += 1
    assert done == 400


@pytest.mark.parametrize("name", ["c1_20k", "c1_20k_affine", "mix", "mix_affine", "mix_i0",
                                  "mix_k21_l60", "c1_20k_narrow", "c2_20k_names"])
def test_emulated_alignment_output_matches_reference(emu, name):
    """The device item logic of the alignment-output mode (flipped seeds, the
    query's reverse complement in the DP, the record list, the record text),
    driven sequentially on the host: the reference's .aln bytes."""
    import hashlib
    import json
    import os
    from fixtures import FIXTURES, aln_flags, params, upper
    m = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                    "manifest.json")))[name]
    gen, flags = FIXTURES[name]
    kw = params(aln_flags(flags))
    kw.pop("consensus_threshold")
    a = emu.align_output(upper(gen()), **kw)
    assert len(a) == m["aln_bytes"]
    assert hashlib.md5(a).hexdigest() == m["aln_md5"]


@pytest.mark.parametrize("name", ["merge_pairs", "merge_pairs_affine", "merge_c1_20k"])
def test_emulated_merge_matches_reference(oracle, emu, name):
    """--merge through the device item logic (overhang walk, extension letters,
    pair merge) on the host: the oracle's overhang votes and the reference's
    _merged.fasta / _unmerged.fasta."""
    import hashlib
    import json
    import os
    from fixtures import MERGE_FIXTURES
    from hero_testlib import format_merged
    m = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                    "manifest.json")))[name]
    gen, flags = MERGE_FIXTURES[name]
    rs = gen()
    got = emu.merge(upper(rs), **params(flags))
    want = oracle.correct(upper(rs), merge=True, **params(flags))
    assert np.array_equal(got["overhang"], want["overhang"])
    merged, unmerged = format_merged(rs.names, got["merged_seq"], rs.off, got["merged_len"])
    assert hashlib.md5(merged).hexdigest() == m["merged_fasta_md5"]
    assert hashlib.md5(unmerged).hexdigest() == m["unmerged_fasta_md5"]


def test_ops_summary_by_lane_groups(emu):
    """The DP summary of a packed op range: against the fields read one by one,
    and as the parts of G lanes (every G-th word each) merged by the kernel's
    shuffle tree, for every G from 1 to 32."""
    import numpy as np
    rng = np.random.default_rng(17)
    for trial in range(400):
        words = int(rng.integers(1, 40))
        kind = trial % 4
        if kind == 0:    # uniform random ops
            w = rng.integers(0, 2**32, size=words, dtype=np.uint64).astype(np.uint32)
        else:            # long runs of one op, a few others
            ops = np.full(words * 16, int(rng.integers(0, 4)), np.uint32)
            for _ in range(int(rng.integers(0, 4))):
                a = int(rng.integers(0, words * 16))
                ops[a:a + int(rng.integers(1, 20))] = int(rng.integers(0, 4))
            w = np.zeros(words, np.uint32)
            for p in range(words * 16):
                w[p >> 4] |= np.uint32(ops[p] << (2 * (p & 15)))
        total = words * 16
        P = int(rng.integers(1, total + 1))
        first = int(rng.integers(0, total - P + 1)) if trial % 3 else total - P  # kernel: ranges end at the last word
        w = np.ascontiguousarray(w)
        r = emu.lib.emu_ops_summary_groups(w.ctypes.data, first, P)
        assert r == 0, (trial, words, first, P, r)
