"""Banded DP kernels (global and affine) through hero_align_segments, on the
exact segments the oracle's aligner was called with, and on random ones."""
import numpy as np
import pytest
from fixtures import FIXTURES, params, upper

pytestmark = pytest.mark.gpu

ACGT = np.frombuffer(b"ACGT", np.uint8)


@pytest.mark.parametrize("name", ["c1_20k", "c1_20k_narrow", "c2_30k", "c2_30k_narrow",
                                  "mix_i0"])
def test_dp_segments_of_a_run(gpu_lib, oracle, name):
    from hero_b200 import Hero
    gen, flags = FIXTURES[name]
    rs = upper(gen())
    kw = params(flags)
    want = oracle.correct(rs, keep_segments=True, **kw)
    sg = want["segments"]
    n = len(sg["s0"])
    assert n > 0
    with Hero(**kw) as h:
        ops, off, nops = h.align_segments(kw["aligner"] == "affine", rs.seq, rs.off, rs.seq, rs.off,
                                          sg["subject"], sg["orient"], sg["query"], sg["s0"],
                                          sg["s1"], sg["q0"], sg["q1"], sg["flags"], sg["band"])
    wl = np.diff(sg["ops_off"]).astype(np.int64)
    assert np.array_equal(nops.astype(np.int64), wl)
    for i in np.nonzero(nops)[0][:: max(1, n // 20000)]:
        a = ops[int(off[i]):int(off[i]) + int(nops[i])]
        b = sg["ops"][int(sg["ops_off"][i]):int(sg["ops_off"][i + 1])]
        assert np.array_equal(a, b), i
    # full comparison, vectorised: gather both op strings into one buffer each
    got = np.concatenate([ops[int(off[i]):int(off[i]) + int(nops[i])] for i in range(n)])
    assert np.array_equal(got, sg["ops"][:len(got)])


@pytest.mark.parametrize("affine", [0, 1])
def test_dp_random_segments(gpu_lib, oracle, affine):
    from hero_b200 import Hero
    rng = np.random.default_rng(7 + affine)
    n = 4000
    subj, query, want = [], [], []
    bands, rights, lefts = [], [], []
    for _ in range(n):
        ls, lq = int(rng.integers(1, 120)), int(rng.integers(1, 120))
        s = ACGT[rng.integers(0, 4, ls)]
        q = ACGT[rng.integers(0, 4, lq)] if rng.random() < 0.4 else np.resize(s, lq).copy()
        q[rng.random(lq) < 0.1] = ACGT[rng.integers(0, 4)]
        band = int(rng.choice([0, 1, 2, 5, 17, 300]))
        r, l = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        w, _ = oracle.align(affine, bytes(s), bytes(q), band, r, l)
        subj.append(bytes(s))
        query.append(bytes(q))
        want.append(w)
        bands.append(band)
        rights.append(r)
        lefts.append(l)
    soff = np.zeros(n + 1, np.uint64)
    soff[1:] = np.cumsum([len(x) for x in subj])
    qoff = np.zeros(n + 1, np.uint64)
    qoff[1:] = np.cumsum([len(x) for x in query])
    sseq = np.frombuffer(b"".join(subj), np.uint8)
    qseq = np.frombuffer(b"".join(query), np.uint8)
    idx = np.arange(n, dtype=np.uint32)
    zeros = np.zeros(n, np.int32)
    flags = np.array(rights, np.uint8) | (np.array(lefts, np.uint8) << 1)
    with Hero() as h:
        ops, off, nops = h.align_segments(affine, sseq, soff, qseq, qoff, idx,
                                          np.zeros(n, np.uint8), idx, zeros,
                                          np.diff(soff).astype(np.int32), zeros,
                                          np.diff(qoff).astype(np.int32), flags,
                                          np.array(bands, np.int64))
    for i in range(n):
        got = ops[int(off[i]):int(off[i]) + int(nops[i])]
        assert np.array_equal(got, want[i]), (i, affine, bands[i], rights[i], lefts[i])
