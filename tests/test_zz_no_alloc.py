"""The allocation-free DP entry point (hero_align_segments_noalloc).

It exists for callers that cannot allocate device memory themselves -- code
embedded in a host framework that owns the GPU allocator and hands out device
buffers.  Here the test plays that caller: it owns every device buffer (made
with torch), calls the entry point through the C ABI twice in a row, and
checks each result against the regular hero_align_segments entry point on the
same segments and directly against the oracle's aligner, segment by segment
(exact: the ops of a DP path are integers).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_SIDE = 128
ACGT = np.frombuffer(b"ACGT", np.uint8)


def _lib():
    from hero_b200 import load_library
    lib = load_library()
    vp = C.c_void_p
    f = lib.hero_align_segments_noalloc
    f.restype = C.c_int
    f.argtypes = ([C.c_int, vp, vp, C.c_uint64, vp, vp, C.c_uint64, C.c_uint64] + [vp] * 9 +
                  [C.c_int32, vp, vp, vp, vp])
    return lib


def _segments(seed, n_reads=300, n_seg=3000):
    """Reads (ACGT, 40..300 bp) and DP segments inside them, sides 1..MAX_SIDE."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(40, 301, size=n_reads)
    off = np.zeros(n_reads + 1, np.uint64)
    off[1:] = np.cumsum(lens)
    seq = ACGT[rng.integers(0, 4, size=int(off[-1]))]
    subj = rng.integers(0, n_reads, size=n_seg).astype(np.uint32)
    qry = rng.integers(0, n_reads, size=n_seg).astype(np.uint32)
    s0 = np.zeros(n_seg, np.int32)
    s1 = np.zeros(n_seg, np.int32)
    q0 = np.zeros(n_seg, np.int32)
    q1 = np.zeros(n_seg, np.int32)
    for i in range(n_seg):
        ls_read, lq_read = int(lens[subj[i]]), int(lens[qry[i]])
        a = int(rng.integers(1, min(MAX_SIDE, ls_read) + 1))
        b = int(rng.integers(1, min(MAX_SIDE, lq_read) + 1))
        s0[i] = rng.integers(0, ls_read - a + 1)
        s1[i] = s0[i] + a
        q0[i] = rng.integers(0, lq_read - b + 1)
        q1[i] = q0[i] + b
        if rng.random() < 0.3:  # related sequences, so the paths are not all noise
            src = seq[int(off[subj[i]]) + s0[i]:int(off[subj[i]]) + s1[i]]
            dst = np.resize(src, b).copy()
            dst[rng.random(b) < 0.05] = ACGT[rng.integers(0, 4)]
            seq[int(off[qry[i]]) + q0[i]:int(off[qry[i]]) + q1[i]] = dst
    orient = rng.integers(0, 2, size=n_seg).astype(np.uint8)
    flags = rng.integers(0, 4, size=n_seg).astype(np.uint8) & np.uint8(3)
    flags[flags == 3] = 1
    band = rng.choice([0, 1, 3, 8, 40, 300], size=n_seg).astype(np.int64)
    return seq, off, dict(subject=subj, orient=orient, query=qry, s0=s0, s1=s1, q0=q0, q1=q1,
                          flags=flags, band=band)


def _expected(affine, seq, off, sg):
    from hero_b200 import Hero
    with Hero() as h:
        ops, ops_off, nops = h.align_segments(affine, seq, off, seq, off, sg["subject"],
                                              sg["orient"], sg["query"], sg["s0"], sg["s1"],
                                              sg["q0"], sg["q1"], sg["flags"], sg["band"])
    return ops, ops_off, nops


def _noalloc(lib, affine, seq, off, sg, ops_off, max_side=MAX_SIDE):
    import torch
    dev = torch.device("cuda", 0)

    def d(a, dt=None):
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint64:
            a = a.view(np.int64)
        elif a.dtype == np.uint32:
            a = a.view(np.int32)
        return torch.from_numpy(a).to(dev)

    keep = [d(seq), d(off)] + [d(sg[k]) for k in ("subject", "orient", "query", "s0", "s1", "q0",
                                                   "q1", "flags", "band")] + [d(ops_off)]
    ops = torch.zeros(int(ops_off[-1]), dtype=torch.uint8, device=dev)
    nops = torch.zeros(len(sg["s0"]), dtype=torch.int32, device=dev)
    p = [t.data_ptr() for t in keep]
    n_reads = len(off) - 1
    rc = lib.hero_align_segments_noalloc(int(affine), p[0], p[1], n_reads, p[0], p[1], n_reads,
                                         len(sg["s0"]), *p[2:11], max_side, p[11],
                                         ops.data_ptr(), nops.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, ops.cpu().numpy(), nops.cpu().numpy()


def _compare(ops_a, off_a, n_a, ops_b, n_b):
    assert np.array_equal(n_a.astype(np.int64), n_b.astype(np.int64))
    for i in range(len(n_a)):
        a = ops_a[int(off_a[i]):int(off_a[i]) + int(n_a[i])]
        b = ops_b[int(off_a[i]):int(off_a[i]) + int(n_b[i])]
        assert np.array_equal(a, b), i


COMP = np.arange(256, dtype=np.uint8)
COMP[ord("A")], COMP[ord("T")], COMP[ord("C")], COMP[ord("G")] = ord("T"), ord("A"), ord("G"), ord("C")


def _oracle_ops(oracle, affine, seq, off, sg, i):
    """The oracle's aligner on segment i: the subject slice (of the reverse
    complement for orientation 1) against the query slice."""
    si, qi = int(sg["subject"][i]), int(sg["query"][i])
    sread = seq[int(off[si]):int(off[si + 1])]
    if sg["orient"][i]:
        sread = COMP[sread[::-1]]
    s = bytes(sread[int(sg["s0"][i]):int(sg["s1"][i])])
    q = bytes(seq[int(off[qi]) + int(sg["q0"][i]):int(off[qi]) + int(sg["q1"][i])])
    f = int(sg["flags"][i])
    ops, _ = oracle.align(affine, s, q, int(sg["band"][i]), f & 1, (f >> 1) & 1)
    return ops


def test_noalloc_matches_regular_entry_point_twice(oracle):
    lib = _lib()
    # first call: affine aligner; second call, same working array: global aligner
    for call, (seed, affine) in enumerate(((11, 1), (12, 0))):
        seq, off, sg = _segments(seed)
        want_ops, ops_off, want_n = _expected(affine, seq, off, sg)
        rc, got_ops, got_n = _noalloc(lib, affine, seq, off, sg, ops_off)
        assert rc == 0, f"call {call}: rc {rc}"
        _compare(want_ops, ops_off, want_n, got_ops, got_n)
        for i in range(len(got_n)):
            got = got_ops[int(ops_off[i]):int(ops_off[i]) + int(got_n[i])]
            assert np.array_equal(got, _oracle_ops(oracle, affine, seq, off, sg, i)), (call, i)


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = _lib()
    seq, off, sg = _segments(13, n_reads=40, n_seg=50)
    cap = ((sg["s1"] - sg["s0"]) + (sg["q1"] - sg["q0"])).astype(np.uint64)
    ops_off = np.zeros(len(cap) + 1, np.uint64)
    ops_off[1:] = np.cumsum(cap)
    rc, _, _ = _noalloc(lib, 1, seq, off, sg, ops_off, max_side=MAX_SIDE + 1)
    assert rc == -1  # HERO_E_INPUT before any launch
    # one segment wider than the limit: reported per segment, the others still aligned
    sg["s0"][0], sg["s1"][0] = 0, 0
    sg["q0"][0], sg["q1"][0] = 0, 0
    big = int(np.argmax(np.diff(off)))
    sg["subject"][0] = big
    sg["s1"][0] = min(int(off[big + 1] - off[big]), 200)
    sg["q1"][0] = 5
    cap[0] = sg["s1"][0] + 5
    ops_off[1:] = np.cumsum(cap)
    rc, _, n = _noalloc(lib, 1, seq, off, sg, ops_off)
    assert sg["s1"][0] > MAX_SIDE
    assert rc == -1 and n[0] == -1 and (n[1:] > 0).all()
    # a decreasing ops_off pair: refused for that segment instead of writing
    # through a wrapped capacity
    seq, off, sg = _segments(14, n_reads=40, n_seg=50)
    cap = ((sg["s1"] - sg["s0"]) + (sg["q1"] - sg["q0"])).astype(np.uint64)
    ops_off = np.zeros(len(cap) + 1, np.uint64)
    ops_off[1:] = np.cumsum(cap)
    ops_off[3] = ops_off[1]  # ops_off[3] < ops_off[2]: segment 2 has no valid slot
    rc, _, n = _noalloc(lib, 1, seq, off, sg, ops_off)
    assert rc == -1 and n[2] == -1
    assert (np.delete(n, 2) > 0).all()  # the other segments are still aligned
