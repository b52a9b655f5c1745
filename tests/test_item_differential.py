"""Randomised differential checks of items whose rules are subtle, each through
the shared device logic (hero_core.cuh, host build) and through the oracle's
independent restatement: the --merge pair merge (QueryRead::mergingPairedReads),
the alignment output's record list (SubjectRead::addAlignment keyed by query
uniqueId), a record's score from its run ends and DP-piece summaries
(AlignmentRecord::calculateScore), the chaining of a query group
(isFromTheSameAlignment's ratio test, markTheBestPossibleAlignment) and the
consensus call of a column (QueryRead::callConsensus, whose
device form scans integer counts and divides only the two kept ones)."""
import numpy as np
from hero_testlib import chain, columns, merge_pair, record_list, record_score, record_text

COMP = bytes.maketrans(b"ACGTN", b"TGCAJ")


def _ext(rng, seq: bytes, n: int, noise: float):
    """Overhang votes that spell seq's first n letters (with noise votes)."""
    m = np.zeros((20, 4), np.uint32)
    code = {ord("A"): 0, ord("C"): 1, ord("T"): 2, ord("G"): 3}
    for i in range(min(n, 20, len(seq))):
        m[i, code.get(seq[i], 0)] += rng.integers(1, 6)
        if rng.random() < noise:
            m[i, rng.integers(4)] += rng.integers(1, 6)  # ties and other letters
    return m.reshape(-1)


def test_pair_merge_agrees(oracle, emu):
    rng = np.random.default_rng(17)
    bases = np.frombuffer(b"ACGT", np.uint8)
    merged = 0
    for t in range(3000):
        flen = int(rng.integers(60, 320))
        frag = bases[rng.integers(0, 4, flen)].tobytes()
        la, lb = int(rng.integers(20, 160)), int(rng.integers(20, 160))
        left = frag[:la]
        right = frag[max(0, flen - lb):][::-1].translate(COMP)  # reverse complement of the end
        if rng.random() < 0.3:  # a substitution somewhere
            b = bytearray(left if rng.random() < 0.5 else right)
            if b:
                b[int(rng.integers(len(b)))] = int(bases[rng.integers(4)])
            left, right = (bytes(b), right) if len(b) == len(left) and rng.random() < 0.5 else (left, bytes(b) if len(b) == len(right) else right)
        if rng.random() < 0.05:
            left = left[:-1] + b"N"
        # extensions: what lies past each read's end on the fragment (or noise)
        extL = _ext(rng, frag[la:], int(rng.integers(0, 21)), 0.2)
        tail = frag[:max(0, flen - lb)][::-1].translate(COMP)
        extR = _ext(rng, tail, int(rng.integers(0, 21)), 0.2)
        a = merge_pair(oracle.lib, "hero_oracle", left, right, extL, extR)
        b = merge_pair(emu.lib, "emu", left, right, extL, extR)
        assert a == b, (t, left, right)
        merged += a is not None
    assert 300 < merged < 2900  # both outcomes are exercised


def test_record_list_agrees(oracle, emu):
    rng = np.random.default_rng(19)
    for t in range(2000):
        n = int(rng.integers(0, 40))
        # few distinct keys in arbitrary order (repeats, descending runs), few rate
        # values and lengths (ties on both)
        key = rng.integers(0, 12, n).astype(np.uint64)
        if rng.random() < 0.3:
            key = np.sort(key)
        rate = rng.integers(0, 4, n) / 8.0
        length = rng.integers(40, 44, n).astype(np.float64)
        a = record_list(oracle.lib, "hero_oracle", key, rate, length)
        b = record_list(emu.lib, "emu", key, rate, length)
        assert a == b, (t, key.tolist(), rate.tolist(), length.tolist())


def test_consensus_columns_agree(oracle, emu):
    rng = np.random.default_rng(23)
    parts = [rng.integers(0, 6, (20000, 4)),                      # small counts: ties
             rng.integers(0, 200, (20000, 4)),
             rng.integers(0, 2 ** 20, (5000, 4)),                 # deep columns
             np.array([[0, 0, 0, 0], [1, 0, 0, 0], [3, 2, 0, 0], [2, 2, 1, 0],
                       [0, 3, 0, 2], [6, 0, 4, 0], [5, 0, 0, 0], [4, 1, 0, 0]])]
    counts = np.concatenate(parts).astype(np.uint32)
    # fractions exactly at the threshold: a = round(thr * s) + b
    for s_ in (5, 10, 20, 50, 100, 1000):
        for thr in (0.6, 0.7, 0.5):
            a = int(round(thr * s_))
            counts = np.concatenate([counts, np.array([[a, s_ - a, 0, 0], [0, s_ - a, a, 0]],
                                                       np.uint32)])
    for thr in (0.6, 0.7, 0.5, 0.0 + 1e-12, 0.99):
        a = columns(oracle.lib, "hero_oracle", counts, thr)
        b = columns(emu.lib, "emu", counts, thr)
        bad = np.nonzero(a != b)[0]
        assert bad.size == 0, (thr, counts[bad[:5]].tolist(), a[bad[:5]], b[bad[:5]])


def test_record_scores_agree(oracle, emu):
    """Records as the chain walk builds them: k-mer runs (M, and I / D between
    keys) and DP pieces of single steps (M, mismatch with a letter, I, D)."""
    rng = np.random.default_rng(29)
    letters = np.frombuffer(b"ACGT", np.uint8)
    for t in range(3000):
        piece, typ, count, letter = [], [], [], []
        npc = 0
        for _ in range(int(rng.integers(1, 7))):
            if rng.random() < 0.5:  # a run outside the DP
                piece.append(0)
                typ.append(int(rng.choice([0, 0, 2, 3])))
                count.append(int(rng.integers(1, 40)))
                letter.append(0)
            else:  # a DP piece: steps with runs of equal ops
                npc += 1
                for _ in range(int(rng.integers(1, 6))):
                    op = int(rng.choice([0, 0, 1, 2, 3]))
                    for _ in range(int(rng.integers(1, 5))):
                        piece.append(npc)
                        typ.append(op)
                        count.append(1)
                        letter.append(int(letters[rng.integers(4)]))
        a = record_score(oracle.lib, "hero_oracle", piece, typ, count, letter)
        b = record_score(emu.lib, "emu", piece, typ, count, letter)
        assert a == b, (t, list(zip(piece, typ, count)))


def test_chaining_agrees(oracle, emu):
    """Groups of hits sorted by (posQ, posS); indel rates include ratios that a
    candidate hit meets exactly (the test is a strict >)."""
    rng = np.random.default_rng(31)
    for t in range(3000):
        k = int(rng.choice([21, 31, 39]))
        n = int(rng.integers(1, 25))
        q = rng.integers(0, 120, n)
        d = rng.integers(-6, 7, n) * (rng.random(n) < 0.5)  # near-diagonal and off-diagonal hits
        s_ = np.clip(q + 10 + d + rng.integers(0, 3, n) * 40, 0, 300)
        order = np.lexsort((s_, q))
        q, s_ = q[order], s_[order]
        if rng.random() < 0.5:  # a ratio some pair meets exactly
            i, j = sorted(rng.choice(n, 2)) if n > 1 else (0, 0)
            lq, ls = abs(int(q[j]) - int(q[i])), abs(int(s_[j]) - int(s_[i]))
            rate = abs(lq - ls) / (max(lq, ls) + k)
        else:
            rate = float(rng.choice([0.0, 0.01, 0.02, 0.05, 0.2, 1.0]))
        a = chain(oracle.lib, "hero_oracle", k, rate, q, s_)
        b = chain(emu.lib, "emu", k, rate, q, s_)
        assert a == b, (t, k, rate, q.tolist(), s_.tolist())


def test_chain_layout_agrees(oracle, emu):
    """getAlignment2 on random chains: every geometry of the start, middle and end
    pieces (keys overlapping, adjacent, apart; diagonal shifts both ways; reads
    of unequal length), with and without early exits: the DP calls made, the
    record's position and its fate."""
    from hero_testlib import chain_layout
    rng = np.random.default_rng(37)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    fates = set()
    for t in range(1500):
        k = int(rng.choice([11, 21, 39]))
        n = int(rng.integers(1, 6))
        q0, s0 = int(rng.integers(0, 60)), int(rng.integers(0, 60))
        if rng.random() < 0.2:
            q0 = 0
        if rng.random() < 0.2:
            s0 = 0
        pq, ps = [q0], [s0]
        for _ in range(n - 1):
            dq = int(rng.integers(1, 2 * k + 10))
            ds = dq if rng.random() < 0.4 else int(rng.integers(1, 2 * k + 10))
            pq.append(pq[-1] + dq)
            ps.append(ps[-1] + ds)
        Lq = pq[-1] + k + int(rng.integers(0, 60))
        Ls = ps[-1] + k + int(rng.integers(0, 60))
        if rng.random() < 0.15:
            Ls = ps[-1] + k  # the last key at the subject's end
        query = acgt[rng.integers(0, 4, Lq)].tobytes()
        subject = bytearray(acgt[rng.integers(0, 4, Ls)].tobytes())
        for a, b in zip(pq, ps):  # the keys match
            subject[b:b + k] = query[a:a + k]
        mis, ind = (1.0, 1.0) if rng.random() < 0.5 else (float(rng.choice([0.02, 0.1, 0.3])),
                                                           float(rng.choice([0.01, 0.05, 0.2])))
        l = int(rng.choice([20, 40, 80]))
        affine = bool(rng.random() < 0.5)
        a = chain_layout(oracle.lib, "hero_oracle", k, l, affine, mis, ind, query, bytes(subject),
                         pq, ps)
        b = chain_layout(emu.lib, "emu", k, l, affine, mis, ind, query, bytes(subject), pq, ps)
        assert a == b, (t, k, l, affine, mis, ind, pq, ps, Lq, Ls)
        fates.add(a[2])
    assert fates == {0, 1, 2}


def test_record_text_agrees(oracle, emu):
    """.aln record text: run-length entries across runs and DP pieces, mismatch
    letters from the (reverse-complemented) query, inserted bases of inner I
    entries only; ids above 2^63 print unsigned, positions signed."""
    rng = np.random.default_rng(41)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    for t in range(2000):
        piece, typ, count = [], [], []
        npc, qlen = 0, 0
        for _ in range(int(rng.integers(1, 7))):
            if rng.random() < 0.5:
                op = int(rng.choice([0, 0, 2, 3]))
                c = int(rng.integers(1, 30))
                piece.append(0)
                typ.append(op)
                count.append(c)
                qlen += c if op != 3 else 0
            else:
                npc += 1
                for _ in range(int(rng.integers(1, 8))):
                    op = int(rng.choice([0, 1, 1, 2, 3]))
                    piece.append(npc)
                    typ.append(op)
                    count.append(1)
                    qlen += 1 if op != 3 else 0
        query = acgt[rng.integers(0, 4, qlen + int(rng.integers(0, 5)))].tobytes()
        key = int(rng.choice([0, 7, 12345, 2 ** 64 - 5]))
        orient = int(rng.integers(0, 2))
        pos = int(rng.integers(0, 300))
        qrc = bool(rng.random() < 0.5)
        a = record_text(oracle.lib, "hero_oracle", key, orient, pos, piece, typ, count, query, qrc)
        b = record_text(emu.lib, "emu", key, orient, pos, piece, typ, count, query, qrc)
        assert a == b, (t, a, b)


def test_query_key_positions_agree(oracle, emu):
    """The k-mers a query read puts in the table (every k-th, then the tail).
    Reads shorter than k are outside the reference's domain (its substr throws)."""
    import ctypes as C
    out_a = np.zeros(2048, np.int64)
    out_b = np.zeros(2048, np.int64)
    for k in range(1, 64):
        for L in range(k, 400):
            na = oracle.lib.hero_oracle_key_positions(L, k, out_a.ctypes.data_as(C.c_void_p))
            nb = emu.lib.emu_key_positions(L, k, out_b.ctypes.data_as(C.c_void_p))
            assert na == nb and np.array_equal(out_a[:na], out_b[:nb]), (L, k)
