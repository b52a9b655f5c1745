"""Test-side helpers: builds and binds the CPU checkers (oracle restatement and
the host build of the device item logic).  Only the tests use this module."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_ref", "libhero_oracle.so")
REF_BIN = os.path.join(ORACLE_DIR, "_ref", "hero_ref")
EMU_SRC = os.path.join(ROOT, "tests", "emu", "core_emu.cpp")
EMU_LIB = os.path.join(ROOT, "_build", "libcore_emu.so")


def _vp(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def build_oracle():
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("hero_oracle.cpp", "hero_oracle.h")]
    if (not os.path.exists(ORACLE_LIB) or
            any(os.path.getmtime(s) > os.path.getmtime(ORACLE_LIB) for s in srcs)):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "oracle"], check=True)
    return ORACLE_LIB


def build_emu():
    core = os.path.join(ROOT, "hero_b200", "csrc", "hero_core.cuh")
    if (not os.path.exists(EMU_LIB) or
            any(os.path.getmtime(s) > os.path.getmtime(EMU_LIB) for s in (EMU_SRC, core))):
        os.makedirs(os.path.dirname(EMU_LIB), exist_ok=True)
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", EMU_LIB, EMU_SRC],
                       check=True)
    return EMU_LIB


class OracleParams(C.Structure):
    _fields_ = [("k", C.c_int32), ("min_overlap", C.c_int32), ("affine", C.c_int32),
                ("keep_segments", C.c_int32), ("mis_rate", C.c_double),
                ("indel_rate", C.c_double), ("consensus_thr", C.c_double),
                ("aln_mode", C.c_int32), ("merge_pairs", C.c_int32), ("mapping", C.c_int32)]


class OracleStats(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in (
        "probes", "hits", "chains", "chains_kept", "records_built", "records_accepted",
        "records_kept", "dp_segments", "dp_cells")]


class Oracle:
    """CPU restatement of the reference path (oracle/hero_oracle.cpp)."""

    def __init__(self):
        lib = C.CDLL(build_oracle())
        vp = C.c_void_p
        lib.hero_oracle_correct.restype = vp
        lib.hero_oracle_correct.argtypes = [C.POINTER(OracleParams), C.c_int, C.c_uint64, vp, vp,
                                            vp, C.c_uint64, vp, vp, vp]
        lib.hero_oracle_free.argtypes = [vp]
        lib.hero_oracle_stats_get.argtypes = [vp, C.POINTER(OracleStats)]
        lib.hero_oracle_consensus.argtypes = [vp] * 8
        lib.hero_oracle_votes.argtypes = [vp, vp]
        lib.hero_oracle_num_records.argtypes = [vp]
        lib.hero_oracle_num_records.restype = C.c_uint64
        lib.hero_oracle_record_ops_total.argtypes = [vp]
        lib.hero_oracle_record_ops_total.restype = C.c_uint64
        lib.hero_oracle_num_segments.argtypes = [vp]
        lib.hero_oracle_num_segments.restype = C.c_uint64
        lib.hero_oracle_segment_ops_total.argtypes = [vp]
        lib.hero_oracle_segment_ops_total.restype = C.c_uint64
        lib.hero_oracle_segments.argtypes = [vp] * 12
        lib.hero_oracle_align.restype = C.c_int
        lib.hero_oracle_align.argtypes = [C.c_int, vp, C.c_int32, vp, C.c_int32, C.c_int64,
                                          C.c_int, C.c_int, vp, C.c_int32, C.POINTER(C.c_int64)]
        lib.hero_oracle_quality_filter.argtypes = [vp, C.c_uint64]
        lib.hero_oracle_aln_size.argtypes = [vp]
        lib.hero_oracle_aln_size.restype = C.c_uint64
        lib.hero_oracle_aln.argtypes = [vp, vp]
        lib.hero_oracle_merged.argtypes = [vp, vp, vp]
        lib.hero_oracle_overhang.argtypes = [vp, vp]
        lib.hero_oracle_mapping_histogram.argtypes = [vp, vp, C.c_uint64]
        lib.hero_oracle_mapping_histogram.restype = C.c_uint64
        lib.hero_oracle_merge_pair.argtypes = [vp, C.c_int32, vp, C.c_int32, vp, vp, vp]
        lib.hero_oracle_merge_pair.restype = C.c_int
        lib.hero_oracle_record_list.argtypes = [C.c_uint32, vp, vp, vp, vp]
        lib.hero_oracle_record_list.restype = C.c_int32
        lib.hero_oracle_columns.argtypes = [C.c_uint64, vp, C.c_double, vp]
        lib.hero_oracle_record_score.argtypes = [C.c_uint32, vp, vp, vp, vp, vp]
        lib.hero_oracle_chain.argtypes = [C.c_int32, C.c_double, C.c_uint32, vp, vp, vp, vp]
        lib.hero_oracle_chain.restype = C.c_int32
        lib.hero_oracle_chain_layout.argtypes = ([C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                                  C.c_double, vp, C.c_int32, vp, C.c_int32,
                                                  C.c_uint32, vp, vp, vp, C.c_int32, vp, vp])
        lib.hero_oracle_chain_layout.restype = C.c_int32
        lib.hero_oracle_record_text.argtypes = ([C.c_uint64, C.c_uint32, C.c_int64, C.c_uint32, vp,
                                                 vp, vp, vp, C.c_int32, C.c_int32, vp, C.c_int32])
        lib.hero_oracle_record_text.restype = C.c_int32
        lib.hero_oracle_key_positions.argtypes = [C.c_int64, C.c_int64, vp]
        lib.hero_oracle_key_positions.restype = C.c_int32
        self.lib = lib

    def correct(self, reads, subjects=None, k=39, min_overlap=40, aligner="global",
                max_mismatch_rate=1.0, max_indel_rate=1.0, consensus_threshold=0.6,
                keep_segments=False, threads=8, aln=False, merge=False, mapping=False):
        """aln=True: the alignment-output mode (no -c); res["aln"] holds the .aln bytes.
        merge=True: --merge; res["merged_seq"], res["merged_len"], res["overhang"]."""
        subj = subjects if subjects is not None else reads
        p = OracleParams(k, min_overlap, 1 if aligner in ("a", "affine") else 0,
                         1 if keep_segments else 0, max_mismatch_rate, max_indel_rate,
                         consensus_threshold, 1 if aln else 0, 1 if merge else 0,
                         1 if mapping else 0)
        qs, qo, qu = reads.seq, reads.off.astype(np.uint64), reads.names.astype(np.int64)
        ss, so, su = subj.seq, subj.off.astype(np.uint64), subj.names.astype(np.int64)
        h = self.lib.hero_oracle_correct(C.byref(p), threads, reads.n, _vp(qs), _vp(qo), _vp(qu),
                                         subj.n, _vp(ss), _vp(so), _vp(su))
        if not h:
            raise RuntimeError("oracle rejected the input")
        try:
            n, nb = reads.n, len(reads.seq)
            res = dict(seq=np.zeros(nb, np.uint8), imin=np.zeros(n, np.uint32),
                       imed=np.zeros(n, np.uint32), imax=np.zeros(n, np.uint32),
                       mismatch_rate=np.zeros(n), gc=np.zeros(n), good=np.zeros(n, np.uint8))
            self.lib.hero_oracle_consensus(h, *[_vp(res[k_]) for k_ in (
                "seq", "imin", "imed", "imax", "mismatch_rate", "gc", "good")])
            cov = np.zeros(nb * 4, np.uint32)
            self.lib.hero_oracle_votes(h, _vp(cov))
            res["votes"] = cov
            if merge:
                res["merged_seq"] = np.zeros(nb, np.uint8)
                res["merged_len"] = np.zeros(n // 2, np.uint32)
                res["overhang"] = np.zeros(n * 80, np.uint32)
                self.lib.hero_oracle_merged(h, _vp(res["merged_seq"]), _vp(res["merged_len"]))
                self.lib.hero_oracle_overhang(h, _vp(res["overhang"]))
            if mapping:
                nh = self.lib.hero_oracle_mapping_histogram(h, None, 0)
                hb = np.zeros(max(1, nh), np.uint8)
                self.lib.hero_oracle_mapping_histogram(h, _vp(hb), nh)
                res["histogram"] = hb[:nh].tobytes()
            if aln:
                buf = np.zeros(max(1, self.lib.hero_oracle_aln_size(h)), np.uint8)
                self.lib.hero_oracle_aln(h, _vp(buf))
                res["aln"] = buf[:self.lib.hero_oracle_aln_size(h)].tobytes()
            st = OracleStats()
            self.lib.hero_oracle_stats_get(h, C.byref(st))
            res["stats"] = {f: getattr(st, f) for f, _ in st._fields_}
            if keep_segments:
                ns = self.lib.hero_oracle_num_segments(h)
                tot = self.lib.hero_oracle_segment_ops_total(h)
                seg = dict(subject=np.zeros(ns, np.uint32), orient=np.zeros(ns, np.uint8),
                           query=np.zeros(ns, np.uint32), s0=np.zeros(ns, np.int32),
                           s1=np.zeros(ns, np.int32), q0=np.zeros(ns, np.int32),
                           q1=np.zeros(ns, np.int32), flags=np.zeros(ns, np.uint8),
                           band=np.zeros(ns, np.int64), ops_off=np.zeros(ns + 1, np.uint64),
                           ops=np.zeros(max(tot, 1), np.uint8))
                self.lib.hero_oracle_segments(h, *[_vp(seg[k_]) for k_ in (
                    "subject", "orient", "query", "s0", "s1", "q0", "q1", "flags", "band",
                    "ops_off", "ops")])
                res["segments"] = seg
            return res
        finally:
            self.lib.hero_oracle_free(h)

    def align(self, affine, subj: bytes, query: bytes, band, right=False, left=False):
        s = np.frombuffer(subj, np.uint8).copy()
        q = np.frombuffer(query, np.uint8).copy()
        ops = np.zeros(len(s) + len(q) + 1, np.uint8)
        bu = C.c_int64()
        n = self.lib.hero_oracle_align(int(affine), _vp(s), len(s), _vp(q), len(q), int(band),
                                       int(right), int(left), _vp(ops), len(ops), C.byref(bu))
        return ops[:n].copy(), bu.value


class Emu:
    """Host build of hero_core.cuh (the device item logic) driven sequentially."""

    def __init__(self):
        lib = C.CDLL(build_emu())
        vp = C.c_void_p
        lib.emu_align.argtypes = [C.c_int, vp, C.c_int32, vp, C.c_int32, C.c_int64, C.c_int,
                                  C.c_int, C.c_int, vp, C.c_int32]
        lib.emu_align_wave.argtypes = [C.c_int, vp, C.c_int32, vp, C.c_int32, C.c_int64, C.c_int,
                                       C.c_int, vp, C.c_int32]
        lib.emu_correct.argtypes = ([C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                     C.c_double, C.c_uint64] + [vp] * 11)
        lib.emu_align_output.argtypes = ([C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                          C.c_uint64, vp, vp, vp, vp, C.c_uint64])
        lib.emu_align_output.restype = C.c_int64
        lib.emu_merge.argtypes = ([C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                   C.c_double, C.c_uint64] + [vp] * 7)
        lib.emu_merge.restype = C.c_int
        lib.emu_merge_pair.argtypes = [vp, C.c_int32, vp, C.c_int32, vp, vp, vp]
        lib.emu_merge_pair.restype = C.c_int
        lib.emu_record_list.argtypes = [C.c_uint32, vp, vp, vp, vp]
        lib.emu_record_list.restype = C.c_int32
        lib.emu_columns.argtypes = [C.c_uint64, vp, C.c_double, vp]
        lib.emu_record_score.argtypes = [C.c_uint32, vp, vp, vp, vp, vp]
        lib.emu_chain.argtypes = [C.c_int32, C.c_double, C.c_uint32, vp, vp, vp, vp]
        lib.emu_chain.restype = C.c_int32
        lib.emu_chain_layout.argtypes = ([C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                          vp, C.c_int32, vp, C.c_int32, C.c_uint32, vp, vp, vp,
                                          C.c_int32, vp, vp])
        lib.emu_chain_layout.restype = C.c_int32
        lib.emu_record_text.argtypes = ([C.c_uint64, C.c_uint32, C.c_int64, C.c_uint32, vp, vp, vp,
                                         vp, C.c_int32, C.c_int32, vp, C.c_int32])
        lib.emu_record_text.restype = C.c_int32
        lib.emu_key_positions.argtypes = [C.c_int64, C.c_int64, vp]
        lib.emu_key_positions.restype = C.c_int32
        lib.emu_ops_summary_groups.argtypes = [vp, C.c_uint32, C.c_uint32]
        lib.emu_ops_summary_groups.restype = C.c_int32
        self.lib = lib

    def merge(self, reads, k=39, min_overlap=40, aligner="global", max_mismatch_rate=1.0,
              max_indel_rate=1.0, consensus_threshold=0.6):
        """--merge: the corrected reads, the merged pairs and the overhang votes."""
        n, nb = reads.n, len(reads.seq)
        res = dict(seq=np.zeros(nb, np.uint8), merged_seq=np.zeros(nb, np.uint8),
                   merged_len=np.zeros(n // 2, np.uint32), overhang=np.zeros(n * 80, np.uint32))
        off = reads.off.astype(np.uint64)
        uid = reads.names.astype(np.int64)
        rc = self.lib.emu_merge(k, min_overlap, 1 if aligner in ("a", "affine") else 0,
                                max_mismatch_rate, max_indel_rate, consensus_threshold, n,
                                _vp(reads.seq), _vp(off), _vp(uid), _vp(res["seq"]),
                                _vp(res["merged_seq"]), _vp(res["merged_len"]),
                                _vp(res["overhang"]))
        if rc != 0:
            raise ValueError("an odd number of reads cannot be paired")
        return res

    def align_output(self, reads, k=39, min_overlap=40, aligner="global", max_mismatch_rate=1.0,
                     max_indel_rate=1.0, cap=None):
        """The .aln text of the alignment-output mode (reads against themselves)."""
        cap = cap or (len(reads.seq) * 64 + reads.n * 64 + 1024)
        out = np.zeros(cap, np.uint8)
        off = reads.off.astype(np.uint64)
        uid = reads.names.astype(np.int64)
        n = self.lib.emu_align_output(k, min_overlap, 1 if aligner in ("a", "affine") else 0,
                                      max_mismatch_rate, max_indel_rate, reads.n, _vp(reads.seq),
                                      _vp(off), _vp(uid), _vp(out), cap)
        if n < 0:
            return self.align_output(reads, k, min_overlap, aligner, max_mismatch_rate,
                                     max_indel_rate, cap * 4)
        return out[:n].tobytes()

    def align(self, affine, subj: bytes, query: bytes, band, right=False, left=False, strip16=False):
        s = np.frombuffer(subj, np.uint8).copy()
        q = np.frombuffer(query, np.uint8).copy()
        ops = np.zeros(len(s) + len(q) + 1, np.uint8)
        n = self.lib.emu_align(int(affine), _vp(s), len(s), _vp(q), len(q), int(band), int(right),
                               int(left), int(strip16), _vp(ops), len(ops))
        return ops[:n].copy()

    def align_wave(self, affine, subj: bytes, query: bytes, band, right=False, left=False):
        s = np.frombuffer(subj, np.uint8).copy()
        q = np.frombuffer(query, np.uint8).copy()
        ops = np.zeros(len(s) + len(q) + 1, np.uint8)
        n = self.lib.emu_align_wave(int(affine), _vp(s), len(s), _vp(q), len(q), int(band),
                                    int(right), int(left), _vp(ops), len(ops))
        return ops[:n].copy()

    def correct(self, reads, k=39, min_overlap=40, aligner="global", max_mismatch_rate=1.0,
                max_indel_rate=1.0, consensus_threshold=0.6):
        n, nb = reads.n, len(reads.seq)
        res = dict(seq=np.zeros(nb, np.uint8), imin=np.zeros(n, np.uint32),
                   imed=np.zeros(n, np.uint32), imax=np.zeros(n, np.uint32),
                   mismatch_rate=np.zeros(n), gc=np.zeros(n))
        cov = np.zeros(nb * 4, np.uint32)
        ctr = np.zeros(8, np.uint64)
        off = reads.off.astype(np.uint64)
        uid = reads.names.astype(np.int64)
        self.lib.emu_correct(k, min_overlap, 1 if aligner in ("a", "affine") else 0,
                             max_mismatch_rate, max_indel_rate, consensus_threshold, n,
                             _vp(reads.seq), _vp(off), _vp(uid), *[_vp(res[k_]) for k_ in (
                                 "seq", "imin", "imed", "imax", "mismatch_rate", "gc")],
                             _vp(cov), _vp(ctr))
        res["votes"] = cov
        res["counters"] = ctr
        return res


CONSENSUS_KEYS = ("seq", "imin", "imed", "imax")


def assert_same_consensus(a, b, what=""):
    """Exact equality of corrected reads, statistics and the two double columns (bitwise)."""
    for key in CONSENSUS_KEYS:
        if not np.array_equal(a[key], b[key]):
            idx = np.nonzero(a[key] != b[key])[0][:5]
            raise AssertionError(f"{what}: {key} differs at {idx}")
    for key in ("mismatch_rate", "gc"):
        x = np.asarray(a[key], np.float64).view(np.uint64)
        y = np.asarray(b[key], np.float64).view(np.uint64)
        nan = np.isnan(a[key]) & np.isnan(b[key])
        bad = (x != y) & ~nan
        if bad.any():
            raise AssertionError(f"{what}: {key} differs at {np.nonzero(bad)[0][:5]}")


def format_outputs(uid, seq, off, imin, imed, imax, mis, gc):
    """.fasta/.info bytes as QueryDataset::writeQueryOut prints them (--singleReads)."""
    fa = []
    info = []
    for i in range(len(uid)):
        s = bytes(seq[int(off[i]):int(off[i + 1])])
        fa.append(b">%d\n%s\n" % (int(uid[i]), s))
        info.append(b"%d\t%d\t%d\t%d\t%d\t%s\t%s\n" % (
            int(uid[i]), int(imin[i]), int(imed[i]), int(imax[i]), int(off[i + 1] - off[i]),
            _g(mis[i]), _g(gc[i])))
    return b"".join(fa), b"".join(info)


def format_merged(uid, merged_seq, off, merged_len):
    """QueryDataset::writeQueryOut with --merge (QueryDataset.cpp:417-459): per
    pair (2p, 2p+1), the merged read into _merged.fasta, else both reads into
    _unmerged.fasta (isGoodRead() is always true)."""
    merged, unmerged = [], []
    for p in range(len(merged_len)):
        a = int(off[2 * p])
        if merged_len[p]:
            merged.append(b">%d\n%s\n" % (int(uid[2 * p]), bytes(merged_seq[a:a + int(merged_len[p])])))
        else:
            for r in (2 * p, 2 * p + 1):
                unmerged.append(b">%d\n%s\n" % (int(uid[r]), bytes(merged_seq[int(off[r]):int(off[r + 1])])))
    return b"".join(merged), b"".join(unmerged)


def _g(x: float) -> bytes:
    # std::ostream default formatting (precision 6, %g style)
    if x != x:
        return b"nan" if np.copysign(1.0, x) > 0 else b"-nan"
    return (b"%g" % x)


def merge_pair(lib, prefix, left: bytes, right: bytes, extL, extR):
    """One pair through <prefix>_merge_pair (oracle or emulator): merged bytes or None."""
    l = np.frombuffer(left, np.uint8).copy()
    r = np.frombuffer(right, np.uint8).copy()
    eL = np.ascontiguousarray(extL, np.uint32)
    eR = np.ascontiguousarray(extR, np.uint32)
    out = np.zeros(len(l) + len(r) + 1, np.uint8)
    n = getattr(lib, prefix + "_merge_pair")(_vp(l), len(l), _vp(r), len(r), _vp(eL), _vp(eR),
                                             _vp(out))
    return out[:n].tobytes() if n else None


def record_list(lib, prefix, key, rate_sum, length):
    """Record indices kept by SubjectRead::addAlignment's list, in list order."""
    k = np.ascontiguousarray(key, np.uint64)
    r = np.ascontiguousarray(rate_sum, np.float64)
    ln = np.ascontiguousarray(length, np.float64)
    out = np.zeros(max(1, len(k)), np.uint32)
    n = getattr(lib, prefix + "_record_list")(len(k), _vp(k), _vp(r), _vp(ln), _vp(out))
    return out[:n].tolist()


def columns(lib, prefix, counts, thr):
    """Called row per consensus column (counts [n][4], A,C,T,G), -1 where none."""
    c = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros(max(1, len(c)), np.int32)
    getattr(lib, prefix + "_columns")(len(c), _vp(c), float(thr), _vp(out))
    return out[:len(c)]


def record_score(lib, prefix, piece, typ, count, letter):
    """(mismatches, indels, length) of a record given as events (see the oracle header)."""
    pc = np.ascontiguousarray(piece, np.uint32)
    t = np.ascontiguousarray(typ, np.uint8)
    c = np.ascontiguousarray(count, np.int32)
    le = np.ascontiguousarray(letter, np.uint8)
    out = np.zeros(3, np.int64)
    getattr(lib, prefix + "_record_score")(len(t), _vp(pc), _vp(t), _vp(c), _vp(le), _vp(out))
    return tuple(int(x) for x in out)


def chain(lib, prefix, k, indel_rate, posQ, posS):
    """Chain of each hit and the kept chains of one query group (hits sorted)."""
    q = np.ascontiguousarray(posQ, np.int64)
    s_ = np.ascontiguousarray(posS, np.int64)
    chain_of = np.zeros(max(1, len(q)), np.uint32)
    kept = np.zeros(max(1, len(q)), np.uint8)
    nch = getattr(lib, prefix + "_chain")(k, float(indel_rate), len(q), _vp(q), _vp(s_),
                                          _vp(chain_of), _vp(kept))
    return chain_of[:len(q)].tolist(), kept[:nch].tolist()


def chain_layout(lib, prefix, k, l, affine, mis_rate, indel_rate, query: bytes, subject: bytes,
                 posQ, posS):
    """(DP calls as 6-tuples, record position, status) of one chain of keys."""
    q = np.frombuffer(query, np.uint8).copy()
    s_ = np.frombuffer(subject, np.uint8).copy()
    pq = np.ascontiguousarray(posQ, np.int64)
    ps = np.ascontiguousarray(posS, np.int64)
    cap = 2 * len(pq) + 4
    seg = np.zeros(6 * cap, np.int64)
    pos = C.c_int64()
    st = C.c_int32()
    n = getattr(lib, prefix + "_chain_layout")(k, l, int(affine), float(mis_rate),
                                              float(indel_rate), _vp(q), len(q), _vp(s_), len(s_),
                                              len(pq), _vp(pq), _vp(ps), _vp(seg), cap,
                                              C.byref(pos), C.byref(st))
    return [tuple(seg[6 * i:6 * i + 6].tolist()) for i in range(n)], pos.value, st.value


def record_text(lib, prefix, key, orient, pos, piece, typ, count, query: bytes, qrc):
    """One .aln record's text from events (see the oracle header)."""
    pc = np.ascontiguousarray(piece, np.uint32)
    t = np.ascontiguousarray(typ, np.uint8)
    c = np.ascontiguousarray(count, np.int32)
    q = np.frombuffer(query, np.uint8).copy()
    cap = 64 + 16 * len(t) + 2 * len(q)
    out = np.zeros(cap, np.uint8)
    n = getattr(lib, prefix + "_record_text")(key, orient, pos, len(t), _vp(pc), _vp(t), _vp(c),
                                              _vp(q), len(q), int(qrc), _vp(out), cap)
    assert n >= 0
    return out[:n].tobytes()
