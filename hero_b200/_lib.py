"""ctypes binding of libhero_b200.so (the C ABI declared in include/hero_gpu.h).

The library is built in-tree by ``hero_b200.build`` (nvcc, sm_100a).  Loading
fails loudly when it is missing: there is no CPU path behind this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhero_b200.so")

HERO_OK = 0
ERRORS = {-1: "HERO_E_INPUT", -2: "HERO_E_OOM", -3: "HERO_E_CUDA", -4: "HERO_E_STATE",
          -5: "HERO_E_TIMEOUT"}
ALIGNER_AFFINE = 0
ALIGNER_GLOBAL = 1

# every entry point include/hero_gpu.h declares
EXPORTS = [
    "hero_default_params", "hero_create", "hero_destroy", "hero_last_error",
    "hero_set_queries", "hero_build_index", "hero_align_subjects", "hero_align_self",
    "hero_consensus", "hero_get_votes", "hero_get_stats", "hero_align_segments",
    "hero_reset_votes", "hero_align_segments_noalloc", "hero_round", "hero_fetch",
    "hero_set_query_jobs", "hero_server_create", "hero_server_destroy", "hero_job_submit",
    "hero_job_poll", "hero_job_wait", "hero_job_result", "hero_job_error", "hero_job_release",
    "hero_server_get_stats", "hero_job_bytes", "hero_round_admit", "hero_set_dp_tuning",
    "hero_server_set_dp_tuning", "hero_alignments_size", "hero_alignments_take",
    "hero_align_self_range", "hero_votes_words", "hero_votes_save", "hero_votes_load",
    "hero_merge_pairs", "hero_get_overhang", "hero_mapping_histogram", "hero_set_vote_buffer",
    "hero_consensus_range", "hero_server_set_round_policy", "hero_server_worker_stats",
    "hero_server_workers", "hero_dp_tuning_check", "hero_device_init",
]

# hero_params.flags: the alignment-output mode (HERO without -c); --merge
FLAG_ALIGNMENT_OUTPUT = 1
FLAG_MERGE_PAIRS = 2
FLAG_MAPPING = 4

# the autotuner's record (hero_b200.autotune); loaded by every Hero unless told otherwise
TUNING_PATH = os.path.join(HERE, "tuning.json")

JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


class HeroParams(C.Structure):
    _fields_ = [
        ("k", C.c_int32), ("min_overlap", C.c_int32), ("aligner", C.c_int32),
        ("device", C.c_int32), ("max_mismatch_rate", C.c_double),
        ("max_indel_rate", C.c_double), ("consensus_threshold", C.c_double),
        ("device_memory_budget", C.c_uint64), ("subject_batch", C.c_uint32),
        ("flags", C.c_uint32), ("stream", C.c_void_p),
    ]


_STAT_FIELDS = [
    "queries", "good_queries", "index_keys", "index_slots", "subjects", "probes", "hits",
    "chains", "chains_kept", "records_built", "records_accepted", "records_kept",
    "dp_segments", "dp_segments_ref", "dp_cells", "vote_anomalies", "device_bytes_peak",
    "kernel_launches",
]
_STAT_MS = ["ms_upload", "ms_index", "ms_seed", "ms_chain", "ms_dp", "ms_record", "ms_vote",
            "ms_consensus", "ms_dp_kernel", "ms_align_wall"]


class HeroStats(C.Structure):
    _fields_ = ([(f, C.c_uint64) for f in _STAT_FIELDS] + [(f, C.c_double) for f in _STAT_MS] +
                [("graph_rounds", C.c_uint64), ("dp_cells_computed", C.c_uint64),
                 ("dp_rows_max", C.c_uint64), ("dp_cells_pairs", C.c_uint64),
                 ("buffer_allocs", C.c_uint64), ("ms_alloc", C.c_double),
                 ("dp_tasks_staged", C.c_uint64), ("dp_stage_timeouts", C.c_uint64)])


class DpTuning(C.Structure):
    _fields_ = [("rows_max", C.c_int32), ("warps_per_block", C.c_int32),
                ("pair_strips", C.c_uint32), ("chunk_strips", C.c_uint32),
                ("regs_per_thread", C.c_int32)]


def load_tuning(path: str | None = None, aligner: str = "affine") -> list[dict]:
    """Classes recorded by the autotuner for an aligner (empty when there is no
    record): "classes" holds the affine aligner's, "classes_global" the global's."""
    import json
    p = path or os.environ.get("HERO_B200_TUNING") or TUNING_PATH
    if not p or not os.path.exists(p):
        return []
    with open(p) as f:
        rec = json.load(f)
    key = "classes" if aligner in ("a", "affine") else "classes_global"
    return rec.get(key, [])


class JobInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("round", C.c_uint64),
                ("round_jobs", C.c_uint32), ("reserved", C.c_uint32), ("bases", C.c_uint64),
                ("reads", C.c_uint64), ("submit_ms", C.c_double), ("start_ms", C.c_double),
                ("done_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = ([(f, C.c_uint64) for f in ("jobs_submitted", "jobs_done", "jobs_failed", "rounds",
                                            "bases_done", "round_bytes_budget")] +
                [("busy_ms", C.c_double), ("uptime_ms", C.c_double),
                 ("overlapped_rounds", C.c_uint64), ("ms_stage_in", C.c_double),
                 ("ms_round_calls", C.c_double), ("ms_stage_out", C.c_double),
                 ("buffer_allocs", C.c_uint64), ("ms_alloc", C.c_double),
                 ("overlapped_compute", C.c_uint64)])


_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("HERO_B200_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build it with `python -m hero_b200.build` (nvcc, sm_100a). "
            "There is no CPU fallback.")
    lib = C.CDLL(p)
    vp = C.c_void_p
    lib.hero_default_params.argtypes = [C.POINTER(HeroParams)]
    lib.hero_create.argtypes = [C.POINTER(HeroParams), C.POINTER(vp)]
    lib.hero_create.restype = C.c_int
    lib.hero_destroy.argtypes = [vp]
    lib.hero_last_error.argtypes = [vp]
    lib.hero_last_error.restype = C.c_char_p
    lib.hero_set_queries.argtypes = [vp, vp, vp, vp, C.c_uint64]
    lib.hero_build_index.argtypes = [vp]
    lib.hero_align_subjects.argtypes = [vp, vp, vp, vp, C.c_uint64]
    lib.hero_align_self.argtypes = [vp]
    lib.hero_reset_votes.argtypes = [vp]
    lib.hero_round.argtypes = [vp, C.c_uint32]
    lib.hero_fetch.argtypes = [vp] * 8
    lib.hero_consensus.argtypes = [vp] * 8
    lib.hero_get_votes.argtypes = [vp, vp]
    lib.hero_alignments_size.argtypes = [vp, C.POINTER(C.c_uint64)]
    lib.hero_alignments_take.argtypes = [vp, vp, C.c_uint64]
    lib.hero_align_self_range.argtypes = [vp, C.c_uint64, C.c_uint64]
    lib.hero_merge_pairs.argtypes = [vp, vp, vp]
    lib.hero_get_overhang.argtypes = [vp, vp]
    lib.hero_mapping_histogram.argtypes = [vp, vp, C.c_uint64, C.POINTER(C.c_uint64)]
    lib.hero_set_vote_buffer.argtypes = [vp, vp, C.c_uint64]
    lib.hero_server_set_round_policy.argtypes = [vp, C.c_uint64, C.c_uint64]
    lib.hero_server_worker_stats.argtypes = [vp, C.c_int32, C.POINTER(HeroStats)]
    lib.hero_server_workers.restype = C.c_int32
    lib.hero_consensus_range.argtypes = [vp, C.c_uint64, C.c_uint64] + [vp] * 7
    lib.hero_votes_words.argtypes = [vp, C.POINTER(C.c_uint64)]
    lib.hero_votes_save.argtypes = [vp, vp]
    lib.hero_votes_load.argtypes = [vp, vp]
    lib.hero_get_stats.argtypes = [vp, C.POINTER(HeroStats)]
    lib.hero_align_segments.argtypes = ([vp, C.c_int, vp, vp, C.c_uint64, vp, vp, C.c_uint64,
                                         C.c_uint64] + [vp] * 12)
    lib.hero_set_query_jobs.argtypes = [vp, vp, C.c_uint64]
    lib.hero_set_dp_tuning.argtypes = [vp, C.POINTER(DpTuning), C.c_uint32]
    lib.hero_set_dp_tuning.restype = C.c_int
    lib.hero_server_set_dp_tuning.argtypes = [vp, C.POINTER(DpTuning), C.c_uint32]
    lib.hero_server_set_dp_tuning.restype = C.c_int
    lib.hero_server_create.argtypes = [C.POINTER(HeroParams), C.c_uint64, C.POINTER(vp)]
    lib.hero_server_destroy.argtypes = [vp]
    lib.hero_job_submit.argtypes = [vp, vp, vp, vp, C.c_uint64, C.POINTER(C.c_uint64)]
    lib.hero_job_poll.argtypes = [vp, C.c_uint64, C.POINTER(JobInfo)]
    lib.hero_job_wait.argtypes = [vp, C.c_uint64, C.c_int64, C.POINTER(JobInfo)]
    lib.hero_job_result.argtypes = [vp, C.c_uint64] + [vp] * 7
    lib.hero_job_error.argtypes = [vp, C.c_uint64]
    lib.hero_job_error.restype = C.c_char_p
    lib.hero_job_release.argtypes = [vp, C.c_uint64]
    lib.hero_server_get_stats.argtypes = [vp, C.POINTER(ServerStats)]
    lib.hero_job_bytes.argtypes = [C.c_uint64, C.c_uint64, C.c_int32]
    lib.hero_job_bytes.restype = C.c_uint64
    lib.hero_round_admit.argtypes = [vp, C.c_uint64, C.c_uint64]
    lib.hero_round_admit.restype = C.c_uint64
    for f in ("hero_set_queries", "hero_build_index", "hero_align_subjects", "hero_align_self",
              "hero_reset_votes", "hero_round", "hero_fetch",
              "hero_consensus", "hero_get_votes", "hero_get_stats", "hero_align_segments",
              "hero_set_query_jobs", "hero_server_create", "hero_job_submit", "hero_job_poll",
              "hero_job_wait", "hero_job_result", "hero_job_release", "hero_server_get_stats"):
        getattr(lib, f).restype = C.c_int
    if path is None:
        _lib = lib
    return lib


def _ptr(a: np.ndarray | None):
    return None if a is None else C.c_void_p(a.ctypes.data)


class HeroError(RuntimeError):
    pass


class Hero:
    """One device context: a query set, its k-mer table and its vote matrix.

    Mirrors the reference's driver sequence (main.cpp:36-104): queries are
    loaded, the table is built, subject reads are aligned in chunks, then the
    consensus is called.
    """

    def __init__(self, k: int = 39, min_overlap: int = 40, aligner: str = "global",
                 max_mismatch_rate: float = 1.0, max_indel_rate: float = 1.0,
                 consensus_threshold: float = 0.6, device: int = 0, subject_batch: int = 0,
                 device_memory_budget: int = 0, stream: int | None = None,
                 tuning: list[dict] | str | None = None, alignment_output: bool = False,
                 merge_pairs: bool = False, mapping: bool = False):
        """alignment_output=True: HERO without -c -- the .aln records of every
        subject (alignments()) instead of votes and a consensus.
        merge_pairs=True: --merge -- overhang votes, then merge_pairs() after
        the consensus."""
        self.lib = load_library()
        p = HeroParams()
        self.lib.hero_default_params(C.byref(p))
        p.k = k
        p.min_overlap = min_overlap
        p.aligner = ALIGNER_AFFINE if aligner in ("a", "affine") else ALIGNER_GLOBAL
        p.device = device
        p.max_mismatch_rate = max_mismatch_rate
        p.max_indel_rate = max_indel_rate
        p.consensus_threshold = consensus_threshold
        p.subject_batch = subject_batch
        p.device_memory_budget = device_memory_budget
        p.stream = stream
        p.flags = ((FLAG_ALIGNMENT_OUTPUT if alignment_output else 0) |
                   (FLAG_MERGE_PAIRS if merge_pairs else 0) |
                   (FLAG_MAPPING if mapping else 0))
        self.params = p
        h = C.c_void_p()
        rc = self.lib.hero_create(C.byref(p), C.byref(h))
        if rc != HERO_OK:
            raise HeroError(f"hero_create failed: {ERRORS.get(rc, rc)}")
        self.h = h
        self.nq = 0
        self.nqb = 0
        # DP kernel shapes: the given classes, a record file, or the default record
        self.set_tuning(load_tuning(tuning, aligner) if not isinstance(tuning, list) else tuning)

    def set_tuning(self, classes: list[dict]):
        """DP kernel shapes per class of batch ([] = the library's defaults)."""
        arr = (DpTuning * max(1, len(classes)))()
        for i, t in enumerate(classes):
            arr[i] = DpTuning(int(t["rows_max"]), int(t["warps_per_block"]),
                              int(t["pair_strips"]), int(t["chunk_strips"]),
                              int(t.get("regs_per_thread", 0)))
        self._check(self.lib.hero_set_dp_tuning(self.h, arr, len(classes)), "set_tuning")

    def _check(self, rc: int, what: str):
        if rc != HERO_OK:
            msg = self.lib.hero_last_error(self.h)
            raise HeroError(f"{what}: {ERRORS.get(rc, rc)}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.hero_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _arrays(seq, off, uid):
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.uint64)
        uid = np.ascontiguousarray(uid, dtype=np.int64)
        return seq, off, uid

    def set_queries(self, seq, off, uid):
        seq, off, uid = self._arrays(seq, off, uid)
        self._qkeep = (seq, off, uid)
        self.nq = len(off) - 1
        self.nqb = int(off[-1]) if self.nq else 0
        self._check(self.lib.hero_set_queries(self.h, _ptr(seq), _ptr(off), _ptr(uid), self.nq),
                    "set_queries")

    def set_query_jobs(self, job):
        """Tags each query read with its job so one round corrects several jobs."""
        job = np.ascontiguousarray(job, dtype=np.uint32)
        self._jobkeep = job
        self._check(self.lib.hero_set_query_jobs(self.h, _ptr(job), len(job)), "set_query_jobs")

    def reset_votes(self):
        self._check(self.lib.hero_reset_votes(self.h), "reset_votes")

    def set_queries_ptr(self, seq_ptr: int, off_ptr: int, uid_ptr: int, n: int, nbases: int):
        """Raw host pointers (e.g. pinned buffers); the caller keeps them alive."""
        self.nq, self.nqb = n, nbases
        self._check(self.lib.hero_set_queries(self.h, C.c_void_p(seq_ptr), C.c_void_p(off_ptr),
                                              C.c_void_p(uid_ptr), n), "set_queries")

    def consensus_ptr(self, seq=0, imin=0, imed=0, imax=0, mis=0, gc=0, good=0):
        """Consensus into raw host pointers; 0 leaves that output on the device."""
        v = [C.c_void_p(x) if x else None for x in (seq, imin, imed, imax, mis, gc, good)]
        self._check(self.lib.hero_consensus(self.h, *v), "consensus")

    def round(self, graph: bool = True):
        """One correction round over the resident reads (batched form: CUDA graph)."""
        self._check(self.lib.hero_round(self.h, 1 if graph else 0), "round")

    def fetch(self):
        n, nb = self.nq, self.nqb
        res = dict(seq=np.empty(nb, np.uint8), imin=np.empty(n, np.uint32),
                   imed=np.empty(n, np.uint32), imax=np.empty(n, np.uint32),
                   mismatch_rate=np.empty(n, np.float64), gc=np.empty(n, np.float64),
                   good=np.empty(n, np.uint8))
        self._check(self.lib.hero_fetch(
            self.h, _ptr(res["seq"]), _ptr(res["imin"]), _ptr(res["imed"]), _ptr(res["imax"]),
            _ptr(res["mismatch_rate"]), _ptr(res["gc"]), _ptr(res["good"])), "fetch")
        return res

    def fetch_ptr(self, seq=0, imin=0, imed=0, imax=0, mis=0, gc=0, good=0):
        v = [C.c_void_p(x) if x else None for x in (seq, imin, imed, imax, mis, gc, good)]
        self._check(self.lib.hero_fetch(self.h, *v), "fetch")

    def build_index(self):
        self._check(self.lib.hero_build_index(self.h), "build_index")

    def align_self(self):
        self._check(self.lib.hero_align_self(self.h), "align_self")

    def align_subjects(self, seq, off, uid):
        seq, off, uid = self._arrays(seq, off, uid)
        self._check(self.lib.hero_align_subjects(self.h, _ptr(seq), _ptr(off), _ptr(uid),
                                                 len(off) - 1), "align_subjects")

    def consensus(self, out=None):
        n, nb = self.nq, self.nqb
        res = dict(seq=np.empty(nb, np.uint8) if out is None else out,
                   imin=np.empty(n, np.uint32), imed=np.empty(n, np.uint32),
                   imax=np.empty(n, np.uint32), mismatch_rate=np.empty(n, np.float64),
                   gc=np.empty(n, np.float64), good=np.empty(n, np.uint8))
        self._check(self.lib.hero_consensus(
            self.h, _ptr(res["seq"]), _ptr(res["imin"]), _ptr(res["imed"]), _ptr(res["imax"]),
            _ptr(res["mismatch_rate"]), _ptr(res["gc"]), _ptr(res["good"])), "consensus")
        return res

    def align_self_range(self, first: int, count: int):
        """The query reads [first, first + count) as subjects (one shard of align_self)."""
        self._check(self.lib.hero_align_self_range(self.h, int(first), int(count)),
                    "align_self_range")

    def votes_words(self) -> int:
        """Size of the additive vote state in 32-bit words (5 per query base)."""
        n = C.c_uint64()
        self._check(self.lib.hero_votes_words(self.h, C.byref(n)), "votes_words")
        return n.value

    def set_vote_buffer(self, dev_ptr: int, nbytes: int):
        """Votes into caller-owned device memory from the next set_queries on
        (hero_set_vote_buffer); 0 returns to the context's own buffers."""
        self._check(self.lib.hero_set_vote_buffer(self.h, C.c_void_p(dev_ptr) if dev_ptr else None,
                                                  int(nbytes)), "set_vote_buffer")

    def consensus_range(self, first: int, count: int, nbases: int | None = None,
                        fetch: bool = True) -> dict | None:
        """The consensus of the query reads [first, first + count) (hero_consensus_range);
        nbases, the range's bases, is needed when the reads were set by pointer.
        fetch=False leaves the results on the device."""
        if not fetch:
            self._check(self.lib.hero_consensus_range(self.h, int(first), int(count), *([None] * 7)),
                        "consensus_range")
            return None
        if nbases is None:
            off = self._qkeep[1]
            nbases = int(off[first + count] - off[first])
        nb = int(nbases)
        res = dict(seq=np.empty(nb, np.uint8), imin=np.empty(count, np.uint32),
                   imed=np.empty(count, np.uint32), imax=np.empty(count, np.uint32),
                   mismatch_rate=np.empty(count, np.float64), gc=np.empty(count, np.float64),
                   good=np.empty(count, np.uint8))
        self._check(self.lib.hero_consensus_range(
            self.h, int(first), int(count), *[_ptr(res[k]) for k in (
                "seq", "imin", "imed", "imax", "mismatch_rate", "gc", "good")]), "consensus_range")
        return res

    def votes_save(self, dev_ptr: int):
        """Copies the vote state into a device buffer (e.g. a CUDA tensor's data_ptr())."""
        self._check(self.lib.hero_votes_save(self.h, C.c_void_p(dev_ptr)), "votes_save")

    def votes_load(self, dev_ptr: int):
        """Replaces the vote state from a device buffer (the shards' sum)."""
        self._check(self.lib.hero_votes_load(self.h, C.c_void_p(dev_ptr)), "votes_load")

    def merge_pairs(self) -> dict:
        """--merge after the consensus: merged_seq (read layout, pair p's merged read
        from its first base) and merged_len (per pair, 0 = not merged)."""
        res = dict(merged_seq=np.empty(max(1, self.nqb), np.uint8),
                   merged_len=np.empty(max(1, self.nq // 2), np.uint32))
        self._check(self.lib.hero_merge_pairs(self.h, _ptr(res["merged_seq"]),
                                              _ptr(res["merged_len"])), "merge_pairs")
        res["merged_seq"] = res["merged_seq"][:self.nqb]
        res["merged_len"] = res["merged_len"][:self.nq // 2]
        return res

    def mapping_histogram(self) -> np.ndarray:
        """--mapping: bases per vote-count sum (hero_mapping_histogram)."""
        n = C.c_uint64()
        self._check(self.lib.hero_mapping_histogram(self.h, None, 0, C.byref(n)), "mapping_histogram")
        out = np.zeros(n.value, np.uint64)
        if n.value:
            self._check(self.lib.hero_mapping_histogram(self.h, _ptr(out), n.value, C.byref(n)),
                        "mapping_histogram")
        return out

    @staticmethod
    def mapping_text(hist: np.ndarray) -> bytes:
        """The histogram file QueryDataset::getCoverageAndWriteResults writes
        (QueryDataset.cpp:589-596)."""
        lines = [b"COV\tFRE\n"] + [b"%d\t%d\n" % (i, int(v)) for i, v in enumerate(hist) if v]
        return b"".join(lines)

    def overhang(self):
        """--merge: the overhang votes, uint32 [reads * 20 * 4]."""
        out = np.empty(max(1, self.nq * 80), np.uint32)
        self._check(self.lib.hero_get_overhang(self.h, _ptr(out)), "overhang")
        return out[:self.nq * 80]

    def alignments(self) -> bytes:
        """The .aln text of every subject aligned since the last call (and drops it)."""
        n = C.c_uint64()
        self._check(self.lib.hero_alignments_size(self.h, C.byref(n)), "alignments")
        buf = np.empty(max(1, n.value), np.uint8)
        self._check(self.lib.hero_alignments_take(self.h, _ptr(buf), n.value), "alignments")
        return buf[:n.value].tobytes()

    def votes(self):
        cov = np.empty(self.nqb * 4, np.uint32)
        self._check(self.lib.hero_get_votes(self.h, _ptr(cov)), "votes")
        return cov

    def stats(self) -> dict:
        s = HeroStats()
        self._check(self.lib.hero_get_stats(self.h, C.byref(s)), "stats")
        return {f: getattr(s, f) for f, _ in s._fields_}

    def align_segments(self, affine, subj_seq, subj_off, query_seq, query_off, seg_subject,
                       seg_orient, seg_query, s0, s1, q0, q1, flags, band):
        subj_seq = np.ascontiguousarray(subj_seq, np.uint8)
        subj_off = np.ascontiguousarray(subj_off, np.uint64)
        query_seq = np.ascontiguousarray(query_seq, np.uint8)
        query_off = np.ascontiguousarray(query_off, np.uint64)
        a = [np.ascontiguousarray(x, t) for x, t in (
            (seg_subject, np.uint32), (seg_orient, np.uint8), (seg_query, np.uint32),
            (s0, np.int32), (s1, np.int32), (q0, np.int32), (q1, np.int32), (flags, np.uint8),
            (band, np.int64))]
        n = len(a[0])
        cap = (a[4] - a[3]).astype(np.uint64) + (a[6] - a[5]).astype(np.uint64)
        ops_off = np.zeros(n + 1, np.uint64)
        ops_off[1:] = np.cumsum(cap)
        ops = np.zeros(int(ops_off[-1]), np.uint8)
        nops = np.zeros(n, np.int32)
        self._check(self.lib.hero_align_segments(
            self.h, int(affine), _ptr(subj_seq), _ptr(subj_off), len(subj_off) - 1,
            _ptr(query_seq), _ptr(query_off), len(query_off) - 1, n, *[_ptr(x) for x in a],
            _ptr(ops_off), _ptr(ops), _ptr(nops)), "align_segments")
        return ops, ops_off, nops


def _params(k=39, min_overlap=40, aligner="global", max_mismatch_rate=1.0, max_indel_rate=1.0,
            consensus_threshold=0.6, device=0, subject_batch=0, device_memory_budget=0):
    lib = load_library()
    p = HeroParams()
    lib.hero_default_params(C.byref(p))
    p.k, p.min_overlap, p.device = k, min_overlap, device
    p.aligner = ALIGNER_AFFINE if aligner in ("a", "affine") else ALIGNER_GLOBAL
    p.max_mismatch_rate, p.max_indel_rate = max_mismatch_rate, max_indel_rate
    p.consensus_threshold = consensus_threshold
    p.subject_batch, p.device_memory_budget = subject_batch, device_memory_budget
    return p


class HeroServer:
    """Serving form: independent correction jobs, continuous batching (hero_server_*)."""

    def __init__(self, round_bytes: int = 0, tuning: list[dict] | str | None = None, **kw):
        self.lib = load_library()
        self.params = _params(**kw)
        h = C.c_void_p()
        rc = self.lib.hero_server_create(C.byref(self.params), int(round_bytes), C.byref(h))
        if rc != HERO_OK:
            raise HeroError(f"hero_server_create failed: {ERRORS.get(rc, rc)}")
        self.h = h
        self._sizes: dict[int, tuple[int, int]] = {}
        classes = (load_tuning(tuning, kw.get("aligner", "global")) if not isinstance(tuning, list)
                   else tuning)
        arr = (DpTuning * max(1, len(classes)))()
        for i, t in enumerate(classes):
            arr[i] = DpTuning(int(t["rows_max"]), int(t["warps_per_block"]),
                              int(t["pair_strips"]), int(t["chunk_strips"]),
                              int(t.get("regs_per_thread", 0)))
        rc = self.lib.hero_server_set_dp_tuning(self.h, arr, len(classes))
        if rc != HERO_OK:
            self.close()
            raise HeroError(f"hero_server_set_dp_tuning: {ERRORS.get(rc, rc)} (a class the library refuses)")

    ROUND_BASES_DEFAULT = 8_000_000
    OVERLAP_BASES_DEFAULT = 64_000_000

    def set_round_policy(self, round_bases_max: int = ROUND_BASES_DEFAULT,
                         overlap_bases_max: int = OVERLAP_BASES_DEFAULT):
        """Round policy (hero_server_set_round_policy): bases a round admits
        beyond its first job, and the size under which a round may run beside
        another (0: no limit for either)."""
        rc = self.lib.hero_server_set_round_policy(self.h, int(round_bases_max), int(overlap_bases_max))
        if rc != HERO_OK:
            raise HeroError(f"hero_server_set_round_policy: {ERRORS.get(rc, rc)}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.hero_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, seq, off, uid) -> int:
        seq, off, uid = Hero._arrays(seq, off, uid)
        jid = C.c_uint64()
        rc = self.lib.hero_job_submit(self.h, _ptr(seq), _ptr(off), _ptr(uid), len(off) - 1,
                                      C.byref(jid))
        if rc != HERO_OK:
            raise HeroError(f"hero_job_submit: {ERRORS.get(rc, rc)}")
        self._sizes[jid.value] = (len(off) - 1, int(off[-1]) if len(off) > 1 else 0)
        return jid.value

    @staticmethod
    def _info(i: JobInfo) -> dict:
        return {f: getattr(i, f) for f, _ in i._fields_ if f != "reserved"}

    def poll(self, jid: int) -> dict:
        i = JobInfo()
        rc = self.lib.hero_job_poll(self.h, jid, C.byref(i))
        if rc != HERO_OK:
            raise HeroError(f"hero_job_poll: {ERRORS.get(rc, rc)}")
        return self._info(i)

    def wait(self, jid: int, timeout_ms: int = -1) -> dict:
        i = JobInfo()
        rc = self.lib.hero_job_wait(self.h, jid, int(timeout_ms), C.byref(i))
        if rc != HERO_OK:
            raise HeroError(f"hero_job_wait: {ERRORS.get(rc, rc)}")
        return self._info(i)

    def result(self, jid: int) -> dict:
        n, nb = self._sizes[jid]
        res = dict(seq=np.empty(nb, np.uint8), imin=np.empty(n, np.uint32),
                   imed=np.empty(n, np.uint32), imax=np.empty(n, np.uint32),
                   mismatch_rate=np.empty(n, np.float64), gc=np.empty(n, np.float64),
                   good=np.empty(n, np.uint8))
        rc = self.lib.hero_job_result(self.h, jid, *[_ptr(res[k]) for k in (
            "seq", "imin", "imed", "imax", "mismatch_rate", "gc", "good")])
        if rc != HERO_OK:
            err = self.lib.hero_job_error(self.h, jid)
            raise HeroError(f"hero_job_result: {ERRORS.get(rc, rc)}: {err.decode() if err else ''}")
        return res

    def release(self, jid: int):
        self.lib.hero_job_release(self.h, jid)
        self._sizes.pop(jid, None)

    def stats(self) -> dict:
        s = ServerStats()
        self.lib.hero_server_get_stats(self.h, C.byref(s))
        return {f: getattr(s, f) for f, _ in s._fields_}

    def worker_stats(self) -> list[dict]:
        """Each worker context's statistics as of its last round."""
        out = []
        for w in range(self.lib.hero_server_workers()):
            s = HeroStats()
            self.lib.hero_server_worker_stats(self.h, w, C.byref(s))
            out.append({f: getattr(s, f) for f, _ in s._fields_})
        return out


def correct(reads, **kw):
    """Corrects a read set against itself (HERO run with -q X -s X); returns consensus arrays."""
    with Hero(**kw) as h:
        h.set_queries(reads.seq, reads.off, reads.names)
        h.build_index()
        h.align_self()
        res = h.consensus()
        res["stats"] = h.stats()
        return res


def align_output(reads, **kw) -> bytes:
    """The .aln file of HERO run without -c (-q X -s X): every read's records."""
    with Hero(alignment_output=True, **kw) as h:
        h.set_queries(reads.seq, reads.off, reads.names)
        h.build_index()
        h.align_self()
        return h.alignments()
