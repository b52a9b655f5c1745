"""Serving form: admission logic (CPU) and job-alone == job-in-mix (GPU).

A server corrects independent jobs together: their reads share one query set
and one k-mer table, each key tagged with its job.  Every job's output must be
byte-identical to the output of the same job corrected alone."""
import ctypes as C

import numpy as np
import pytest

from hero_b200 import load_library, synth


def _admit(sizes, budget):
    lib = load_library()
    a = np.ascontiguousarray(sizes, np.uint64)
    return lib.hero_round_admit(C.c_void_p(a.ctypes.data) if len(a) else None, len(a), budget)


def test_admission_takes_the_longest_fitting_prefix():
    assert _admit([], 100) == 0
    assert _admit([10, 20, 30], 100) == 3
    assert _admit([10, 20, 30, 50], 60) == 3
    assert _admit([10, 20, 30, 50], 59) == 2
    assert _admit([70, 10], 60) == 1            # an oversized head job runs alone
    assert _admit([10, 70, 10], 60) == 1        # FIFO: no skipping ahead


def test_job_bytes_grow_with_the_job():
    lib = load_library()
    a = lib.hero_job_bytes(1_000_000, 10_000, 39)
    b = lib.hero_job_bytes(2_000_000, 20_000, 39)
    c = lib.hero_job_bytes(1_000_000, 10_000, 21)  # shorter keys: more of them
    assert 0 < a < b and c > a
    # votes alone are 20 bytes per base
    assert a > 20 * 1_000_000


def _jobs():
    """Small jobs of different lengths/coverages, plus a renamed twin of job 0
    (identical bases): without job tags its reads would meet job 0's."""
    js = [synth.Job(i, 0.0, 100 + i, g, L, cov).reads() for i, (g, L, cov) in
          enumerate([(30_000, 150, 40.0), (20_000, 100, 30.0), (25_000, 250, 25.0)])]
    twin = js[0]
    js.append(synth.ReadSet(twin.seq.copy(), twin.off.copy(), twin.names + 10_000_000,
                            twin.qual))
    return js


@pytest.mark.gpu
def test_jobs_in_a_shared_round_match_jobs_alone():
    from hero_b200 import HeroServer, correct
    jobs = _jobs()
    alone = [correct(rs, aligner="affine") for rs in jobs]
    with HeroServer(aligner="affine") as srv:
        ids = [srv.submit(rs.seq, rs.off, rs.names) for rs in jobs]
        infos = [srv.wait(j, 120_000) for j in ids]
        got = [srv.result(j) for j in ids]
        st = srv.stats()
    assert all(i["state"] == 2 for i in infos), infos
    assert st["jobs_done"] == len(jobs) and st["jobs_failed"] == 0
    assert max(i["round_jobs"] for i in infos) > 1, "no round held more than one job"
    for k, (a, b) in enumerate(zip(alone, got)):
        for f in ("seq", "imin", "imed", "imax", "good"):
            assert np.array_equal(a[f], b[f]), (k, f)
        for f in ("mismatch_rate", "gc"):
            assert np.array_equal(a[f].view(np.uint64), b[f].view(np.uint64)), (k, f)


@pytest.mark.gpu
def test_rounds_tagged_by_hand_match_rounds_alone():
    """hero_set_query_jobs on one context, two jobs concatenated."""
    from hero_b200 import Hero, correct
    jobs = _jobs()[:2]
    alone = [correct(rs, aligner="affine") for rs in jobs]
    seq = np.concatenate([j.seq for j in jobs])
    off = np.concatenate([jobs[0].off, jobs[1].off[1:] + jobs[0].off[-1]])
    uid = np.concatenate([j.names for j in jobs])
    tag = np.repeat(np.arange(2, dtype=np.uint32), [jobs[0].n, jobs[1].n])
    with Hero(aligner="affine") as h:
        h.set_queries(seq, off, uid)
        h.set_query_jobs(tag)
        h.build_index()
        h.align_self()
        res = h.consensus()
    n0, b0 = jobs[0].n, int(jobs[0].off[-1])
    assert np.array_equal(res["seq"][:b0], alone[0]["seq"])
    assert np.array_equal(res["seq"][b0:], alone[1]["seq"])
    assert np.array_equal(res["imed"][:n0], alone[0]["imed"])
    assert np.array_equal(res["imed"][n0:], alone[1]["imed"])


def _same(a, b, k):
    for f in ("seq", "imin", "imed", "imax", "good"):
        assert np.array_equal(a[f], b[f]), (k, f)
    for f in ("mismatch_rate", "gc"):
        assert np.array_equal(a[f].view(np.uint64), b[f].view(np.uint64)), (k, f)


@pytest.mark.gpu
def test_a_shared_round_outlives_the_release_of_its_other_jobs():
    """A round's results are one block its jobs share: releasing some jobs of
    the round leaves the others' slices intact."""
    from hero_b200 import HeroServer, correct
    jobs = _jobs()
    alone = [correct(rs, aligner="affine") for rs in jobs]
    with HeroServer(aligner="affine") as srv:
        srv.set_round_policy(0, 0)
        ids = [srv.submit(rs.seq, rs.off, rs.names) for rs in jobs]
        infos = [srv.wait(j, 120_000) for j in ids]
        assert max(i["round_jobs"] for i in infos) > 1
        for j in ids[::2]:
            srv.release(j)
        for k in range(1, len(jobs), 2):
            _same(alone[k], srv.result(ids[k]), k)


@pytest.mark.gpu
def test_round_policy_one_job_a_round_and_no_overlap():
    """round_bases_max=1 admits no job beside a round's first; overlap_bases_max=1
    starts no round's device phase while another's (of more than one base) runs."""
    from hero_b200 import HeroServer, correct
    jobs = _jobs()
    alone = [correct(rs, aligner="affine") for rs in jobs]
    with HeroServer(aligner="affine") as srv:
        srv.set_round_policy(1, 1)
        s0 = srv.stats()
        ids = [srv.submit(rs.seq, rs.off, rs.names) for rs in jobs]
        infos = [srv.wait(j, 120_000) for j in ids]
        got = [srv.result(j) for j in ids]
        s1 = srv.stats()
    assert all(i["round_jobs"] == 1 for i in infos)
    assert s1["rounds"] - s0["rounds"] == len(jobs)
    assert s1["overlapped_compute"] == s0["overlapped_compute"]
    for k, (a, b) in enumerate(zip(alone, got)):
        _same(a, b, k)


@pytest.mark.gpu
def test_wait_with_a_limit_times_out_and_later_completes():
    from hero_b200 import HeroError, HeroServer
    rs = synth.config2(seed=9, genome_bp=200_000)
    with HeroServer(aligner="affine") as srv:
        j = srv.submit(rs.seq, rs.off, rs.names)
        with pytest.raises(HeroError, match="TIMEOUT"):
            srv.wait(j, 0)
        info = srv.wait(j, 120_000)
        assert info["state"] == 2 and info["done_ms"] >= info["submit_ms"]
        assert info["bases"] == int(rs.off[-1]) and info["reads"] == rs.n


@pytest.mark.gpu
def test_new_contexts_start_from_zeroed_counters():
    """Device memory freed by an earlier owner is not zero: a new context's work
    counters (and its buffer-overflow flag) must not inherit what was there."""
    import torch

    from hero_b200 import Hero, correct
    x = torch.full((1 << 30,), 0xFF, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    del x
    torch.cuda.empty_cache()
    for _ in range(4):
        with Hero(aligner="affine") as h:
            s = h.stats()
        assert s["hits"] == 0 and s["dp_segments_ref"] == 0 and s["dp_cells"] == 0, s
    rs = synth.config2(seed=11, genome_bp=30_000)
    res = correct(rs, aligner="affine")
    assert res["stats"]["dp_cells"] > 0
