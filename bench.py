"""Benchmark: corrected bases/s of the HERO read-correction path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl hero|reference]

Headline workload (N=1): the plain workload -- a 1 Mbp iid genome, 100 bp
reads at 30x (300,000 reads, 30 Mbp), strand 50/50, 1 % iid substitutions, no
indels, seeded synthetic data; HERO run as `-q X -s X -c --covinfo
--singleReads` (global aligner, defaults k=39, l=40, m=i=100 %).  Both arms
run exactly this workload: `--impl reference` times the reference itself
(oracle/_ref/hero_ref, built from the reference sources) on the same FASTQ
with the same flags on all host cores, so the two lines share one `config`.

A step is one whole correction of the read set: k-mer table build, seeding,
chaining, banded DP, record selection, votes and consensus.
  value : device-resident reads (uploaded once), the batched form (the round
          replayed as one CUDA graph); CUDA events on the library's stream
          around each step, the L2 flushed (a 256 MB write) between steps.
  e2e   : the same through the C ABI with pinned host buffers: every step
          uploads the reads (H2D) and reads back corrected reads and
          statistics (D2H).
Multi-GPU (torchrun): one job split across the ranks by subject reads (every
rank aligns its range against the whole table; the vote states are summed in
one NCCL all-reduce) -- strong scaling, value = the job's bases / the slowest
rank's device time.  --replicas instead corrects one copy of the job per rank.

The default line also carries:
  roofline          the DP kernel against the measured integer peak of the
                    instruction forms it issues (peaks of each form listed)
  seeding_roofline  probes + hit sort against the measured HBM bandwidth
  cpu_baseline      the reference on the host cores, one run of the same workload
  affine_batched    the affine/indel workload (5 Mbp + 40 repeats, 150 bp at
                    50x, 1.67 M reads, `-a a`) with its own value, e2e,
                    roofline and plain form; the reference's full-run time on
                    it is the one recorded by tests/golden/make_golden.py
  served            a stream of independent jobs through a hero_server
                    (Poisson arrivals): p50/p99 job latency, aggregate
                    bases/s, served == alone
  file_e2e          the drop-in program, FASTQ file to .fasta/.info files
  alignment_output  the same reads without -c: the whole .aln text in host memory
  merge             -c --merge on paired reads (corrected and merged bases/s)

Other workloads (--workload): config2 (affine/indel alone), config3 (mixed
lengths 75-250 bp, 12.3 M reads), config5 (diploid, 20 M reads), config4 (the
serving stream alone: p50/p99 job latency).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM traffic (read + write) of one DP kernel launch per band cell, from one
# ncu capture of a whole k_dp_wave launch per aligner (dram__bytes_read.sum +
# dram__bytes_write.sum over that launch's reference cells).  The traffic is per
# segment (codes in, ops and summaries out), so it scales with the cells of a
# launch.  Captures of the tuned shapes (1-warp blocks, tagged 16-bit pairs):
# affine, 150 bp reads at 50x on a 100 kbp genome, rows staged by bulk copies:
# 1.4643 GB + 0.7123 GB over 23,186,600,877 cells; global, 100 bp reads at 30x
# on a 200 kbp genome, before row staging: 180.80 MB + 89.73 MB over
# 1,766,508,768 cells.
DP_DRAM_BYTES_PER_CELL = {"affine": (1.464261e9 + 0.712347e9) / 23_186_600_877,
                          "global": (180.799744e6 + 89.734656e6) / 1_766_508_768}

# the reference's wall time on the whole affine/indel workload (1,666,666 reads,
# -a a), 8 threads, recorded by tests/golden/make_golden.py --full config2_full
REF_CONFIG2_FULL_SECONDS_8T = 665.75

L2_FLUSH_BYTES = 256 << 20  # larger than the B200's 126 MB L2


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hero", choices=["hero", "reference"])
    ap.add_argument("--workload", default="config1",
                    choices=["config1", "config2", "config3", "config4", "config5"])
    ap.add_argument("--served-jobs", type=int, default=40,
                    help="jobs of the served block added to the default line (0: none)")
    ap.add_argument("--jobs-scale", type=float, default=0.0,
                    help="genome-size scale of the served jobs (default 1.0: the stream's sizes)")
    ap.add_argument("--genome-bp", type=int, default=0, help="override the genome size")
    ap.add_argument("--cpu-sample-bp", type=int, default=60000,
                    help="genome size of the bounded sample the reference runs on for "
                         "workloads other than config1 (config1 runs whole)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-affine-block", action="store_true",
                    help="skip the affine/indel block of the default line")
    ap.add_argument("--no-alignment-output", action="store_true",
                    help="skip the alignment-output (.aln) line")
    ap.add_argument("--no-merge", action="store_true", help="skip the --merge line")
    ap.add_argument("--replicas", action="store_true",
                    help="with several ranks: one copy of the job per rank (weak scaling) "
                         "instead of one job split by subject reads")
    ap.add_argument("--shard", action="store_true",
                    help="split one job by subject reads even at one rank")
    ap.add_argument("--profile", action="store_true",
                    help="run --warmup then --steps device-resident steps and exit (for ncu)")
    return ap.parse_args()


def make_workload(name: str, genome_bp: int = 0, seed: int | None = None):
    from hero_b200 import synth
    if name == "config1":
        rs = synth.config1(seed=seed or 1, genome_bp=genome_bp or 1_000_000)
        desc = (f"plain/global: {rs.meta['genome_bp']} bp iid genome, 100 bp reads at 30x "
                f"({rs.n} reads), 1% substitutions")
        return rs, dict(aligner="global"), ["-c", "--covinfo", "--singleReads"], desc
    aff = ["-c", "--covinfo", "--singleReads", "-a", "a"]
    if name == "config3":
        rs = synth.config3(seed=seed or 3, genome_bp=genome_bp or 20_000_000)
        desc = (f"mixed lengths: {rs.meta['genome_bp']} bp genome (GC 42 %), reads U{{75..250}} bp "
                f"at 100x ({rs.n} reads), subs 0.1->2%, indels 0.05%/base")
        return rs, dict(aligner="affine"), aff, desc
    if name == "config5":
        rs = synth.config5(seed=seed or 5, genome_bp=genome_bp or 100_000_000)
        desc = (f"diploid: two {rs.meta['genome_bp']} bp haplotypes (0.1 % SNPs, 0.01 % indels), "
                f"150 bp reads at 30x ({rs.n} reads), subs 0.1->2%, indels 0.05%/base")
        return rs, dict(aligner="affine"), aff, desc
    rs = synth.config2(seed=seed or 2, genome_bp=genome_bp or 5_000_000)
    desc = (f"affine/indel: {rs.meta['genome_bp']} bp genome + 40 repeat copies, 150 bp reads "
            f"at 50x ({rs.n} reads), subs 0.1->2%, indels 0.05%/base")
    return rs, dict(aligner="affine"), ["-c", "--covinfo", "--singleReads", "-a", "a"], desc


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference runs (the reference binary built from its sources)
# ---------------------------------------------------------------------------
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "hero_ref")


def run_reference_once(fq: str, flags: list[str], workdir: str, threads: int) -> float:
    out = os.path.join(workdir, "out")
    for ext in (".fasta", ".info"):  # the reference appends
        if os.path.exists(out + ext):
            os.remove(out + ext)
    t0 = time.perf_counter()
    subprocess.run([REF_BIN, "-q", fq, "-s", fq, "-t", str(threads), "-o", out] + flags,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, check=True)
    return time.perf_counter() - t0


def workload_config(rs, flags: list[str], desc: str) -> dict:
    """The `config` object of a line: the same for the GPU arm and the reference
    arm when both run the same workload."""
    return {"workload": desc, "reads": rs.n, "bases": rs.total_bases, "flags": " ".join(flags),
            "l2": "L2 flushed between timed steps (256 MB write); the step's vote state "
                  f"({20 * rs.total_bases / 1e9:.2f} GB) and table exceed L2"}


def reference_workload(args):
    """What the reference runs: the whole workload for config1 (about ten seconds
    on the host cores), else a bounded sample of the same generator (smaller
    genome, same coverage, read lengths and errors)."""
    if args.workload == "config1":
        rs, _, flags, desc = make_workload("config1", args.genome_bp)
        return rs, flags, desc, True
    rs, _, flags, desc = make_workload(args.workload, args.cpu_sample_bp)
    return rs, flags, desc, False


CLI_BIN = os.path.join(ROOT, "hero_b200", "bin", "hero_b200")


def measure_file_e2e(rs, flags: list[str]) -> dict | None:
    """The drop-in program file to file: FASTQ in, .fasta and .info out, with the
    reference's flags (parsing, upload, correction, download and writing)."""
    if not os.path.exists(CLI_BIN):
        return None
    with tempfile.TemporaryDirectory() as d:
        fq = os.path.join(d, "in.fq")
        rs.write_fastq(fq)
        out = os.path.join(d, "out")
        t0 = time.perf_counter()
        r = subprocess.run([CLI_BIN, "-q", fq, "-s", fq, "-o", out] + flags,
                           stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        wall = time.perf_counter() - t0
    if r.returncode != 0:
        return {"error": r.stdout[-300:]}
    return {"seconds": wall, "bases_per_s": rs.total_bases / wall,
            "command": "hero_b200/bin/hero_b200 -q in.fq -s in.fq -o out " + " ".join(flags),
            "includes": "process start, FASTQ parse, device setup, correction, .fasta/.info writing"}


def measure_cpu_baseline(args) -> dict:
    if not os.path.exists(REF_BIN):
        return {"value": None, "unit": "bases/s", "cores": 0, "kind": "reference",
                "sample": "reference binary not built"}
    rs, flags, desc, whole = reference_workload(args)
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        fq = os.path.join(d, "in.fq")
        rs.write_fastq(fq)
        wall = run_reference_once(fq, flags, d, threads)
    what = "the whole workload" if whole else "a bounded sample"
    return {"value": rs.total_bases / wall, "unit": "bases/s", "cores": threads,
            "kind": "reference",
            "sample": f"{what}: {desc}; one run, {rs.total_bases} bases, {wall:.2f} s wall "
                      f"(reads parsed from FASTQ, outputs written)"}


def bench_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/hero_ref not built"}))
        return
    rs, flags, desc, whole = reference_workload(args)
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        fq = os.path.join(d, "in.fq")
        rs.write_fastq(fq)
        for _ in range(args.warmup):
            run_reference_once(fq, flags, d, threads)
        walls = [run_reference_once(fq, flags, d, threads) for _ in range(args.steps)]
    total = sum(walls)
    value = rs.total_bases * len(walls) / total
    what = "the whole workload" if whole else "a bounded sample of the workload"
    sample = (f"{what}: {desc}; each step one whole reference run on {threads} host threads "
              f"({rs.total_bases} bases, FASTQ in, .fasta/.info out)")
    line = {
        "impl": "reference", "metric": "corrected bases/s", "value": value, "unit": "bases/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(walls), "higher_is_better": True,
        "scaling": "strong" if args.gpus > 1 else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, no public dataset)",
        "config": workload_config(rs, flags, desc),
        "cpu_baseline": {"value": value, "unit": "bases/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "bases/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "step_seconds": [round(w, 3) for w in walls],
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU path
# ---------------------------------------------------------------------------
def hbm_peak_gbs() -> tuple[float, str]:
    """Measured HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), else
    the recorded fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


PEAK_FORMS = {"add_max_c": 0, "viaddmax_s32": 1, "vimax3_s32": 2, "viaddmax_s16x2": 3,
              "vimax3_s16x2": 4}


def int_peaks(device: int) -> dict:
    """Measured integer peaks (tera-ops/s, every lane's adds and maxes counted) of
    each instruction form the DP kernels issue (hero_b200/csrc/int_peak.cu)."""
    import ctypes as C
    from hero_b200 import build
    lib = C.CDLL(build.build_peak())
    lib.hero_form_peak_tops.restype = C.c_double
    lib.hero_form_peak_tops.argtypes = [C.c_int, C.c_int, C.c_int]
    out = {}
    for name, form in PEAK_FORMS.items():
        v = lib.hero_form_peak_tops(device, form, 5)
        out[name] = v if v > 0 else None
    return out


def dp_roofline(cells: int, dp_ms: float, aligner: str, peaks: dict, launches: int,
                pair_share: float = 0.0) -> dict:
    """The DP kernel's roofline: cells x ops a cell (6 global, 10 affine)
    over its device time, against the largest measured peak of the instruction
    forms it issues: the packed 16-bit DPX forms (2 lanes each) when most of its
    cells ran as 16-bit pairs (pair_share > 0.5), else the 32-bit forms."""
    ops_per_cell = 10 if aligner == "affine" else 6
    achieved = cells * ops_per_cell / (dp_ms / 1e3) / 1e12 if dp_ms > 0 else None
    pairs = pair_share > 0.5
    forms = (["viaddmax_s16x2", "vimax3_s16x2"] if pairs else
             ["add_max_c", "viaddmax_s32", "vimax3_s32"])
    vals = [(peaks.get(f), f) for f in forms if peaks.get(f)]
    peak, form = max(vals) if vals else (None, None)
    per_cell = DP_DRAM_BYTES_PER_CELL.get(aligner)
    traffic = per_cell * cells / launches if (per_cell is not None and launches) else None
    return {"bound": "alu", "kernel": f"k_dp_wave ({aligner} banded DP + traceback)",
            "achieved": achieved, "peak": peak, "unit": "Tops/s",
            "frac": (achieved / peak) if (achieved and peak) else None,
            "traffic": traffic, "ops_per_cell": ops_per_cell,
            "peak_source": f"measured in this run: the fastest of the kernel's instruction "
                           f"forms ({form}); MEASURED_PEAKS.json has no integer peak",
            "cells_as_16bit_pairs": round(pair_share, 4),
            "peaks_tops": peaks}


def flush_l2(stream, buf):
    """Writes a buffer larger than L2 on the stream (outside the timed events)."""
    import torch
    with torch.cuda.stream(stream):
        buf.fill_(1)


def _job_reads(job):
    rs = job.reads()
    return job.job_id, rs.seq, rs.off, rs.names


def job_stream(jobs, procs: int = 0):
    """The jobs' reads in job order, each generated from its seed in a spawn
    pool ahead of its use (no process is forked after CUDA starts)."""
    import multiprocessing as mp
    procs = procs or min(16, os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(procs) as pool:
        for jid, seq, off, names in pool.imap(_job_reads, jobs, chunksize=1):
            yield jid, (seq, off, names)


def _digest(res: dict) -> str:
    """md5 of a job's corrected reads, statistics and the doubles' bits."""
    import hashlib
    h = hashlib.md5()
    for f in ("seq", "imin", "imed", "imax", "good", "mismatch_rate", "gc"):
        h.update(np.ascontiguousarray(res[f]).tobytes())
    return h.hexdigest()


def run_alone(stream, h) -> tuple[dict, dict, float, int]:
    """Every job corrected on its own, one after another, through one context
    (host reads in, results in host memory out): wall time and digest per job."""
    times, digests, bases = {}, {}, 0
    for jid, (seq, off, names) in stream:
        t0 = time.perf_counter()
        h.set_queries(seq, off, names)
        h.build_index()
        h.align_self()
        res = h.consensus()
        times[jid] = time.perf_counter() - t0
        digests[jid] = _digest(res)
        bases += int(off[-1])
    return times, digests, sum(times.values()), bases


def warm_server(srv, item):
    """Both workers' contexts sized for the given job (one copy each, submitted
    together), as a server that has run for a while is."""
    _, (seq, off, names) = item
    ids = [srv.submit(seq, off, names) for _ in range(2)]
    for i in ids:
        srv.wait(i)
        srv.release(i)


def run_server(srv, stream, arrivals=None) -> dict:
    """Submits the jobs to a server -- all at once (arrivals None) or at the
    given arrival times (s) -- and reports per-job latency (submit -> results
    ready), aggregate throughput, the server's busy fraction and the digests."""
    import threading
    ids = {}
    late = []

    def submitter():
        start = time.perf_counter()
        for jid, (seq, off, names) in stream:
            if arrivals is not None:
                dt = arrivals[jid] - (time.perf_counter() - start)
                if dt > 0:
                    time.sleep(dt)
                else:
                    late.append(-dt)
            ids[jid] = srv.submit(seq, off, names)

    s0 = srv.stats()
    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    infos = {jid: srv.wait(i) for jid, i in ids.items()}
    s1 = srv.stats()
    digests = {jid: _digest(srv.result(i)) for jid, i in ids.items()}
    for i in ids.values():
        srv.release(i)
    lat = np.array([i["done_ms"] - i["submit_ms"] for i in infos.values()])
    first = min(i["submit_ms"] for i in infos.values())
    last = max(i["done_ms"] for i in infos.values())
    bases = sum(i["bases"] for i in infos.values())
    rounds = s1["rounds"] - s0["rounds"]
    return {"jobs": len(infos), "bases": bases,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "bases_per_s": bases / ((last - first) / 1e3),
            "busy_frac": (s1["busy_ms"] - s0["busy_ms"]) / (last - first),
            "rounds": rounds, "mean_jobs_per_round": len(infos) / max(rounds, 1),
            "overlapped_rounds": s1["overlapped_rounds"] - s0["overlapped_rounds"],
            "overlapped_device_phases": s1["overlapped_compute"] - s0["overlapped_compute"],
            "worker_ms": {k: round(s1[k] - s0[k], 1) for k in
                          ("ms_stage_in", "ms_round_calls", "ms_stage_out", "ms_alloc")},
            "buffer_allocs": s1["buffer_allocs"] - s0["buffer_allocs"],
            "arrivals_late_s": float(max(late)) if late else 0.0, "_digests": digests}


def serve_workload(jobs, dev: int, in_memory: bool, load: float = 0.95) -> dict:
    """The serving stream: each job alone (one at a time, one context), the
    server with every job submitted at once (its capacity), then the same
    server under Poisson arrivals at `load` of the better of the two rates (so
    the load is a true fraction of what the device sustains).  Both arms are
    warm: the context and both server workers first run the stream's largest
    job, so device buffers are sized as in a long-running service (buffer
    growth is a one-time cost either arm would pay).  served == alone compares
    every job's digest."""
    from hero_b200 import Hero, HeroServer
    if in_memory:
        data = dict(job_stream(jobs))

        def stream():
            return iter([(j.job_id, data[j.job_id]) for j in jobs])
    else:
        def stream():
            return job_stream(jobs)
    big = max(jobs, key=lambda j: j.genome_bp * j.coverage)
    warm = (list(job_stream([big], procs=1)) if not in_memory else [(big.job_id, data[big.job_id])])
    with Hero(aligner="affine", device=dev) as h:
        run_alone(iter(warm), h)
        times, alone_dig, alone_s, bases = run_alone(stream(), h)
    with HeroServer(aligner="affine", device=dev) as srv:
        warm_server(srv, warm[0])
        closed = run_server(srv, stream())
        mean_bases = bases / len(jobs)
        lam = load * max(closed["bases_per_s"], bases / alone_s) / mean_bases  # jobs/s
        # the stream's Poisson arrival times (config4_jobs draws them at 1 job/s), rescaled
        arrivals = {j.job_id: j.arrival_s / lam for j in jobs}
        poisson = run_server(srv, stream(), arrivals)
    same = sum(int(poisson["_digests"][j] == alone_dig[j] and closed["_digests"][j] == alone_dig[j])
               for j in alone_dig)
    for r in (closed, poisson):
        del r["_digests"]
    return {
        "jobs": len(jobs), "bases": bases,
        "p50_ms": poisson["p50_ms"], "p99_ms": poisson["p99_ms"], "mean_ms": poisson["mean_ms"],
        "max_ms": poisson["max_ms"], "bases_per_s": poisson["bases_per_s"],
        "arrival_rate_per_s": lam, "load_of_capacity": load,
        "busy_frac": poisson["busy_frac"], "rounds": poisson["rounds"],
        "mean_jobs_per_round": poisson["mean_jobs_per_round"],
        "overlapped_rounds": poisson["overlapped_rounds"],
        "overlapped_device_phases": poisson["overlapped_device_phases"],
        "arrivals_late_s": poisson["arrivals_late_s"],
        "capacity_bases_per_s": closed["bases_per_s"],
        "capacity_mean_jobs_per_round": closed["mean_jobs_per_round"],
        "capacity_worker_ms": closed["worker_ms"],
        "one_at_a_time_bases_per_s": bases / alone_s,
        "capacity_vs_one_at_a_time": closed["bases_per_s"] / (bases / alone_s),
        "alone_p50_ms": float(np.percentile([1e3 * t for t in times.values()], 50)),
        "served_equals_alone": f"{same}/{len(alone_dig)}",
        "warm": "context and both workers first ran the stream's largest job",
    }


def run_served_block(args, dev: int, n_jobs: int = 0, scale: float = 0.0) -> dict:
    """A served block of the default line: the first jobs of the serving stream
    (genome log-uniform 0.5-20 Mbp times `scale`, L in {100,150,250}, coverage
    U(20,80), affine errors), held in host memory."""
    from hero_b200 import synth
    n_jobs = n_jobs or args.served_jobs
    scale = scale or args.jobs_scale or 1.0
    jobs = synth.config4_jobs(n_jobs=n_jobs, scale=scale)
    with ClockSampler(dev) as sclk:
        served = serve_workload(jobs, dev, in_memory=True)
    served["clocks"] = sclk.summary()
    served["workload"] = (f"the first {n_jobs} jobs of the serving stream: Poisson arrivals, "
                          f"genome log-uniform 0.5-20 Mbp x {scale}, L in {{100,150,250}}, "
                          "coverage U(20,80), affine/indel errors")
    return served


def bench_served(args):
    """The serving workload alone: 200 jobs generated lazily from their seeds;
    one JSON line with p50/p99 job latency."""
    import torch

    from hero_b200 import build, synth
    if not os.environ.get("HERO_B200_LIB"):
        build.build_library()
    scale = args.jobs_scale or 1.0
    jobs = synth.config4_jobs(200, scale=scale)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    with ClockSampler(dev) as clk:
        r = serve_workload(jobs, dev, in_memory=False)
    line = {"metric": "p50/p99 job latency", "value": r["p50_ms"], "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "p99_ms": r["p99_ms"],
            "served_bases_per_s": r["bases_per_s"], "dtype": "int32",
            "data": "synthetic (seeded generator, no public dataset)",
            "config": {"workload": f"serving stream: 200 jobs, Poisson arrivals, genome "
                                   f"log-uniform 0.5-20 Mbp x {scale}, L in {{100,150,250}}, "
                                   f"coverage U(20,80), affine/indel errors",
                       "flags": "-c --covinfo --singleReads -a a"},
            "served": r, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def measure_workload(rs, kw, dev: int, steps: int, warmup: int, peaks: dict,
                     world: int = 1, barrier=None, max_over_ranks=None, clocks: bool = True):
    """One workload through Hero: the batched form with device-resident reads
    (value), the same through pinned host buffers (e2e), the plain form, the DP
    roofline and the seeding roofline."""
    import torch

    from hero_b200 import Hero
    n, nb = rs.n, rs.total_bases
    barrier = barrier or (lambda: None)
    max_over_ranks = max_over_ranks or (lambda x: x)
    seq_p = torch.from_numpy(rs.seq).pin_memory()
    off_p = torch.from_numpy(rs.off.view(np.int64)).pin_memory()
    uid_p = torch.from_numpy(rs.names.astype(np.int64)).pin_memory()
    out_seq = torch.empty(nb, dtype=torch.uint8).pin_memory()
    out_u32 = [torch.empty(n, dtype=torch.int32).pin_memory() for _ in range(3)]
    out_f64 = [torch.empty(n, dtype=torch.float64).pin_memory() for _ in range(2)]
    h2d = nb + 8 * (n + 1) + 8 * n
    d2h = nb + 3 * 4 * n + 2 * 8 * n
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=torch.device("cuda", dev))
    h = Hero(device=dev, stream=stream.cuda_stream, **kw)

    def e2e_step():
        # host buffers in, corrected reads and statistics out, every step
        h.set_queries_ptr(seq_p.data_ptr(), off_p.data_ptr(), uid_p.data_ptr(), n, nb)
        h.round(graph=True)
        h.fetch_ptr(out_seq.data_ptr(), out_u32[0].data_ptr(), out_u32[1].data_ptr(),
                    out_u32[2].data_ptr(), out_f64[0].data_ptr(), out_f64[1].data_ptr())

    def device_step(graph=True):
        h.round(graph=graph)

    # warm-up: the first round runs eagerly (plain form) and is captured as a
    # graph; later rounds replay it (the batched form)
    for _ in range(warmup):
        e2e_step()
    torch.cuda.synchronize()

    def timed(fn, k):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k)]
        barrier()
        torch.cuda.synchronize()
        for a, b in ev:
            flush_l2(stream, flush)
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / 1e3)

    s0 = h.stats()
    if clocks:
        with ClockSampler(dev) as clk:
            t_dev = timed(device_step, steps)
        clock_summary = clk.summary()
    else:
        t_dev = timed(device_step, steps)
        clock_summary = None
    s1 = h.stats()
    t_e2e = timed(e2e_step, steps)
    p0 = h.stats()
    plain_steps = max(1, min(steps, 2))
    t_plain = timed(lambda: device_step(graph=False), plain_steps)
    p1 = h.stats()
    h.close()

    launches = s1["kernel_launches"] - s0["kernel_launches"]
    if launches == 0:  # graph replays launch kernels without host calls: count one plain round
        launches = (p1["kernel_launches"] - p0["kernel_launches"]) // plain_steps * steps
    cells = s1["dp_cells"] - s0["dp_cells"]
    dp_ms = s1["ms_dp_kernel"] - s0["ms_dp_kernel"]
    computed = s1["dp_cells_computed"] - s0["dp_cells_computed"]
    pair_share = (s1["dp_cells_pairs"] - s0["dp_cells_pairs"]) / computed if computed else 0.0
    per = {k: round((p1[k] - p0[k]) / plain_steps, 3)
           for k in ("ms_index", "ms_seed", "ms_chain", "ms_dp", "ms_dp_kernel", "ms_record",
                     "ms_vote", "ms_consensus", "ms_align_wall")}
    dp_launches = steps * ((n + 131071) // 131072)  # one DP launch per subject batch
    # seeding against HBM: per probe one 24-byte key+value slot read, per hit the
    # hit value (8 B) read and the hit tuple (16 B) written, the subject reads at
    # 2 bits a base (algorithmic bytes of the probe phase)
    probes = (p1["probes"] - p0["probes"]) / plain_steps
    hits = (p1["hits"] - p0["hits"]) / plain_steps
    seed_bytes = 24 * probes + 24 * hits + nb / 4
    seed_ms = per["ms_seed"]
    hbm_peak, hbm_src = hbm_peak_gbs()
    seed_gbs = seed_bytes / (seed_ms / 1e3) / 1e9 if seed_ms > 0 else None
    return {
        "value": world * nb * steps / t_dev, "ms_per_step": 1e3 * t_dev / steps,
        "e2e": {"value": world * nb * steps / t_e2e, "unit": "bases/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": dp_roofline(cells, dp_ms, kw["aligner"], peaks, dp_launches, pair_share),
        "seeding_roofline": {"bound": "hbm", "kernels": "k_probe (count, emit) + k_sort_hits",
                             "achieved": seed_gbs, "peak": hbm_peak, "unit": "GB/s",
                             "frac": (seed_gbs / hbm_peak) if seed_gbs else None,
                             "algorithmic_bytes_per_step": seed_bytes, "peak_source": hbm_src},
        "gcups": cells / (dp_ms / 1e3) / 1e9 if dp_ms > 0 else None,
        "form": "batched (whole round replayed as one CUDA graph)",
        "plain_form": {"value": world * nb * plain_steps / t_plain,
                       "ms_per_step": 1e3 * t_plain / plain_steps, "stage_ms_per_step": per},
        "clocks": clock_summary, "gpu_launches": launches,
        "work_per_step": {"dp_cells": cells // steps,
                          "dp_segments": (s1["dp_segments"] - s0["dp_segments"]) // steps,
                          "probes": int(probes), "hits": int(hits)},
    }


def bench_hero(args):
    import torch
    import torch.distributed as dist

    from hero_b200 import build, shard
    if not os.environ.get("HERO_B200_LIB"):
        build.build_library()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900),
                                device_id=torch.device("cuda", dev))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return shard.max_over_ranks(x, device="cuda")

    rs, kw, flags, desc = make_workload(args.workload, args.genome_bp)
    log(f"[rank {rank}] workload: {desc}")
    if args.profile:
        from hero_b200 import Hero
        with Hero(device=dev, **kw) as h:
            h.set_queries(rs.seq, rs.off, rs.names)
            for _ in range(args.warmup + args.steps):
                h.round(graph=False)
            torch.cuda.synchronize()
            log(json.dumps({"rounds": args.warmup + args.steps, "stats": h.stats()}))
        return

    peaks = int_peaks(dev)
    main = measure_workload(rs, kw, dev, args.steps, args.warmup, peaks, world, barrier,
                            max_over_ranks)
    solo = rank == 0 and world == 1
    affine = None
    if solo and args.workload == "config1" and not args.no_affine_block:
        rs2, kw2, flags2, desc2 = make_workload("config2")
        affine = measure_workload(rs2, kw2, dev, args.steps, args.warmup, peaks)
        affine["config"] = workload_config(rs2, flags2, desc2)
        affine["reference_full_run"] = {
            "seconds": REF_CONFIG2_FULL_SECONDS_8T, "threads": 8,
            "bases_per_s": rs2.total_bases / REF_CONFIG2_FULL_SECONDS_8T,
            "note": "the reference on this whole workload, timed once on the 8 cores of the "
                    "build host by tests/golden/make_golden.py (not timed in this run)"}
        del rs2
    served_form = None
    if solo and args.workload in ("config3", "config5"):
        # the same job through a hero_server (host reads in, results in host
        # memory out), against the plain and batched forms of the main line
        from hero_b200 import HeroServer
        with HeroServer(aligner=kw["aligner"], device=dev) as srv:
            walls = []
            for _ in range(2):
                t0 = time.perf_counter()
                jid = srv.submit(rs.seq, rs.off, rs.names)
                srv.wait(jid)
                srv.result(jid)
                walls.append(time.perf_counter() - t0)
                srv.release(jid)
        sv = rs.total_bases / walls[-1]
        served_form = {"value": sv, "unit": "bases/s", "seconds": walls[-1],
                       "batched_vs_plain": main["value"] / main["plain_form"]["value"],
                       "served_vs_plain": sv / main["plain_form"]["value"],
                       "note": "one job submitted to a hero_server, submit to results in host "
                               "memory (second of two runs)"}
    served = served_small = None
    if solo and args.served_jobs and args.workload == "config1":
        served = run_served_block(args, dev)
        # small jobs (genome sizes x 0.02): where sharing rounds pays, since a
        # round's fixed cost outweighs a small job's alignment work
        served_small = run_served_block(args, dev, n_jobs=100, scale=0.02)
    aln = merge = cpu = file_e2e = None
    small = args.workload in ("config1", "config2")  # the .aln text of a large job is tens of GB
    if solo and not args.no_alignment_output and small:
        aln = measure_alignment_output(rs, kw, dev)
    if solo and not args.no_merge and small:
        merge = measure_merge(dev)
    if solo and not args.no_cpu_baseline:
        cpu = measure_cpu_baseline(args)
    if solo:
        file_e2e = measure_file_e2e(rs, flags)

    if rank == 0:
        line = {
            "metric": "corrected bases/s", "value": main["value"], "unit": "bases/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": main["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator, no public dataset)",
            "config": workload_config(rs, flags, desc),
            "parallelism": f"one copy of the job per rank x{world}",
            "e2e": main["e2e"],
            "roofline": main["roofline"],
            "seeding_roofline": main["seeding_roofline"],
            "gcups": main["gcups"], "form": main["form"], "plain_form": main["plain_form"],
            "cpu_baseline": cpu, "file_e2e": file_e2e, "clocks": main["clocks"],
            "gpu_launches": main["gpu_launches"], "work_per_step": main["work_per_step"],
            "affine_batched": affine, "served_form": served_form, "served": served,
            "served_small_jobs": served_small,
            "alignment_output": aln,
            "merge": merge,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def measure_alignment_output(rs, kw, dev):
    """The alignment-output mode (HERO without -c) on the same reads: host reads
    in, the whole .aln text in host memory out; wall time of the second of two
    runs (table, seeding, chaining, DP, record lists, text, copy out)."""
    from hero_b200 import Hero
    walls, size = [], 0
    with Hero(alignment_output=True, device=dev, **kw) as h:
        for _ in range(2):
            t0 = time.perf_counter()
            h.set_queries(rs.seq, rs.off, rs.names)
            h.build_index()
            h.align_self()
            text = h.alignments()
            walls.append(time.perf_counter() - t0)
            size = len(text)
            del text
        st = h.stats()
    return {"metric": "aligned bases/s (.aln text in host memory)",
            "value": rs.total_bases / walls[-1], "unit": "bases/s", "seconds": walls[-1],
            "aln_bytes": size, "records": st["records_kept"] // 2,
            "flags": "as the main line without -c"}


def bench_sharded(args):
    """One correction split across the ranks by subject reads (hero_b200.shard):
    every rank holds the whole query set and table, aligns its range of subject
    reads into a vote buffer of its own, each owner's slice of the votes is
    reduced to it in place (one NCCL reduce a slice, over NVLink), and every
    rank calls the consensus of the query reads it owns.  Strong scaling: value
    = the job's bases over the slowest rank's device time of a step."""
    import torch
    import torch.distributed as dist

    from hero_b200 import Hero, build, shard
    if not os.environ.get("HERO_B200_LIB"):
        build.build_library()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900),
                                device_id=torch.device("cuda", dev))
    rs, kw, flags, desc = make_workload(args.workload, args.genome_bp)
    n, nb = rs.n, rs.total_bases
    a, b = shard.shard_range(n, rank, world)
    seq_p = torch.from_numpy(rs.seq).pin_memory()
    off_p = torch.from_numpy(rs.off.view(np.int64)).pin_memory()
    uid_p = torch.from_numpy(rs.names.astype(np.int64)).pin_memory()
    out_seq = torch.empty(nb, dtype=torch.uint8).pin_memory()
    out_u32 = [torch.empty(n, dtype=torch.int32).pin_memory() for _ in range(3)]
    out_f64 = [torch.empty(n, dtype=torch.float64).pin_memory() for _ in range(2)]
    stream = torch.cuda.Stream(device=dev)
    h = Hero(device=dev, stream=stream.cuda_stream, **kw)
    # the vote state in a buffer of ours, reduced in place to the owners of
    # query-read ranges; each rank calls the consensus of its own reads
    owners = shard.owner_slices(rs.off, world)
    first, count, own_bases, _ = owners[rank]
    state = torch.zeros(5 * nb + 64, dtype=torch.int32, device=torch.device("cuda", dev))
    h.set_vote_buffer(state.data_ptr(), state.numel() * 4)
    h.set_queries_ptr(seq_p.data_ptr(), off_p.data_ptr(), uid_p.data_ptr(), n, nb)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=torch.device("cuda", dev))

    def exchange():
        if world > 1:
            stream.synchronize()
            with torch.cuda.stream(stream):
                shard.reduce_votes_to_owners(state, owners)

    def device_step():
        h.reset_votes()
        h.build_index()
        h.align_self_range(a, b - a)
        exchange()
        h.consensus_range(first, count, own_bases, fetch=False)

    def e2e_step():
        h.set_queries_ptr(seq_p.data_ptr(), off_p.data_ptr(), uid_p.data_ptr(), n, nb)
        h.build_index()
        h.align_self_range(a, b - a)
        exchange()
        r = h.consensus_range(first, count, own_bases)
        out_seq[:own_bases].copy_(torch.from_numpy(r["seq"]))

    def timed(fn, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for e0, e1 in ev:
            flush_l2(stream, flush)
            e0.record(stream)
            fn()
            e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return shard.max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in ev) / 1e3, "cuda")

    for _ in range(args.warmup):
        device_step()
    s0 = h.stats()
    with ClockSampler(dev) as clk:
        t_dev = timed(device_step, args.steps)
    s1 = h.stats()
    t_e2e = timed(e2e_step, args.steps)
    cells = s1["dp_cells"] - s0["dp_cells"]
    dp_ms = s1["ms_dp_kernel"] - s0["ms_dp_kernel"]
    launches = s1["kernel_launches"] - s0["kernel_launches"]
    h.close()
    computed = s1["dp_cells_computed"] - s0["dp_cells_computed"]
    roof = dp_roofline(cells, dp_ms, kw["aligner"], int_peaks(dev),
                       args.steps * ((b - a + 131071) // 131072),
                       (s1["dp_cells_pairs"] - s0["dp_cells_pairs"]) / computed if computed else 0.0)
    roof["kernel"] += " (rank 0's DP launches)"
    if rank == 0:
        line = {
            "metric": "corrected bases/s", "value": nb * args.steps / t_dev, "unit": "bases/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator, no public dataset)",
            "config": workload_config(rs, flags, desc),
            "parallelism": f"one job, subject reads sharded x{world}, each owner's slice of "
                           "the votes reduced to it",
            "e2e": {"value": nb * args.steps / t_e2e, "unit": "bases/s",
                    "h2d_bytes_per_step": nb + 8 * (n + 1) + 8 * n,
                    "d2h_bytes_per_step": own_bases + 3 * 4 * count + 2 * 8 * count + count},
            "roofline": roof,
            "cpu_baseline": None,
            "exchange": "one NCCL reduce of each owner's slice of the vote state (20 B a "
                        "query base) to its owner, in place; each rank calls the consensus of "
                        "its own query reads",
            "exchange_bytes_per_rank": 20 * nb * (world - 1) // max(world, 1),
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def measure_merge(dev):
    """-c --merge on paired reads of the same size as the main workload (5 Mbp
    genome, fragments 160-290 bases read from both ends, 150 bp, 50x, 0.5 %
    substitutions): host reads in, corrected and merged reads out; wall time of
    the second of two runs (table, seeding, DP, votes with overhang votes,
    consensus, pair merge, copies)."""
    from hero_b200 import Hero, synth
    rs = synth.paired()
    walls = []
    with Hero(aligner="affine", device=dev, merge_pairs=True) as h:
        for _ in range(2):
            t0 = time.perf_counter()
            h.set_queries(rs.seq, rs.off, rs.names)
            h.build_index()
            h.align_self()
            h.consensus()
            mg = h.merge_pairs()
            walls.append(time.perf_counter() - t0)
    return {"metric": "corrected and merged bases/s (-c --merge, paired reads)",
            "value": rs.total_bases / walls[-1], "unit": "bases/s", "seconds": walls[-1],
            "reads": rs.n, "pairs_merged": int((mg["merged_len"] > 0).sum()),
            "workload": "5 Mbp genome, fragments U{160..290} read from both ends, 150 bp, "
                        "50x, 0.5 % substitutions, affine"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        bench_reference(args)
    elif args.workload == "config4":
        bench_served(args)
    elif args.shard or (world > 1 and not args.replicas):
        bench_sharded(args)
    else:
        bench_hero(args)


if __name__ == "__main__":
    main()
