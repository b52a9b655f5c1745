"""Regenerates the golden manifest from the reference itself.

Runs the unmodified reference (oracle/_ref/hero_ref, built from the reference
sources by oracle/Makefile) on every fixture input and records md5 sums of the
input FASTQ, of the reference .fasta/.info (consensus mode, -c) and of its .aln
(alignment-output mode: the same flags without -c); the .fasta/.info of the
fixtures in STORED are kept gzipped.  The MERGE_FIXTURES (paired input) get
the md5 and size of the reference's _merged.fasta, _unmerged.fasta and .info
with -c --covinfo --merge; the MAPPING_FIXTURES the md5 of the coverage
histogram of -c --mapping.  Usage:  python tests/golden/make_golden.py

    python tests/golden/make_golden.py --full NAME...

regenerates the named entries of manifest_full.json (whole-size workloads and
reduced-genome instances of the larger ones; minutes each) and keeps the rest.

    python tests/golden/make_golden.py --config4-sample

runs the reference on the sampled jobs of the serving stream (synth.config4_jobs():
every job of at most 2 Mbp plus 5 larger ones drawn with a fixed seed; affine,
-c --covinfo --singleReads -a a) and records each job's .fasta/.info md5 in
manifest_config4.json, saving after every job (hours in all; a rerun skips the
jobs already recorded).
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from fixtures import FIXTURES, MAPPING_FIXTURES, MERGE_FIXTURES, STORED, aln_flags  # noqa: E402

from hero_b200 import synth  # noqa: E402

# name -> (generator call as recorded, generator, reference flags)
FULL = {
    "config1_full": ("synth.config1()", lambda: synth.config1(), []),
    "config2_full": ("synth.config2()", lambda: synth.config2(), ["-a", "a"]),
    "config3_full": ("synth.config3()", lambda: synth.config3(), ["-a", "a"]),
    "config3_reduced": ("synth.config3(genome_bp=200000)",
                        lambda: synth.config3(genome_bp=200_000), ["-a", "a"]),
    "config5_reduced": ("synth.config5(genome_bp=1000000)",
                        lambda: synth.config5(genome_bp=1_000_000), ["-a", "a"]),
}

REF = os.path.join(ROOT, "oracle", "_ref", "hero_ref")


def md5(b: bytes) -> str:
    return hashlib.md5(b).hexdigest()


def run_reference(fq: str, flags: list[str], workdir: str) -> tuple[bytes, bytes]:
    out = os.path.join(workdir, "out")
    for ext in (".fasta", ".info"):  # outputs are opened in append mode
        if os.path.exists(out + ext):
            os.remove(out + ext)
    subprocess.run([REF, "-q", fq, "-s", fq, "-c", "--covinfo", "--singleReads", "-t",
                    str(os.cpu_count() or 1), "-o", out] + flags,
                   stdout=subprocess.DEVNULL, check=True)
    with open(out + ".fasta", "rb") as f:
        fa = f.read()
    with open(out + ".info", "rb") as f:
        info = f.read()
    return fa, info


def run_reference_aln(fq: str, flags: list[str], workdir: str) -> bytes:
    """The .aln of the alignment-output mode (no -c; SubjectReadAligner::writeToFile)."""
    out = os.path.join(workdir, "aln")
    if os.path.exists(out + ".aln"):  # opened in append mode
        os.remove(out + ".aln")
    subprocess.run([REF, "-q", fq, "-s", fq, "--singleReads", "-t", str(os.cpu_count() or 1),
                    "-o", out] + aln_flags(flags), stdout=subprocess.DEVNULL, check=True)
    with open(out + ".aln", "rb") as f:
        return f.read()


def run_reference_merge(fq: str, flags: list[str], workdir: str) -> dict:
    """--merge (paired input): md5 and size of _merged.fasta, _unmerged.fasta, .info."""
    out = os.path.join(workdir, "merge")
    exts = ("_merged.fasta", "_unmerged.fasta", ".info")
    for e in exts:  # opened in append mode
        if os.path.exists(out + e):
            os.remove(out + e)
    subprocess.run([REF, "-q", fq, "-s", fq, "-c", "--covinfo", "--merge", "-t",
                    str(os.cpu_count() or 1), "-o", out] + flags,
                   stdout=subprocess.DEVNULL, check=True)
    res = {}
    for e in exts:
        with open(out + e, "rb") as f:
            b = f.read()
        key = e.strip("._").replace(".", "_")
        res[key + "_md5"] = md5(b)
        res[key + "_bytes"] = len(b)
    return res


def run_reference_mapping(fq: str, flags: list[str], workdir: str) -> bytes:
    """-c --mapping: the coverage histogram file (written to the output name as given)."""
    out = os.path.join(workdir, "mapping")
    if os.path.exists(out):  # opened in append mode
        os.remove(out)
    subprocess.run([REF, "-q", fq, "-s", fq, "-c", "--mapping", "--singleReads", "-t",
                    str(os.cpu_count() or 1), "-o", out] + aln_flags(flags),
                   stdout=subprocess.DEVNULL, check=True)
    with open(out, "rb") as f:
        return f.read()


def _host_ram_gb() -> float:
    with open("/proc/meminfo") as f:
        for line in f:
            if line.startswith("MemTotal:"):
                return round(int(line.split()[1]) / 2**20, 1)
    return 0.0


def main_full(names: list[str]):
    import resource
    import time
    path = os.path.join(HERE, "manifest_full.json")
    done = {}
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        for name in names:
            call, gen, flags = FULL[name]
            rs = gen()
            fqb = rs.to_fastq()
            fq = os.path.join(d, "in.fq")
            with open(fq, "wb") as f:
                f.write(fqb)
            nreads, fq_md5 = rs.n, md5(fqb)
            del rs, fqb
            t0 = time.perf_counter()
            fa, info = run_reference(fq, flags, d)
            secs = time.perf_counter() - t0
            rss = resource.getrusage(resource.RUSAGE_CHILDREN).ru_maxrss / 2**20  # KiB -> GiB
            done[name] = {"generator": call, "flags": flags, "reads": nreads,
                          "fastq_md5": fq_md5, "fasta_md5": md5(fa), "info_md5": md5(info),
                          f"reference_seconds_{threads}_threads": round(secs, 2),
                          "reference_peak_rss_gb": round(rss, 2),
                          "host_ram_gb": _host_ram_gb()}
            print(name, done[name], flush=True)
    # re-read before writing: other entries may have been regenerated meanwhile
    manifest = json.load(open(path)) if os.path.exists(path) else {}
    manifest.update(done)
    with open(path, "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


def config4_sample(jobs) -> list:
    """The serving stream's jobs the reference is run on: every job of at most
    2 Mbp and 5 of the larger ones (fixed seed)."""
    import numpy as np
    small = [j for j in jobs if j.genome_bp <= 2_000_000]
    large = [j for j in jobs if j.genome_bp > 2_000_000]
    pick = np.random.default_rng(44).choice(len(large), size=min(5, len(large)), replace=False)
    return sorted(small + [large[int(i)] for i in pick], key=lambda j: j.job_id)


def main_config4():
    import resource
    import time
    path = os.path.join(HERE, "manifest_config4.json")
    manifest = json.load(open(path)) if os.path.exists(path) else {}
    threads = os.cpu_count() or 1
    flags = ["-a", "a"]
    with tempfile.TemporaryDirectory() as d:
        for job in config4_sample(synth.config4_jobs()):
            key = str(job.job_id)
            if key in manifest:
                continue
            rs = job.reads()
            fqb = rs.to_fastq()
            fq = os.path.join(d, "in.fq")
            with open(fq, "wb") as f:
                f.write(fqb)
            nreads, fq_md5 = rs.n, md5(fqb)
            del rs, fqb
            t0 = time.perf_counter()
            fa, info = run_reference(fq, flags, d)
            secs = time.perf_counter() - t0
            manifest[key] = {"genome_bp": job.genome_bp, "read_len": job.read_len,
                             "coverage": job.coverage, "seed": job.seed, "reads": nreads,
                             "flags": flags, "fastq_md5": fq_md5, "fasta_md5": md5(fa),
                             "info_md5": md5(info),
                             f"reference_seconds_{threads}_threads": round(secs, 2),
                             "reference_peak_rss_gb": round(resource.getrusage(
                                 resource.RUSAGE_CHILDREN).ru_maxrss / 2**20, 2)}
            print(key, manifest[key], flush=True)
            with open(path + ".tmp", "w") as f:
                json.dump(manifest, f, indent=1, sort_keys=True)
            os.replace(path + ".tmp", path)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--full":
        return main_full(sys.argv[2:] or list(FULL))
    if len(sys.argv) > 1 and sys.argv[1] == "--config4-sample":
        return main_config4()
    manifest = {}
    with tempfile.TemporaryDirectory() as d:
        for name, (gen, flags) in FIXTURES.items():
            rs = gen()
            fqb = rs.to_fastq()
            fq = os.path.join(d, "in.fq")
            with open(fq, "wb") as f:
                f.write(fqb)
            fa, info = run_reference(fq, flags, d)
            aln = run_reference_aln(fq, flags, d)
            manifest[name] = dict(flags=flags, reads=rs.n, fastq_md5=md5(fqb),
                                  fasta_md5=md5(fa), info_md5=md5(info), aln_md5=md5(aln),
                                  aln_bytes=len(aln))
            if name in MAPPING_FIXTURES:
                manifest[name]["mapping_md5"] = md5(run_reference_mapping(fq, flags, d))
            if name in STORED:
                for ext, data in ((".fasta.gz", fa), (".info.gz", info)):
                    with gzip.GzipFile(os.path.join(HERE, name + ext), "wb", mtime=0) as g:
                        g.write(data)
            print(name, manifest[name], flush=True)
        for name, (gen, flags) in MERGE_FIXTURES.items():
            rs = gen()
            fqb = rs.to_fastq()
            fq = os.path.join(d, "in.fq")
            with open(fq, "wb") as f:
                f.write(fqb)
            manifest[name] = dict(flags=flags, reads=rs.n, fastq_md5=md5(fqb),
                                  **run_reference_merge(fq, flags, d))
            print(name, manifest[name], flush=True)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
