"""Autotuner of the banded-DP kernel shapes.

For each sample read length it builds a correction job with reads of that
length, runs the DP kernel under every candidate shape -- warps per block,
16-bit pairs of segments, row-chunk tracebacks, registers a thread -- and records the
fastest, with every candidate's time, in a JSON file (hero_b200/tuning.json by
default), which hero_b200.Hero loads.  A class is keyed on the longest DP side
the sample's batches showed (read length - k for reads that share a k-mer
anchor, not the read length): its bound ``rows_max`` is the midpoint to the
next sample's longest side, so a batch takes the class of the nearest sample
at or above it, and the last class covers every longer batch.  Shapes never
change results: the tests check every candidate against the default on the
same reads.

Each aligner has its own classes ("classes" for the affine aligner,
"classes_global" for the global one): the two recurrences differ in
instructions and registers, so their fastest shapes may differ.

    python -m hero_b200.autotune [--out PATH] [--genome-bp N] [--aligner affine|global|both]
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import time

ALL = 0xFFFFFFFE  # bit n = n strips, n = 1..31
FROM3 = ALL & ~0x7  # 3 strips and more

# read lengths of the samples, one class each
READ_LENGTHS = [100, 150, 200, 250]
# bound of the last class: every batch the shared-memory kernel takes
ROWS_LAST = 1023


def candidates():
    # row-chunk walks for all strip counts or from three on (one-lane walks never won)
    # 255 registers (8 warps a SM) only with 1-warp blocks
    for warps, pair, chunk, regs in itertools.product((4, 2, 1), (0, ALL), (ALL, FROM3), (128, 168, 255)):
        if regs == 255 and warps != 1:
            continue
        yield {"warps_per_block": warps, "pair_strips": pair, "chunk_strips": chunk,
               "regs_per_thread": regs}


def sample(read_len: int, genome_bp: int, seed: int = 91):
    from hero_b200 import synth
    return synth.Job(0, 0.0, seed + read_len, genome_bp, read_len, 40.0).reads()


def time_dp(h, reads, shape: dict, rounds: int = 2) -> float:
    """Device time of the DP kernels of one correction under a shape (ms, best of rounds)."""
    h.set_tuning([dict(shape, rows_max=ROWS_LAST)])
    best = None
    for _ in range(rounds):
        s0 = h.stats()
        h.reset_votes()
        h.build_index()
        h.align_self()
        ms = h.stats()["ms_dp_kernel"] - s0["ms_dp_kernel"]
        best = ms if best is None else min(best, ms)
    return best


def class_bounds(rows: list[int]) -> list[int]:
    """rows_max of each class from the samples' longest DP sides (ascending)."""
    return [(a + b) // 2 for a, b in zip(rows, rows[1:])] + [ROWS_LAST]


def tune(genome_bp: int = 60_000, device: int = 0, read_lengths=READ_LENGTHS, log=print,
         aligner: str = "affine") -> dict:
    from hero_b200 import Hero
    out = {"device": None, "genome_bp": genome_bp, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
           "aligner": aligner, "classes": []}
    try:
        import torch
        out["device"] = torch.cuda.get_device_name(device)
    except Exception:  # noqa: BLE001 - the name is informational
        pass
    for read_len in sorted(read_lengths):
        reads = sample(read_len, genome_bp)
        with Hero(aligner=aligner, device=device, tuning=[]) as h:
            h.set_queries(reads.seq, reads.off, reads.names)
            timings = []
            for shape in candidates():
                ms = time_dp(h, reads, shape)
                timings.append((ms, shape))
                log(f"  L={read_len} {shape} {ms:.2f} ms")
            rows = int(h.stats()["dp_rows_max"])
        ms, best = min(timings, key=lambda x: x[0])
        out["classes"].append(dict(best, rows_seen=rows, read_len=read_len, ms=round(ms, 3),
                                   candidates=[dict(s, ms=round(t, 3)) for t, s in timings]))
        log(f"L={read_len} (longest DP side {rows}): {best} ({ms:.2f} ms)")
    for c, bound in zip(out["classes"], class_bounds([c["rows_seen"] for c in out["classes"]])):
        c["rows_max"] = bound
    return out


def main():
    ap = argparse.ArgumentParser()
    from hero_b200._lib import TUNING_PATH
    ap.add_argument("--out", default=TUNING_PATH)
    ap.add_argument("--genome-bp", type=int, default=60_000)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--aligner", default="both", choices=["affine", "global", "both"])
    args = ap.parse_args()
    rec = {}
    if os.path.exists(args.out):
        with open(args.out) as f:
            rec = json.load(f)
    for aligner in (("affine", "global") if args.aligner == "both" else (args.aligner,)):
        r = tune(args.genome_bp, args.device, aligner=aligner)
        key = "classes" if aligner == "affine" else "classes_global"
        rec.update({k: r[k] for k in ("device", "genome_bp", "when")})
        rec[key] = r["classes"]
    with open(args.out, "w") as f:
        json.dump(rec, f, indent=1)
    print("wrote", os.path.abspath(args.out))


if __name__ == "__main__":
    main()
