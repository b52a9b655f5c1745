"""Autotuner of the banded-DP kernel shapes.

For each class of subject batch (by the longest DP side, which follows the read
length) it builds a sample correction job with reads of that length, runs the
DP kernel under every candidate shape -- warps per block, 16-bit pairs of
segments, row-chunk or one-lane tracebacks -- and records the fastest per
class, with every candidate's time, in a JSON file (hero_b200/tuning.json by
default), which hero_b200.Hero loads.  Shapes never change results: the tests
check every candidate against the default on the same reads.

    python -m hero_b200.autotune [--out PATH] [--genome-bp N]
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import time

ALL = 0xFFFFFFFE  # bit n = n strips, n = 1..31
FROM3 = ALL & ~0x7  # 3 strips and more

# (read length of the sample, class bound on the longest DP side)
CLASSES = [(100, 112), (150, 168), (200, 224), (250, 1023)]


def candidates():
    for warps, pair, chunk in itertools.product((4, 2), (0, ALL), (ALL, 0, FROM3)):
        yield {"warps_per_block": warps, "pair_strips": pair, "chunk_strips": chunk}


def sample(read_len: int, genome_bp: int, seed: int = 91):
    from hero_b200 import synth
    return synth.Job(0, 0.0, seed + read_len, genome_bp, read_len, 40.0).reads()


def time_dp(h, reads, shape: dict, rows_max: int, rounds: int = 2) -> float:
    """Device time of the DP kernels of one correction under a shape (ms, best of rounds)."""
    h.set_tuning([dict(shape, rows_max=rows_max)])
    best = None
    for _ in range(rounds):
        s0 = h.stats()
        h.reset_votes()
        h.build_index()
        h.align_self()
        ms = h.stats()["ms_dp_kernel"] - s0["ms_dp_kernel"]
        best = ms if best is None else min(best, ms)
    return best


def tune(genome_bp: int = 60_000, device: int = 0, classes=CLASSES, log=print) -> dict:
    from hero_b200 import Hero
    out = {"device": None, "genome_bp": genome_bp, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
           "classes": []}
    try:
        import torch
        out["device"] = torch.cuda.get_device_name(device)
    except Exception:  # noqa: BLE001 - the name is informational
        pass
    for read_len, rows_max in classes:
        reads = sample(read_len, genome_bp)
        with Hero(aligner="affine", device=device, tuning=[]) as h:
            h.set_queries(reads.seq, reads.off, reads.names)
            timings = []
            for shape in candidates():
                ms = time_dp(h, reads, shape, rows_max)
                timings.append((ms, shape))
                log(f"  L={read_len} {shape} {ms:.2f} ms")
        ms, best = min(timings, key=lambda x: x[0])
        out["classes"].append(dict(best, rows_max=rows_max, read_len=read_len, ms=round(ms, 3),
                                   candidates=[dict(s, ms=round(t, 3)) for t, s in timings]))
        log(f"L={read_len}: {best} ({ms:.2f} ms)")
    return out


def main():
    ap = argparse.ArgumentParser()
    from hero_b200._lib import TUNING_PATH
    ap.add_argument("--out", default=TUNING_PATH)
    ap.add_argument("--genome-bp", type=int, default=60_000)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    rec = tune(args.genome_bp, args.device)
    with open(args.out, "w") as f:
        json.dump(rec, f, indent=1)
    print("wrote", os.path.abspath(args.out))


if __name__ == "__main__":
    main()
