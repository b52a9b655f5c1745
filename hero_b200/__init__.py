"""B200-native HERO read-correction path (k-mer seeding, chaining, banded DP,
record selection, consensus) behind a C ABI (include/hero_gpu.h).

    from hero_b200 import Hero, synth
    reads = synth.config1(genome_bp=20_000)
    with Hero(aligner="global") as h:
        h.set_queries(reads.seq, reads.off, reads.names)
        h.build_index()
        h.align_self()
        out = h.consensus()
"""
from ._lib import (EXPORTS, Hero, HeroError, HeroServer, align_output, correct,  # noqa: F401
                   load_library)

__all__ = ["Hero", "HeroError", "HeroServer", "align_output", "correct", "load_library",
           "EXPORTS"]
