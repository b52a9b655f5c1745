"""Builds HERO itself with the hero-b200 drop-in binding (test infrastructure).

The reference program is compiled from its own sources, where they lie, with
three lines of its main.cpp changed -- the edit a HERO maintainer makes to
adopt the library (main.cpp:60-72, 92):

    new HashTableLongKey(queryDataset)     -> new HashTableGpu(queryDataset)
    new SubjectReadAligner(hashTable)      -> new SubjectReadAlignerGpu(hashTable)
    queryDataset->callConsensus()          -> HashTableGpu::callConsensus(queryDataset)

plus the include of oracle/dropin/hero_gpu_binding.h, whose classes derive
from the reference's HashTableMethod and SubjectReadAligner and call the C ABI
of hero_b200/libhero_b200.so.  Everything else -- Config::setConfig, the
QueryDataset parser and quality filter, SubjectDataset's chunk streaming,
writeQueryOut -- is the reference's own code.  Only the edited main.cpp is
written, to a temporary directory; the output is oracle/_ref/hero_ref_gpu
(linked with an rpath to the library in this tree).

    python oracle/dropin/make_dropin.py          # needs the reference sources and the built library

The reference sources are HERO_REFERENCE_SRC, else a checkout named
"reference" beside this repository; without them nothing is built.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
OUT = os.path.join(ORACLE, "_ref", "hero_ref_gpu")
LIBDIR = os.path.join(ROOT, "hero_b200")

# (text in the reference's main.cpp, replacement): each must occur exactly once
EDITS = [
    ('#include "SubjectReadAligner.h"',
     '#include "SubjectReadAligner.h"\n#include "hero_gpu_binding.h"'),
    ("hashTable = new HashTableLongKey(queryDataset);",
     "hashTable = new HashTableGpu(queryDataset);"),
    ("SubjectReadAligner * aligner = new SubjectReadAligner(hashTable);",
     "SubjectReadAlignerGpu * aligner = new SubjectReadAlignerGpu(hashTable);"),
    ("queryDataset->callConsensus();", "HashTableGpu::callConsensus(queryDataset);"),
]


def ref_src() -> str:
    return os.environ.get("HERO_REFERENCE_SRC",
                          os.path.join(os.path.dirname(ROOT), "reference", "src"))


def edited_main(src: str) -> str:
    text = open(os.path.join(src, "main.cpp")).read()
    for old, new in EDITS:
        if text.count(old) != 1:
            raise RuntimeError(f"main.cpp: expected one occurrence of {old!r}")
        text = text.replace(old, new)
    return text


def build(verbose: bool = False) -> str | None:
    src = ref_src()
    if not os.path.isdir(src):
        if verbose:
            print("reference sources not present; nothing built")
        return None
    lib = os.path.join(LIBDIR, "libhero_b200.so")
    if not os.path.exists(lib):
        raise RuntimeError("build hero_b200/libhero_b200.so first (python -m hero_b200.build)")
    others = sorted(p for p in glob.glob(os.path.join(src, "*.cpp"))
                    if os.path.basename(p) != "main.cpp")
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    with tempfile.TemporaryDirectory() as d:
        main = os.path.join(d, "main.cpp")
        with open(main, "w") as f:
            f.write(edited_main(src))
        rpath = "$ORIGIN/" + os.path.relpath(LIBDIR, os.path.dirname(OUT))
        cmd = (["g++", "-std=gnu++98", "-fopenmp", "-O3", "-w", "-I", src, "-I", HERE,
                "-I", os.path.join(ROOT, "include"), "-o", OUT + ".tmp", main] + others +
               [os.path.join(HERE, "hero_gpu_binding.cpp"), "-L", LIBDIR, "-lhero_b200",
                f"-Wl,-rpath,{rpath}"])
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True) or "", file=sys.stderr)
