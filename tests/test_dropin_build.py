"""HERO itself, built with the drop-in binding (oracle/dropin): the three edits
apply to the reference's main.cpp, and the program links libhero_b200.so.
Needs the reference sources (skipped where they are absent)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle", "dropin"))
import make_dropin  # noqa: E402

pytestmark = pytest.mark.skipif(not os.path.isdir(make_dropin.ref_src()),
                                reason="reference sources not present")


def test_edits_apply_once_each():
    text = make_dropin.edited_main(make_dropin.ref_src())
    assert "new HashTableGpu(queryDataset)" in text
    assert "new SubjectReadAlignerGpu(hashTable)" in text
    assert "HashTableGpu::callConsensus(queryDataset)" in text
    assert "new HashTableLongKey(queryDataset)" not in text


def test_hero_builds_against_the_library():
    from hero_b200 import build
    build.build_library()
    out = make_dropin.build()
    assert out and os.path.exists(out)
    libs = subprocess.run(["ldd", out], capture_output=True, text=True).stdout
    assert "libhero_b200.so" in libs
