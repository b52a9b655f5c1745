"""The C ABI library builds for sm_100a and exports every declared entry point."""
import os
import re
import subprocess

from hero_b200 import EXPORTS, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "hero_gpu.h")).read()
    return sorted(set(re.findall(r"\b(hero_[a-z_]+)\s*\(", src)))


def test_header_lists_exports():
    assert sorted(EXPORTS) == declared()


def test_library_exports_every_symbol():
    lib = build.build_library()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared() if s not in syms]
    assert not missing, missing


def test_library_loads_without_gpu():
    from hero_b200 import load_library
    lib = load_library()
    for s in declared():
        assert hasattr(lib, s)


def test_built_for_sm100a_only():
    # the one target of every CUDA build: sm_100a code, no PTX for other archs
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "--use_fast_math" not in build.NVFLAGS and "--fmad=false" in build.NVFLAGS


def test_tuning_record_parses(tmp_path):
    import json

    from hero_b200 import autotune
    from hero_b200._lib import load_tuning
    assert len(list(autotune.candidates())) == 24
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"classes": [{"rows_max": 168, "warps_per_block": 2, "pair_strips": 0,
                                          "chunk_strips": autotune.ALL}]}))
    assert load_tuning(str(p)) == [{"rows_max": 168, "warps_per_block": 2, "pair_strips": 0,
                                    "chunk_strips": autotune.ALL}]
    assert load_tuning(str(tmp_path / "missing.json")) == []


def test_tuning_class_bounds_meet_halfway():
    from hero_b200 import autotune
    # samples whose batches showed longest DP sides 61, 111, 161, 211
    assert autotune.class_bounds([61, 111, 161, 211]) == [86, 136, 186, autotune.ROWS_LAST]
    assert autotune.class_bounds([111]) == [autotune.ROWS_LAST]
