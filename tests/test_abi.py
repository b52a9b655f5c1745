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
    assert len(list(autotune.candidates())) == 28
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


def test_committed_tuning_passes_the_library_check():
    """Every class of the committed tuning record is one the library (contexts
    and servers alike) accepts; refused shapes stay refused."""
    import ctypes as C

    from hero_b200 import load_library
    from hero_b200._lib import DpTuning, load_tuning
    lib = load_library()

    def check(classes):
        arr = (DpTuning * max(1, len(classes)))()
        for i, t in enumerate(classes):
            arr[i] = DpTuning(int(t["rows_max"]), int(t["warps_per_block"]), int(t["pair_strips"]),
                              int(t["chunk_strips"]), int(t.get("regs_per_thread", 0)))
        return lib.hero_dp_tuning_check(arr, C.c_uint32(len(classes)))

    for aligner in ("affine", "global"):
        classes = load_tuning(None, aligner)
        assert classes and check(classes) == 0, aligner
    base = {"rows_max": 100, "pair_strips": 0, "chunk_strips": 0}
    assert check([dict(base, warps_per_block=1, regs_per_thread=255)]) == 0
    assert check([dict(base, warps_per_block=2, regs_per_thread=255)]) != 0
    assert check([dict(base, warps_per_block=3, regs_per_thread=0)]) != 0
    assert check([dict(base, warps_per_block=4, regs_per_thread=200)]) != 0
