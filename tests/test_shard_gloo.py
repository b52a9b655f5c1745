"""The multi-rank paths on the CPU, as world-size-2 gloo process groups: the
rank helpers the bench and the sharded correction use, the vote exchange
(the shards' votes summed by the all-reduce equal the whole run's, checked
with the oracle), and a rank that leaves before the exchange."""
import ast
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return str(s.getsockname()[1])


def _run(case, tmp_path, world=2, timeout=240):
    port = _port()
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "gloo_worker.py"), case, str(r),
                               str(world), port, str(tmp_path)],
                              stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
             for r in range(world)]
    outs = []
    for p in procs:
        try:
            outs.append(p.communicate(timeout=timeout)[0].decode(errors="replace"))
        except subprocess.TimeoutExpired:
            p.kill()
            outs.append(p.communicate()[0].decode(errors="replace"))
    res = {}
    for r in range(world):
        f = tmp_path / f"rank{r}.txt"
        if f.exists():
            res[r] = ast.literal_eval(f.read_text())
    return procs, outs, res


def test_shard_ranges_cover_the_reads():
    from hero_b200.shard import shard_range
    for n in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            got = [shard_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_rank_helpers_over_gloo(tmp_path):
    procs, outs, res = _run("basics", tmp_path)
    assert all(p.returncode == 0 for p in procs), outs
    assert res[0]["world_rank"] == [2, 0] and res[1]["world_rank"] == [2, 1]
    assert res[0]["max"] == res[1]["max"] == 1.5
    assert res[0]["range"] == [0, 501] and res[1]["range"] == [501, 1001]


def test_vote_exchange_gives_the_whole_runs_votes(tmp_path, oracle):
    from fixtures import FIXTURES, params, upper
    procs, outs, res = _run("votes", tmp_path)
    assert all(p.returncode == 0 for p in procs), outs
    gen, flags = FIXTURES["mix_affine"]
    want = oracle.correct(upper(gen()), **params(flags))["votes"]
    for r in range(2):
        got = np.load(tmp_path / f"votes{r}.npy")
        assert np.array_equal(got, want)


def test_reduce_to_owners_gives_each_owner_the_whole_runs_votes(tmp_path, oracle):
    from fixtures import FIXTURES, params, upper
    procs, outs, res = _run("owners", tmp_path)
    assert all(p.returncode == 0 for p in procs), outs
    gen, flags = FIXTURES["mix_affine"]
    want = oracle.correct(upper(gen()), **params(flags))["votes"]
    slices = [res[r]["slice"] for r in range(2)]
    assert slices[0][0] == 0 and slices[0][1] == slices[1][0] and slices[1][1] == len(want)
    for r in range(2):
        lo, hi = slices[r]
        assert np.array_equal(np.load(tmp_path / f"own{r}.npy"), want[lo:hi])


def test_owner_slices_cover_the_state():
    from hero_b200.shard import owner_slices
    off = np.array([0, 10, 25, 25, 40, 100], np.uint64)
    for world in (1, 2, 3):
        o = owner_slices(off, world)
        assert sum(c for _, c, _, _ in o) == 5 and sum(nb for _, _, nb, _ in o) == 100
        assert o[0][3][0][0] == 0 and o[-1][3][0][1] == 400
        assert o[0][3][1][0] == 400 and o[-1][3][1][1] == 500


def test_a_rank_that_leaves_ends_the_exchange_with_an_error(tmp_path):
    procs, outs, res = _run("lost_rank", tmp_path, timeout=120)
    assert procs[1].returncode == 0
    assert res[0]["error"] is not None, outs
