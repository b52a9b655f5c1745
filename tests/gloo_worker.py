"""One rank of the world-size-2 gloo tests (test_shard_gloo.py); run as a process:

    python tests/gloo_worker.py CASE RANK WORLD PORT OUTDIR
"""
import os
import sys
from datetime import timedelta

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.dirname(HERE), HERE, os.path.join(HERE, "golden")]


class Slice:
    """Reads [a, b) of a read set, as the oracle's subject set."""

    def __init__(self, rs, a, b):
        o = rs.off[a:b + 1]
        self.seq = rs.seq[o[0]:o[-1]]
        self.off = o - o[0]
        self.names = rs.names[a:b]
        self.n = b - a


def main():
    case, rank, world, port, out = sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), sys.argv[4], sys.argv[5]
    import numpy as np
    import torch
    import torch.distributed as dist

    from hero_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = port
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20))
    res = {}
    try:
        if case == "basics":
            res["world_rank"] = list(shard.world_rank())
            res["max"] = shard.max_over_ranks(float(rank) + 0.5)
            res["range"] = list(shard.shard_range(1001, rank, world))
        elif case == "votes":
            from fixtures import FIXTURES, params, upper
            from hero_testlib import Oracle
            gen, flags = FIXTURES["mix_affine"]
            rs = upper(gen())
            a, b = shard.shard_range(rs.n, rank, world)
            kw = params(flags)
            v = Oracle().correct(rs, subjects=Slice(rs, a, b), threads=2, **kw)["votes"]
            t = torch.from_numpy(v.view(np.int32).copy())
            shard.allreduce_votes(t)
            np.save(os.path.join(out, f"votes{rank}.npy"), t.numpy().view(np.uint32))
        elif case == "owners":
            # the shards' oracle vote matrices ([bases][4] words) reduced to the
            # owners of query-read ranges: each owner's slice is the whole run's
            from fixtures import FIXTURES, params, upper
            from hero_testlib import Oracle
            gen, flags = FIXTURES["mix_affine"]
            rs = upper(gen())
            a, b = shard.shard_range(rs.n, rank, world)
            v = Oracle().correct(rs, subjects=Slice(rs, a, b), threads=2, **params(flags))["votes"]
            t = torch.from_numpy(v.view(np.int32).copy())
            owners = shard.owner_slices(rs.off, world, words_per_base=4, tail_words=0)
            shard.reduce_votes_to_owners(t, owners)
            lo, hi = owners[rank][3][0]
            np.save(os.path.join(out, f"own{rank}.npy"), t[lo:hi].numpy().view(np.uint32))
            res["slice"] = [lo, hi]
        elif case == "lost_rank":
            if rank == 1:
                os._exit(0)  # leaves between steps, before the exchange
            t = torch.zeros(4, dtype=torch.int32)
            try:
                shard.allreduce_votes(t)
                res["error"] = None
            except Exception as e:  # noqa: BLE001 - the failure is the result
                res["error"] = type(e).__name__
        with open(os.path.join(out, f"rank{rank}.txt"), "w") as f:
            f.write(repr(res))
    finally:
        if case != "lost_rank":
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
