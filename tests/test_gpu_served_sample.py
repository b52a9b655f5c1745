"""The serving stream against the reference: the sampled jobs (every job of at
most 2 Mbp plus 5 larger ones, tests/golden/make_golden.py --config4-sample)
are submitted together to one hero_server, and every served job's .fasta and
.info are byte-identical to the reference's run of that job alone
(golden/manifest_config4.json; skipped until those runs are recorded)."""
import hashlib
import json
import multiprocessing as mp
import os

import pytest
from hero_testlib import format_outputs

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PATH = os.path.join(HERE, "manifest_config4.json")
MANIFEST = json.load(open(PATH)) if os.path.exists(PATH) else {}


def _reads(job):
    rs = job.reads()
    return job.job_id, rs.seq, rs.off, rs.names


@pytest.mark.skipif(not MANIFEST, reason="reference runs of the sampled jobs not recorded yet")
def test_served_jobs_match_the_reference():
    from hero_b200 import HeroServer, synth
    jobs = [j for j in synth.config4_jobs() if str(j.job_id) in MANIFEST]
    # generated in spawn processes before the server starts any CUDA work
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        data = {jid: (seq, off, names) for jid, seq, off, names in pool.map(_reads, jobs)}
    with HeroServer(aligner="affine") as srv:
        ids = {j.job_id: srv.submit(*data[j.job_id]) for j in jobs}
        for jid, i in ids.items():
            info = srv.wait(i)
            assert info["state"] == 2, (jid, info)
            r = srv.result(i)
            seq, off, names = data[jid]
            fa, inf = format_outputs(names, r["seq"], off, r["imin"], r["imed"], r["imax"],
                                     r["mismatch_rate"], r["gc"])
            m = MANIFEST[str(jid)]
            assert off.size - 1 == m["reads"], jid
            assert hashlib.md5(fa).hexdigest() == m["fasta_md5"], jid
            assert hashlib.md5(inf).hexdigest() == m["info_md5"], jid
            srv.release(i)
