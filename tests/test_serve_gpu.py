"""The job server on the GPU: a mix of small 2D and 3D jobs run on 4 worker slots (resident handles,
reconfigured per job, overlapping on the device) gives every job the same result as one slot running
them one at a time, and as a new handle per job."""
from __future__ import annotations

import hashlib

import pytest

from volcano_ca_mc_b200 import capi, serve

pytestmark = pytest.mark.gpu


def _plain(job):
    heights, vents = job.terrain()
    ca = capi.LavaCA(job.ca_params())
    ca.apply_terrain(heights)
    ca.place_seeds(vents)
    ca.run()
    planes = ca.download()
    mc = capi.PottsMC(job.mc_params())
    mc.set_domain_from_ca(ca)
    mc.set_mobility_from_ca(ca, 0.05, True)
    mc.initialize()
    mc.sweep(job.mcs)
    h = hashlib.sha256()
    for a in planes:
        h.update(memoryview(a).cast("B"))
    h.update(memoryview(mc.crystals()).cast("B"))
    mc.close()
    ca.close()
    return h.hexdigest()[:24]


def test_served_mix_equals_one_at_a_time_and_plain():
    jobs = serve.make_mix(16, 21, share_3d=0.4, side_2d=(64, 384), side_3d=(32, 96), steps=(60, 160), mcs=(5, 20))
    many = serve.run(jobs, slots=4)
    one = serve.run(jobs, slots=1)
    assert many["jobs"] == one["jobs"] == len(jobs)
    assert serve.compare(many, one) == 0
    for job in jobs[:4]:
        assert many["records"][job.job_id]["sha"] == _plain(job)


def test_served_realtime_trace():
    jobs = serve.make_mix(12, 4, share_3d=0.3, rate_hz=40.0, side_2d=(64, 256), side_3d=(32, 64), steps=(50, 120),
                          mcs=(5, 10))
    res = serve.run(jobs, slots=4, realtime=True)
    assert res["jobs"] == len(jobs) and res["p99_s"] >= res["p50_s"] > 0
    for r in res["records"].values():
        assert r["start"] >= r["arrival"] - 1e-3 and r["end"] > r["start"]
