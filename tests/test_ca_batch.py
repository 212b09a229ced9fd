"""Batched stepping (vca_ca_batch_*): many grids of different sizes, dimensionality, neighbourhoods,
boundaries, seeds and schedules stepped by shared launches must each end exactly as when run alone
(LavaCA::run, engine/src/ca/LavaCA.hpp:253-256): the same step count, stop reason, per-step
histories and planes, bit for bit -- whether they join together, one after another while others
run, or leave early."""
import numpy as np
import pytest

from tests import cases as C
from volcano_ca_mc_b200 import capi, serve

pytestmark = pytest.mark.gpu


def jobs(n, seed):
    mix = serve.make_mix(n, seed, side_2d=(64, 300), side_3d=(20, 56), steps=(30, 160), mcs=(1, 2))
    for k, j in enumerate(mix):
        j.job_id = k
    return mix


def setup(job, sweep):
    p = job.ca_params()
    p.sweep = sweep
    ca = capi.LavaCA(p)
    heights, vents = job.terrain()
    ca.apply_terrain(heights)
    ca.place_seeds(vents)
    return ca


def outcome(ca):
    info = ca.info()
    return info.steps, info.stop_reason, ca.history(), ca.download()


def same(a, b):
    assert a[:3] == b[:3]
    for x, y in zip(a[3], b[3]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("sweep", [capi.SWEEP_ACTIVE, capi.SWEEP_DENSE], ids=["active", "dense"])
def test_batch_members_match_single_runs(sweep):
    mix = jobs(14, 404)
    alone = []
    for j in mix:
        ca = setup(j, sweep)
        ca.run()
        alone.append(outcome(ca))
        ca.close()
    batch = capi.CaBatch(max_members=64)
    handles = [setup(j, sweep) for j in mix]
    for h in handles:
        batch.add(h)
    order = batch.run()
    assert sorted(id(h) for h in order) == sorted(id(h) for h in handles)
    for h, want in zip(handles, alone):
        same(outcome(h), want)
    assert batch.info()["members"] == 0 and batch.info()["graphs"] > 0
    batch.close()
    for h in handles:
        h.close()


def test_members_join_while_others_run_and_handles_are_reused():
    mix = jobs(10, 77)
    alone = []
    for j in mix:
        ca = setup(j, capi.SWEEP_ACTIVE)
        ca.run()
        alone.append(outcome(ca))
        ca.close()
    batch = capi.CaBatch(max_members=4)
    results = {}
    waiting = list(range(len(mix)))
    live = {}
    while waiting or live:
        while waiting and len(live) < 4:  # at most 4 members at a time: jobs join as others leave
            k = waiting.pop(0)
            h = setup(mix[k], capi.SWEEP_ACTIVE)
            batch.add(h)
            live[id(h)] = (k, h)
        done, _ = batch.advance(max_graphs=1)
        for h in done:
            k, _ = live.pop(id(h))
            results[k] = outcome(h)
            h.close()
    for k, want in enumerate(alone):
        same(results[k], want)
    batch.close()


def test_member_calls_refused_and_remove_mid_run():
    job = jobs(1, 5)[0]
    job.max_steps = 150
    ref = setup(job, capi.SWEEP_ACTIVE)
    ref.run()
    want = outcome(ref)
    ref.close()
    h = setup(job, capi.SWEEP_ACTIVE)
    batch = capi.CaBatch()
    batch.add(h)
    with pytest.raises(capi.VcaError, match=r"\(status 2\).*batch"):
        h.step()
    with pytest.raises(capi.VcaError, match=r"\(status 2\).*batch"):
        h.download()
    batch.advance(max_graphs=2)
    batch.remove(h)
    assert 0 < h.info().steps < 150 or h.info().stop_reason != 0
    h.run()  # the rest alone
    same(outcome(h), want)
    batch.close()
    h.close()


def test_member_without_lava_is_reported_at_once():
    nx, ny, nz = 40, 1, 30
    p = capi.CaParams(nx, ny, nz, max_steps=50)
    h = capi.LavaCA(p)
    h.apply_terrain(C.terrain(nx, ny, nz, 3))
    h.place_seeds([])
    batch = capi.CaBatch()
    batch.add(h)
    done, running = batch.advance()
    assert done == [h] and running == 0
    assert h.info().stop_reason == 1  # no lava (countInitialState, LavaCA.hpp:1272-1279)
    batch.close()
    h.close()
