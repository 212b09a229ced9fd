"""The job server (engine --serve) on the GPU: engine configs sent to one server process, their CA
grids stepped together in the shared batch, give every job the result of a single run of the same
config -- the same digests as the one-at-a-time plain path (one worker, vca_ca_run per job), and,
where the request names an output folder, result files byte-identical to `engine --config`'s."""
from __future__ import annotations

import filecmp
import json
import os
import subprocess

import pytest

from volcano_ca_mc_b200 import capi, serve

pytestmark = pytest.mark.gpu


def test_served_mix_equals_one_at_a_time():
    jobs = serve.make_mix(16, 21, share_3d=0.4, side_2d=(64, 384), side_3d=(32, 96), steps=(60, 160), mcs=(5, 20))
    many = serve.run(jobs, slots=4, batched=True)
    one = serve.run(jobs, slots=1, batched=False)
    assert many["jobs"] == one["jobs"] == len(jobs)
    assert all(r["status"] == "ok" for r in many["records"].values())
    assert serve.compare(many, one) == 0
    assert many["server"]["batch_graphs"] > 0


def test_served_files_equal_single_runs(tmp_path):
    jobs = serve.make_mix(6, 8, share_3d=0.5, side_2d=(64, 256), side_3d=(32, 64), steps=(60, 120), mcs=(5, 10))
    srv = serve.EngineServer(slots=3, batched=True)
    for j in jobs:
        cfg = j.config(str(tmp_path))
        cfg["output"] = {"format": "bin"}
        (tmp_path / f"job{j.job_id}.json").write_text(json.dumps(cfg))
        srv.submit({"id": str(j.job_id), "config": str(tmp_path / f"job{j.job_id}.json"),
                    "out": str(tmp_path / f"served{j.job_id}")})
    assert srv.close() == 0, srv.stderr()
    for j in jobs:
        assert srv.answers[str(j.job_id)]["status"] == "ok"
        single = tmp_path / f"single{j.job_id}"
        r = subprocess.run([capi.ENGINE_PATH, "--config", str(tmp_path / f"job{j.job_id}.json"), "--out", str(single)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        for name in ("ca_result.bin", "mc_result.bin", "mc_stats.csv", "config_used.json"):
            assert filecmp.cmp(single / name, tmp_path / f"served{j.job_id}" / name, shallow=False), (j.job_id, name)
        a = json.loads((single / "stats.json").read_text())
        b = json.loads((tmp_path / f"served{j.job_id}" / "stats.json").read_text())
        assert a == b


def test_budget_governs_allocations():
    """With a budget that holds only a few resident handles, the server frees idle ones to admit new
    shapes and never holds more device bytes than the budget."""
    jobs = serve.make_mix(10, 5, share_3d=0.5, side_2d=(64, 512), side_3d=(32, 96), steps=(40, 80), mcs=(2, 4))
    res = serve.run(jobs, slots=4, batched=True, budget_gb=0.05)
    s = res["server"]
    assert res["jobs"] == len(jobs)
    assert s["peak_allocated_bytes"] <= s["budget_bytes"]
    assert s["handles_freed"] > 0


def test_served_realtime_trace():
    jobs = serve.make_mix(12, 4, share_3d=0.3, rate_hz=40.0, side_2d=(64, 256), side_3d=(32, 64), steps=(50, 120),
                          mcs=(5, 10))
    res = serve.run(jobs, slots=4, realtime=True)
    assert res["jobs"] == len(jobs) and res["p99_s"] >= res["p50_s"] > 0
    for r in res["records"].values():
        assert r["admitted_ms"] >= r["arrival_ms"] - 1e-3 and r["done_ms"] > r["admitted_ms"]


def test_served_sizes_grow_and_shrink(tmp_path):
    """Larger jobs (up to 1.9 M cells) whose sizes grow and shrink from job to job on two workers and
    their resident handles: every result file equals the single run's, and the two modes agree on
    every digest."""
    sizes = [(700, 1, 500), (1500, 1, 900), (300, 1, 400), (160, 160, 80), (1700, 1, 1100), (900, 1, 700)]
    jobs = serve.make_mix(len(sizes), 31, share_3d=0.0, side_2d=(64, 128), steps=(30, 60), mcs=(2, 4))
    for j, (nx, ny, nz) in zip(jobs, sizes):
        j.nx, j.ny, j.nz = nx, ny, nz
        if ny > 1 and j.neighborhood == "hexagonal":  # the reference rejects hexagonal in 3D
            j.neighborhood = "moore"
    srv = serve.EngineServer(slots=2, batched=True)
    for j in jobs:
        cfg = j.config(str(tmp_path))
        cfg["output"] = {"format": "bin"}
        (tmp_path / f"job{j.job_id}.json").write_text(json.dumps(cfg))
        srv.submit({"id": str(j.job_id), "config": str(tmp_path / f"job{j.job_id}.json"),
                    "out": str(tmp_path / f"served{j.job_id}")})
    assert srv.close() == 0, srv.stderr()
    for j in jobs:
        assert srv.answers[str(j.job_id)]["status"] == "ok", srv.answers[str(j.job_id)]
        single = tmp_path / f"single{j.job_id}"
        r = subprocess.run([capi.ENGINE_PATH, "--config", str(tmp_path / f"job{j.job_id}.json"), "--out", str(single)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        for name in ("ca_result.bin", "mc_result.bin"):
            assert filecmp.cmp(single / name, tmp_path / f"served{j.job_id}" / name, shallow=False), (j.job_id, name)
    one = serve.run(jobs, slots=1, batched=False)
    assert all(one["records"][j.job_id]["digest"] == srv.answers[str(j.job_id)]["digest"] for j in jobs)
