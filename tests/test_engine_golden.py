"""The `engine` command on the GPU against the reference engine's own outputs (tests/golden):
every result file byte for byte (ca_result.bin/.txt, mc_result.bin/.txt, mc_stats.csv,
config_used.json, step and MCS snapshots), stats.json equal apart from its "parallel" section, the
section and info keys of times.json a superset of the reference's, --mc-from and --batch runs."""
from __future__ import annotations

import csv
import hashlib
import json
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENGINE = os.path.join(ROOT, "volcano_ca_mc_b200", "bin", "engine")
GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = sorted(f[:-5] for f in os.listdir(os.path.join(GOLDEN, "cases"))
               if f.endswith(".json") and not f.startswith("mcfrom"))

pytestmark = pytest.mark.gpu


def sha(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def run(*args, cwd=None):
    r = subprocess.run([ENGINE, *args], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, cwd=cwd,
                       timeout=300)
    return r


def compare(out, exp, skip=()):
    for name, digest in exp["files"].items():
        if name in skip:
            continue
        assert os.path.exists(os.path.join(out, name)), name
        assert sha(os.path.join(out, name)) == digest, name
    for name, digest in exp["snapshots"].items():
        assert sha(os.path.join(out, name)) == digest, name
    with open(os.path.join(out, "stats.json")) as f:
        stats = json.load(f)
    assert "parallel" in stats
    stats.pop("parallel")
    if "mc_from" in exp:
        stats.pop("source")
    assert stats == exp["stats"]
    if "mc_stats_csv" in exp:
        with open(os.path.join(out, "mc_stats.csv")) as f:
            assert f.read() == exp["mc_stats_csv"]
    with open(os.path.join(out, "times.json")) as f:
        times = json.load(f)
    ignore = {"openmp", "threadStats", "priority"}  # the reference's CPU-thread details
    missing = [k for k in exp["times_keys"] if k not in times and k not in ignore]
    assert not missing, missing


def load_expect(name):
    with open(os.path.join(GOLDEN, name, "expect.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", CASES)
def test_engine_matches_reference(case, tmp_path):
    out = tmp_path / case
    r = run("--config", os.path.join(GOLDEN, "cases", f"{case}.json"), "--out", str(out))
    assert r.returncode == 0, r.stderr
    compare(str(out), load_expect(case))


def test_engine_progress_same_result(tmp_path):
    """--progress steps the CA one launch at a time and the MC one sweep at a time: same results."""
    out = tmp_path / "p"
    r = run("--config", os.path.join(GOLDEN, "cases", "lava2d_moore.json"), "--out", str(out), "--progress")
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("PROGRESS ")]
    assert any(l.startswith("PROGRESS ca ") for l in lines) and any(l.startswith("PROGRESS mc ") for l in lines)
    # every line in the form the reference's GUI job queue parses (gui/jobs.py:63)
    gui = re.compile(r"^PROGRESS (\w+) (\d+)/(\d+)(?: (\w+)=(\d+))?\s*$")
    assert all(gui.match(l) for l in lines), [l for l in lines if not gui.match(l)][:3]
    compare(str(out), load_expect("lava2d_moore"))


def test_engine_mc_from(tmp_path):
    src = tmp_path / "src"
    r = run("--config", os.path.join(GOLDEN, "cases", "lava2d_moore.json"), "--out", str(src))
    assert r.returncode == 0, r.stderr
    out = tmp_path / "mc"
    r = run("--mc-from", str(src), "--config", os.path.join(GOLDEN, "cases", "mcfrom_lava2d.json"), "--out", str(out))
    assert r.returncode == 0, r.stderr
    # config_used.json carries the absolute path of the source folder
    compare(str(out), load_expect("mcfrom_lava2d"), skip={"config_used.json"})


def test_engine_batch(tmp_path):
    cfgs = tmp_path / "cfgs"
    cfgs.mkdir()
    for c in ("classic2d_vn", "mc_full_2d_hex"):
        shutil.copy(os.path.join(GOLDEN, "cases", f"{c}.json"), cfgs / f"{c}.json")
    (cfgs / "_skipped.json").write_text("{}")
    (cfgs / "broken.json").write_text('{"space": {"nx": 0}}')
    out = tmp_path / "out"
    r = run("--batch", str(cfgs), "--out", str(out))
    assert r.returncode == 5, r.stdout + r.stderr
    with open(out / "batch_summary.csv") as f:
        rows = list(csv.DictReader(f))
    assert [row["name"] for row in rows] == ["broken", "classic2d_vn", "mc_full_2d_hex"]
    assert [row["status"] for row in rows] == ["error", "ok", "ok"]
    assert rows[0]["error"].startswith("Błąd konfiguracji")
    for c in ("classic2d_vn", "mc_full_2d_hex"):
        compare(str(out / c), load_expect(c))
