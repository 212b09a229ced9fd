"""Host logic of the `engine` command (no GPU used): the reference's defaults, config validation,
argument errors and exit codes (engine/src/main.cpp:6-8, engine/src/app/Cli.cpp:36-131,
engine/src/app/ConfigCheck.cpp:46-62)."""
from __future__ import annotations

import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENGINE = os.path.join(ROOT, "volcano_ca_mc_b200", "bin", "engine")
GOLDEN = os.path.join(ROOT, "tests", "golden")

pytestmark = pytest.mark.skipif(not os.path.exists(ENGINE), reason="engine not built (make -C volcano_ca_mc_b200/csrc)")


def run(*args, cwd=None):
    return subprocess.run([ENGINE, *args], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, cwd=cwd,
                          timeout=60)


def test_print_defaults_equal_reference():
    r = run("--print-defaults")
    assert r.returncode == 0
    with open(os.path.join(GOLDEN, "print_defaults.json")) as f:
        assert r.stdout == f.read()


def test_help():
    r = run("--help")
    assert r.returncode == 0 and "--config" in r.stdout and "--mc-from" in r.stdout


@pytest.mark.parametrize("case", sorted(f[:-5] for f in os.listdir(os.path.join(GOLDEN, "cases")) if f.endswith(".json")))
def test_validate_golden_cases(case):
    r = run("--validate", "--config", os.path.join(GOLDEN, "cases", f"{case}.json"))
    out = json.loads(r.stdout)
    assert r.returncode == 0 and out["ok"] and out["errors"] == [], out


@pytest.mark.parametrize("overrides", [
    ["space.nx=0"],
    ["neighborhood=hexagonal", "space.ny=5"],
    ["boundary=reflecting"],
    ["mc.Q=1"],
    ["vents.count=0"],
    ["ca.maxSteps=-3"],
    ["terrain.type=file", "terrain.file=does/not/exist.csv"],
    ["mc.enabled=true", "mc.update=random"],
    ["unknownKey=1"],
])
def test_validate_rejects(overrides):
    args = ["--validate"]
    for o in overrides:
        args += ["--set", o]
    r = run(*args)
    out = json.loads(r.stdout)
    assert r.returncode == 1 and not out["ok"] and out["errors"], out


@pytest.mark.parametrize("args", [
    ["--bogus"],
    ["--print-defaults", "--validate"],
    ["--batch", "x", "--config", "y"],
    ["--set", "nokey"],
    ["--set"],
    ["--threads", "-2"],
    ["--validate", "--progress"],
])
def test_argument_errors(args):
    r = run(*args)
    assert r.returncode == 2
    assert r.stderr.startswith("Błąd argumentów: ")


def test_config_error_exit_code(tmp_path):
    r = run("--config", os.path.join(GOLDEN, "cases", "lava2d_moore.json"), "--set", "space.nz=0", "--out",
            str(tmp_path / "o"))
    assert r.returncode == 1
    assert r.stderr.startswith("Błąd konfiguracji: ")


def test_mc_from_missing_folder(tmp_path):
    r = run("--validate", "--mc-from", str(tmp_path / "none"), "--config",
            os.path.join(GOLDEN, "cases", "mcfrom_lava2d.json"))
    out = json.loads(r.stdout)
    assert r.returncode == 1 and any("--mc-from" in e for e in out["errors"])


def test_batch_empty_folder(tmp_path):
    r = run("--batch", str(tmp_path), "--out", str(tmp_path / "out"))
    assert r.returncode == 1
    assert r.stderr.startswith("Błąd konfiguracji: ")


def test_validation_messages_equal_reference():
    """--validate on configs the reference refuses or warns about: the same exit code and the same
    error and warning texts, word for word (tests/golden/config_errors.json, made by make_golden.py
    --config-errors from the reference engine; engine/src/io/Config.cpp:20-437)."""
    with open(os.path.join(GOLDEN, "config_errors.json")) as f:
        cases = json.load(f)
    for case in cases:
        args = ["--validate"]
        for kv in case["set"]:
            args += ["--set", kv]
        r = run(*args)
        out = json.loads(r.stdout)
        assert (r.returncode, out["errors"], out["warnings"]) == (case["exit"], case["errors"], case["warnings"]), case


def test_number_overflow_in_a_config_file(tmp_path):
    """A literal beyond the double range in a config file is the reference's JSON range error, word
    for word and not wrapped as a syntax error: listed by --validate, and in a run the generic error
    (exit 3, prefix "Błąd: "), as the reference engine gives it for the same file."""
    cfg = tmp_path / "overflow.json"
    cfg.write_text('{"mc": {"kT": 1e400}}')
    text = "[json.exception.out_of_range.406] number overflow parsing '1e400'"
    r = run("--validate", "--config", str(cfg))
    assert r.returncode == 1 and json.loads(r.stdout)["errors"] == [text]
    r = run("--config", str(cfg), "--out", str(tmp_path / "out"))
    assert r.returncode == 3 and r.stderr.strip() == "Błąd: " + text


def test_refused_command_lines_equal_reference(tmp_path):
    """Command lines refused before any simulation work: the exit code and the message line are the
    reference engine's, word for word, and --validate's report too (tests/golden/cli_errors.json, made
    by make_golden.py --cli-errors; engine/src/app/Cli.cpp, Batch.cpp, ConfigCheck.cpp).  After an
    argument error both engines print their usage text, which differs: this engine lists --serve."""
    (tmp_path / "c.json").write_text('{"space": {"nx": 40, "ny": 1, "nz": 30}}')
    (tmp_path / "empty").mkdir()
    with open(os.path.join(GOLDEN, "cli_errors.json")) as f:
        cases = json.load(f)
    d = str(tmp_path)
    for case in cases:
        r = run(*[a.replace("{d}", d) for a in case["args"]], cwd=d)
        first = (r.stderr.strip().splitlines() or [""])[0].replace(d, "{d}")
        assert (r.returncode, first) == (case["exit"], case["stderr_first_line"]), case["args"]
        if case["stdout"] is not None:
            assert json.loads(r.stdout.replace(d, "{d}")) == json.loads(case["stdout"]), case["args"]
