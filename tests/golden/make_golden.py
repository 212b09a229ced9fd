"""Generates the golden fixtures under tests/golden/ by running the reference engine.

Run where the reference sources are at hand (the reference engine is built by
``make -C oracle ref REF=<reference checkout>`` into ``oracle/_ref/engine``):

    python tests/golden/make_golden.py                 # the small cases
    python tests/golden/make_golden.py --large         # hashes of the full-size 1024 x 1024 x 256 workload (c3)
    python tests/golden/make_golden.py --large c1 c2   # the same for the 512 x 1 x 256 and 256 x 256 x 128 workloads
    python tests/golden/make_golden.py --config-errors # the reference's validation messages for bad configs
    python tests/golden/make_golden.py --cli-errors    # its messages for refused command lines
    VCA_REFERENCE_DIR=<checkout> python tests/golden/make_golden.py --ref-configs
                                                       # the reference's own configs/*.json (ref_<name>/)

For every case in CASES it writes ``cases/<name>.json`` (the config, in the reference's schema),
runs ``engine --config cases/<name>.json --out <tmp>`` and stores under ``<name>/``:

* ``expect.json``: the SHA-256 of every result file, stats.json without its "parallel" section
  (thread counts of the machine that ran it), the text of mc_stats.csv, the section and info keys
  of times.json, the exit code;
* ``initial.npz`` (CA cases): the state after terrain and vents, i.e. the reference's
  ``snapshots/step_000000.bin``, which the CPU oracle tests start from.

The configs are small (seconds of reference CPU time) and the fixtures a few hundred KB in all.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402

CASES_DIR = os.path.join(HERE, "cases")

COOL_FAST = {"coolingAmbient": 2.0, "coolingLateral": 4.0, "coolingFall": 2.0, "solidusTemp": 800}

CASES: dict[str, dict] = {
    # 2D cross-section (x-z), Moore, absorbing frame, two crater vents, MC with cooling mobility, kT > 0
    "lava2d_moore": {
        "space": {"nx": 128, "ny": 1, "nz": 64}, "boundary": "absorbing", "neighborhood": "moore", "rngSeed": 7,
        "terrain": {"type": "cone", "peakHeight": 40, "baseRadius": 60, "craterRadius": 8, "craterDepth": 5,
                    "noise": 0.05, "file": None},
        "vents": {"count": 2, "placement": "crater", "eruptionSteps": 120, "eruptTemp": 1200},
        "ca": {"mode": "lava", "maxSteps": 3000, **COOL_FAST, "ponding": True},
        "mc": {"enabled": True, "domain": "basalt", "Q": 32, "mcs": 30, "J": 1.0, "kT": 0.6,
               "mobilityFromCooling": True, "mobilityMin": 0.05, "statsEvery": 5, "update": "checkerboard"},
        "output": {"format": "both", "snapshotsEvery": 0},
    },
    # 2D hexagonal neighbourhood, periodic in x, MC at kT = 0 without mobility
    "lava2d_hex_periodic": {
        "space": {"nx": 96, "ny": 1, "nz": 48}, "boundary": "periodic", "neighborhood": "hexagonal", "rngSeed": 11,
        "terrain": {"type": "cone", "peakHeight": 30, "baseRadius": 44, "craterRadius": 5, "craterDepth": 3,
                    "noise": 0.08, "file": None},
        "vents": {"count": 1, "placement": "crater", "eruptionSteps": 80, "eruptTemp": 1150},
        "ca": {"mode": "lava", "maxSteps": 3000, **COOL_FAST, "ponding": True},
        "mc": {"enabled": True, "domain": "basalt", "Q": 20, "mcs": 20, "J": 1.0, "kT": 0.0,
               "mobilityFromCooling": False, "statsEvery": 4, "update": "checkerboard"},
        "output": {"format": "bin", "snapshotsEvery": 0},
    },
    # 3D Moore, absorbing, three randomly placed vents on the flanks
    "lava3d_moore_random": {
        "space": {"nx": 40, "ny": 36, "nz": 24}, "boundary": "absorbing", "neighborhood": "moore", "rngSeed": 5,
        "terrain": {"type": "cone", "peakHeight": 16, "baseRadius": 22, "craterRadius": 3, "craterDepth": 2,
                    "noise": 0.1, "file": None},
        "vents": {"count": 3, "placement": "random", "eruptionSteps": 60, "eruptTemp": 1200},
        "ca": {"mode": "lava", "maxSteps": 3000, **COOL_FAST, "ponding": True},
        "mc": {"enabled": True, "domain": "basalt", "Q": 64, "mcs": 20, "J": 1.0, "kT": 0.5,
               "mobilityFromCooling": True, "mobilityMin": 0.1, "statsEvery": 5, "update": "checkerboard"},
        "output": {"format": "both", "snapshotsEvery": 0},
    },
    # 3D pentagonal, periodic in x and y, vents at given columns, no ponding
    "lava3d_pent_periodic": {
        "space": {"nx": 36, "ny": 28, "nz": 20}, "boundary": "periodic", "neighborhood": "pentagonal", "rngSeed": 9,
        "terrain": {"type": "cone", "peakHeight": 14, "baseRadius": 20, "craterRadius": 3, "craterDepth": 2,
                    "noise": 0.05, "file": None},
        "vents": {"count": 2, "placement": "positions", "positions": [[18, 14], [10, 8]], "eruptionSteps": 50,
                  "eruptTemp": 1200},
        "ca": {"mode": "lava", "maxSteps": 3000, **COOL_FAST, "ponding": False},
        "mc": {"enabled": True, "domain": "basalt", "Q": 16, "mcs": 15, "J": 1.0, "kT": 0.3,
               "mobilityFromCooling": True, "mobilityMin": 0.05, "statsEvery": 3, "update": "checkerboard"},
        "output": {"format": "bin", "snapshotsEvery": 0},
    },
    # 3D von Neumann, periodic with odd nx and ny (three checkerboard colour classes per axis), stopped
    # by ca.maxSteps
    "lava3d_vn_odd": {
        "space": {"nx": 33, "ny": 31, "nz": 20}, "boundary": "periodic", "neighborhood": "von_neumann",
        "rngSeed": 13,
        "terrain": {"type": "cone", "peakHeight": 14, "baseRadius": 18, "craterRadius": 3, "craterDepth": 2,
                    "noise": 0.05, "file": None},
        "vents": {"count": 2, "placement": "crater", "eruptionSteps": 200, "eruptTemp": 1200},
        "ca": {"mode": "lava", "maxSteps": 90, "coolingAmbient": 0.3, "coolingLateral": 1.5, "coolingFall": 0.1,
               "solidusTemp": 800, "ponding": True},
        "mc": {"enabled": True, "domain": "basalt", "Q": 8, "mcs": 12, "J": 1.0, "kT": 1.0,
               "mobilityFromCooling": True, "mobilityMin": 0.05, "statsEvery": 4, "update": "checkerboard"},
        "output": {"format": "bin", "snapshotsEvery": 0},
    },
    # terrain from a CSV heightmap, step snapshots, text output, CA only
    "heightmap_file": {
        "space": {"nx": 48, "ny": 40, "nz": 24}, "boundary": "absorbing", "neighborhood": "moore", "rngSeed": 21,
        "terrain": {"type": "file", "file": "heightmaps/ridge_48x40.csv"},
        "vents": {"count": 1, "placement": "positions", "positions": [[14, 20]], "eruptionSteps": 70,
                  "eruptTemp": 1200},
        "ca": {"mode": "lava", "maxSteps": 3000, **COOL_FAST, "ponding": True},
        "mc": {"enabled": False},
        "output": {"format": "txt", "snapshotsEvery": 25},
    },
    # classic grain growth in 3D (no terrain), Moore, periodic
    "classic3d_moore": {
        "space": {"nx": 24, "ny": 24, "nz": 24}, "boundary": "periodic", "neighborhood": "moore", "rngSeed": 3,
        "vents": {"count": 12}, "ca": {"mode": "classic", "maxSteps": 65535}, "mc": {"enabled": False},
        "output": {"format": "bin", "snapshotsEvery": 0},
    },
    # classic grain growth in 2D (x-y plane), von Neumann, absorbing
    "classic2d_vn": {
        "space": {"nx": 64, "ny": 48, "nz": 1}, "boundary": "absorbing", "neighborhood": "von_neumann",
        "rngSeed": 17, "vents": {"count": 20}, "ca": {"mode": "classic", "maxSteps": 65535},
        "mc": {"enabled": False}, "output": {"format": "both", "snapshotsEvery": 0},
    },
    # Potts MC on the whole 3D space (no CA), periodic, kT > 0, MC snapshots
    "mc_full_3d": {
        "space": {"nx": 24, "ny": 20, "nz": 16}, "boundary": "periodic", "neighborhood": "moore", "rngSeed": 42,
        "mc": {"enabled": True, "domain": "full", "Q": 16, "mcs": 10, "J": 1.0, "kT": 0.5,
               "mobilityFromCooling": False, "statsEvery": 2, "snapshotsEvery": 5, "update": "checkerboard"},
        "output": {"format": "both"},
    },
    # Potts MC on the whole 2D space, hexagonal, absorbing, kT = 0
    "mc_full_2d_hex": {
        "space": {"nx": 64, "ny": 1, "nz": 40}, "boundary": "absorbing", "neighborhood": "hexagonal", "rngSeed": 8,
        "mc": {"enabled": True, "domain": "full", "Q": 10, "mcs": 8, "J": 1.0, "kT": 0.0,
               "mobilityFromCooling": False, "statsEvery": 2, "update": "checkerboard"},
        "output": {"format": "bin"},
    },
}

# --mc-from runs: MC on the CA result of another case, read back from its result folder.
MC_FROM: dict[str, tuple[str, dict]] = {
    "mcfrom_lava2d": ("lava2d_moore", {
        "boundary": "absorbing", "neighborhood": "moore", "rngSeed": 7,
        "mc": {"enabled": True, "domain": "basalt", "Q": 24, "mcs": 10, "J": 1.0, "kT": 0.4,
               "mobilityFromCooling": True, "mobilityMin": 0.2, "statsEvery": 5, "update": "checkerboard"},
        "output": {"format": "bin"},
    }),
}

RESULT_FILES = ("ca_result.bin", "ca_result.txt", "mc_result.bin", "mc_result.txt", "mc_stats.csv",
                "config_used.json")


def ridge_heightmap(nx: int, ny: int) -> str:
    """A ridge along y with a bowl on its west flank, heights in cells (plain arithmetic, no noise)."""
    rows = ["# ridge with a bowl, heights in cells"]
    for y in range(ny):
        vals = []
        for x in range(nx):
            ridge = 16.0 * math.exp(-((x - 30) / 9.0) ** 2)
            bowl = 4.0 * math.exp(-(((x - 14) / 5.0) ** 2 + ((y - 20) / 6.0) ** 2))
            h = max(0.0, 2.0 + ridge + 0.05 * y - bowl)
            vals.append(f"{h:.2f}")
        rows.append(",".join(vals))
    return "\n".join(rows) + "\n"


def sha256(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def write_case(name: str, cfg: dict) -> str:
    path = os.path.join(CASES_DIR, f"{name}.json")
    with open(path, "w") as f:
        json.dump(cfg, f, indent=2)
        f.write("\n")
    return path


def expectation(out: str, rc: int) -> dict:
    exp: dict = {"exit": rc, "files": {}, "snapshots": {}}
    for name in RESULT_FILES:
        p = os.path.join(out, name)
        if os.path.exists(p):
            exp["files"][name] = sha256(p)
    for sub in ("snapshots", "mc_snapshots"):
        d = os.path.join(out, sub)
        if os.path.isdir(d):
            for fn in sorted(os.listdir(d)):
                exp["snapshots"][f"{sub}/{fn}"] = sha256(os.path.join(d, fn))
    with open(os.path.join(out, "stats.json")) as f:
        stats = json.load(f)
    stats.pop("parallel", None)
    exp["stats"] = stats
    csv = os.path.join(out, "mc_stats.csv")
    if os.path.exists(csv):
        with open(csv) as f:
            exp["mc_stats_csv"] = f.read()
    with open(os.path.join(out, "times.json")) as f:
        exp["times_keys"] = list(json.load(f).keys())
    return exp


def run_ref(args: list[str], cwd: str | None = None) -> int:
    r = subprocess.run([O.REF_ENGINE, *args], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, cwd=cwd)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
    return r.returncode


def save_initial(path: str, s: "O.CaState") -> None:
    np.savez_compressed(path, dims=np.array([s.nx, s.ny, s.nz], np.int32), type=s.type, flow=s.flow,
                        temp=s.temp, solid=s.solid, arrival=s.arrival)


def large(name: str = "c3") -> None:
    """A workload of volcano_ca_mc_b200.workloads at its full size (c1 512 x 1 x 256, c2 256 x 256 x 128,
    c3 1024 x 1024 x 256): the reference engine's outputs are too large to commit, so only their
    hashes, the step count, the per-step histories and the MC counters are kept
    (``<name>_large/expect.json``).  Seconds of CPU for c1 and c2, a few minutes for c3."""
    from volcano_ca_mc_b200 import workloads
    w = workloads.get(name)
    tmp = tempfile.mkdtemp(prefix="vca_golden_large_")
    try:
        cfg = w.write(tmp)
        out = os.path.join(tmp, "out")
        rc = run_ref(["--config", cfg, "--out", out, "--threads", str(os.cpu_count() or 1)])
        assert rc == 0
        with open(os.path.join(out, "stats.json")) as f:
            stats = json.load(f)
        with open(os.path.join(out, "mc_stats.csv")) as f:
            csv_text = f.read()
        exp = {"workload": name, "files": {n: sha256(os.path.join(out, n)) for n in ("ca_result.bin", "mc_result.bin")},
               "steps": stats["steps"], "stopReason": stats["stopReason"], "activeCells": stats["activeCells"],
               "changedCells": stats["changedCells"], "totalLavaVolume": stats["totalLavaVolume"],
               "liquidLava": stats["liquidLava"],
               "mc": {k: stats["mc"][k] for k in ("domainCells", "attempts", "accepted", "acceptedUphill", "energyStart",
                                                  "energyEnd", "grainsStart", "grainsEnd")},
               "mc_stats_csv": csv_text}
        dst = os.path.join(HERE, f"{name}_large")
        os.makedirs(dst, exist_ok=True)
        with open(os.path.join(dst, "expect.json"), "w") as f:
            json.dump(exp, f, indent=1)
            f.write("\n")
        print(name, "large ok")
    finally:
        shutil.rmtree(tmp)


# --set overrides that the reference's config validation refuses or warns about, one message each
# (engine/src/io/Config.cpp:20-437): the texts land in batch_summary.csv and in --validate output.
CONFIG_ERRORS: list[list[str]] = [
    ["space.nx=0"], ["space.nx=1.5"], ["space.nx=99999999999999999999"], ["space.nx=1", "space.ny=1"],
    ["space.nx=100000", "space.ny=100000", "space.nz=100"], ["neighborhood=hexagonal", "space.ny=5"],
    ["space.ny=5", "space.nz=1"], ["boundary=reflecting"], ["grid=tiles"], ["mc.Q=1"], ["mc.J=0"], ["mc.kT=-1"],
    ["vents.count=0"], ["ca.maxSteps=-3"], ["ca.ponding=1"], ["unknownKey=1"], ["ca.unknown=2"], ["space=5"],
    ["terrain.type=file"], ["terrain.file=5"], ["vents.positions=5"], ["vents.positions=[[1]]"],
    ["vents.positions=[[500,0]]"], ["vents.placement=positions"],
    ["vents.placement=positions", "vents.positions=[[1,0],[1,0]]", "vents.count=2"],
    ["vents.placement=positions", "vents.positions=[[1,0]]", "vents.count=2"], ["vents.eruptTemp=700"],
    ["ca.mode=classic", "mc.enabled=true"], ["ca.mode=classic", "vents.count=100000000", "space.nx=20", "space.nz=20"],
    ["vents.positions=[[1,0]]"], ["ca.mode=classic", "vents.placement=positions"],
    ["mc.enabled=true", "mc.domain=full", "mc.update=checkerboard"], ["output.format=png"], ["mc.statsEvery=0"],
    ["mc.domain=foo"], ["mc.mobilityMin=-1"], ["mc.mobilityMin=1.5"], ["vents.placement=xyz"], ["terrain.type=xyz"],
    ["terrain.peakHeight=-5"], ["terrain.baseRadius=0"], ["terrain.craterRadius=-1"], ["terrain.noise=-0.5"],
    ["output.snapshotsEvery=-1"], ["ca.coolingAmbient=-1"], ["ca.coolingLateral=-2"], ["ca.coolingFall=-0.1"],
    ["ca.solidusTemp=-5"], ["ca.solidusTemp=2000"], ["rngSeed=-1"], ["rngSeed=1.5"], ["space.nz=0"],
    ["neighborhood=foo"], ["mc.update=foo"], ["mc.mcs=-1"], ["ca.sweep=foo"], ["grid=matrix"],
    ["parallel.threads=-2"], ["parallel.schedule=foo"], ["parallel.chunk=-1"], ["parallel.affinity=foo"],
    ["parallel.priority=foo"], ["mc.Q=100000"], ["mc.snapshotsEvery=-1"], ["vents.eruptionSteps=-1"],
    ["vents.count=-1"], ["ca.mode=foo"], ["mc.enabled=1"], ["output.format=bin", "output.snapshotsEvery=5"],
    ["terrain.type=flat"], ["space.nx=3", "space.nz=3"], ["vents.placement=random"], ["ca.maxSteps=70000"],
    ["ca.maxSteps=1.5"], ["boundary=periodic", "space.nx=1"], ["mc.J=-1"],
    ["mc.domain=full", "mc.enabled=true", "mc.update=checkerboard", "ca.mode=classic"], ["terrain.file=x.csv"],
    ["vents.positions=[[1,2,3]]"], ["space.ny=2", "neighborhood=hexagonal", "space.nz=1"],
    # number literals beyond the double range: an overflow is the JSON library's range error, an
    # underflow the nearest value
    ["mc.kT=1e400"], ["mc.kT=-1e400"], ["space.nx=1e400"], ["mc.kT=1e-400"],
]


def config_errors() -> None:
    """tests/golden/config_errors.json: the reference engine's --validate errors and warnings for
    each override set of CONFIG_ERRORS."""
    out = []
    for sets in CONFIG_ERRORS:
        args = ["--validate"]
        for kv in sets:
            args += ["--set", kv]
        r = subprocess.run([O.REF_ENGINE, *args], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
        res = json.loads(r.stdout)
        out.append({"set": sets, "exit": r.returncode, "errors": res["errors"], "warnings": res["warnings"]})
    with open(os.path.join(HERE, "config_errors.json"), "w") as f:
        json.dump(out, f, indent=1, ensure_ascii=False)
        f.write("\n")
    print("config_errors ok")


# The reference's own config files (configs/*.json of its checkout), run as they are (each takes
# under a second of reference CPU time); mc_basalt is the reference's MC-only config, run with
# --mc-from on the result of REF_MC_FROM's CA run.  Only the reference engine's outputs are kept:
# config_used.json (its merged config), the step-0 state and the hashes.
REF_CONFIGS = ["test_2d", "test_3d", "lava_mc_2d", "lava_mc_3d", "heightmap_kaldera", "heightmap_kanion",
               "heightmap_podwojny", "etna_3d", "etna_real", "etna_real_boczna", "wezuwiusz_real", "classic_ref",
               "mc_full_2d", "mc_full_3d"]
REF_MC_FROM = {"mc_basalt": "lava_mc_3d"}


def ref_configs() -> None:
    """tests/golden/ref_<name>/: the reference engine run on its own configs/<name>.json: expect.json
    (hashes, stats, mc_stats.csv), config_used.json (the engine's merged config) and, for a CA run,
    initial.npz (its step-0 snapshot).  The checkout is the working directory of each run: heightmap
    paths in the configs are relative to it."""
    ref = os.environ.get("VCA_REFERENCE_DIR", "")
    if not ref:
        sys.exit("set VCA_REFERENCE_DIR to the reference checkout")
    tmp = tempfile.mkdtemp(prefix="vca_golden_ref_")
    # bin results (the configs ask for txt too) and the GPU update (a config asking for the random
    # sequential update would be refused by bin/engine)
    over = ["--set", "output.format=bin", "--set", "mc.update=checkerboard"]

    def keep(name: str, out: str, source: str) -> None:
        dst = os.path.join(HERE, f"ref_{name}")
        os.makedirs(dst, exist_ok=True)
        exp = expectation(out, 0)
        exp["source"] = source
        # the generator's scratch folder (named by --mc-from runs) is not part of the fixture
        with open(os.path.join(dst, "expect.json"), "w") as f:
            f.write(json.dumps(exp, indent=1, ensure_ascii=False).replace(tmp, "<scratch>") + "\n")
        with open(os.path.join(out, "config_used.json")) as f:
            used = f.read()
        with open(os.path.join(dst, "config_used.json"), "w") as f:
            f.write(used.replace(tmp, "<scratch>"))

    try:
        outs = {}
        for name in REF_CONFIGS:
            src = os.path.join(ref, "configs", f"{name}.json")
            out = os.path.join(tmp, name)
            assert run_ref(["--config", src, "--out", out, *over], cwd=ref) == 0, name
            outs[name] = out
            keep(name, out, f"configs/{name}.json of the reference")
            with open(os.path.join(out, "config_used.json")) as f:
                used = json.load(f)
            if not (used["mc"]["enabled"] and used["mc"]["domain"] == "full"):
                init = os.path.join(tmp, name + "_init")
                assert run_ref(["--config", src, "--out", init, *over, "--set", "output.snapshotsEvery=65535",
                                "--set", "mc.enabled=false"], cwd=ref) == 0, name
                save_initial(os.path.join(HERE, f"ref_{name}", "initial.npz"),
                             O.read_ca_bin(os.path.join(init, "snapshots", "step_000000.bin")))
            print(name, "ok")
        for name, src_name in REF_MC_FROM.items():
            src = os.path.join(ref, "configs", f"{name}.json")
            out = os.path.join(tmp, name)
            assert run_ref(["--mc-from", outs[src_name], "--config", src, "--out", out, *over], cwd=ref) == 0, name
            keep(name, out, f"configs/{name}.json of the reference, --mc-from the result of ref_{src_name}")
            print(name, "ok")
    finally:
        shutil.rmtree(tmp)


# Command lines that the reference engine refuses before any simulation work (engine/src/app/Cli.cpp,
# Batch.cpp, ConfigCheck.cpp): "{d}" is a scratch folder holding one config, c.json.
CLI_ERRORS: list[list[str]] = [
    ["--out"], ["--config"], ["--frobnicate"], ["--threads", "abc", "--out", "{d}/o"],
    ["--threads", "-3", "--out", "{d}/o"], ["--batch", "{d}", "--config", "{d}/c.json"], ["--batch", "{d}", "--mc-from", "{d}"],
    ["--set"], ["--set", "novalue", "--validate"], ["--print-defaults", "--out", "{d}/o"],
    ["--mc-from", "{d}/nope", "--out", "{d}/o"], ["--config", "{d}/missing.json", "--out", "{d}/o"], ["--batch", "{d}/nope"],
    ["--threads"], ["--progress", "--validate"], ["--timing-detail", "--validate"], ["--set", "=5", "--validate"],
    ["positional"], ["--config", "{d}/c.json", "--batch", "{d}"], ["--validate", "--batch", "{d}"],
    ["--print-defaults", "--validate"], ["--validate", "--mc-from", "{d}/nope"], ["--validate", "--mc-from", "{d}"],
    ["--validate", "--mc-from", "{d}", "--set", "mc.domain=full"], ["--validate", "--config", "{d}/c.json", "--set", "terrain.type=file",
                                                                    "--set", "terrain.file={d}/nope.csv"],
    ["--batch", "{d}/empty", "--out", "{d}/o"],
]


def cli_errors() -> None:
    """tests/golden/cli_errors.json: the reference engine's exit code and first line of stderr (the
    message; its usage text follows argument errors) for each command line of CLI_ERRORS."""
    tmp = tempfile.mkdtemp(prefix="vca_golden_cli_")
    try:
        with open(os.path.join(tmp, "c.json"), "w") as f:
            f.write('{"space": {"nx": 40, "ny": 1, "nz": 30}}')
        os.makedirs(os.path.join(tmp, "empty"))
        out = []
        for args in CLI_ERRORS:
            real = [a.replace("{d}", tmp) for a in args]
            r = subprocess.run([O.REF_ENGINE, *real], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, cwd=tmp)
            first = (r.stderr.strip().splitlines() or [""])[0].replace(tmp, "{d}")
            stdout = r.stdout.replace(tmp, "{d}") if r.stdout.strip() else None  # --validate's report
            out.append({"args": args, "exit": r.returncode, "stderr_first_line": first, "stdout": stdout})
        with open(os.path.join(HERE, "cli_errors.json"), "w") as f:
            json.dump(out, f, indent=1, ensure_ascii=False)
            f.write("\n")
        print("cli_errors ok")
    finally:
        shutil.rmtree(tmp)


def main() -> None:
    if "--config-errors" in sys.argv:
        config_errors()
        return
    if "--cli-errors" in sys.argv:
        cli_errors()
        return
    if "--ref-configs" in sys.argv:
        ref_configs()
        return
    if "--large" in sys.argv:
        names = [a for a in sys.argv[sys.argv.index("--large") + 1:] if not a.startswith("-")] or ["c3"]
        for name in names:
            large(name)
        return
    if not os.path.exists(O.REF_ENGINE):
        ref = os.environ.get("VCA_REFERENCE_DIR", "")
        if not ref:
            sys.exit("the reference engine is not built: set VCA_REFERENCE_DIR to the reference checkout")
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={ref}"], check=True)
    os.makedirs(os.path.join(CASES_DIR, "heightmaps"), exist_ok=True)
    with open(os.path.join(CASES_DIR, "heightmaps", "ridge_48x40.csv"), "w") as f:
        f.write(ridge_heightmap(48, 40))
    tmp = tempfile.mkdtemp(prefix="vca_golden_")
    try:
        outs = {}
        for name, cfg in CASES.items():
            path = write_case(name, cfg)
            out = os.path.join(tmp, name)
            rc = run_ref(["--config", path, "--out", out])
            assert rc == 0, name
            outs[name] = out
            dst = os.path.join(HERE, name)
            os.makedirs(dst, exist_ok=True)
            with open(os.path.join(dst, "expect.json"), "w") as f:
                json.dump(expectation(out, rc), f, indent=1)
                f.write("\n")
            if not (cfg.get("mc", {}).get("enabled") and cfg["mc"].get("domain") == "full"):
                init = os.path.join(tmp, name + "_init")
                rc = run_ref(["--config", path, "--out", init, "--set", "output.snapshotsEvery=65535",
                              "--set", "mc.enabled=false", "--set", "output.format=bin"])
                assert rc == 0, name
                save_initial(os.path.join(dst, "initial.npz"),
                             O.read_ca_bin(os.path.join(init, "snapshots", "step_000000.bin")))
            print(name, "ok")
        for name, (src, cfg) in MC_FROM.items():
            path = write_case(name, cfg)
            out = os.path.join(tmp, name)
            rc = run_ref(["--mc-from", outs[src], "--config", path, "--out", out])
            assert rc == 0, name
            dst = os.path.join(HERE, name)
            os.makedirs(dst, exist_ok=True)
            exp = expectation(out, rc)
            exp["mc_from"] = src
            exp["stats"].pop("source", None)  # holds the absolute folder path of the run
            with open(os.path.join(dst, "expect.json"), "w") as f:
                json.dump(exp, f, indent=1)
                f.write("\n")
            print(name, "ok")
    finally:
        shutil.rmtree(tmp)


if __name__ == "__main__":
    main()
