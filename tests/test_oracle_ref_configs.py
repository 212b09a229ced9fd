"""Pins the CPU oracle to the reference engine run on the reference's own config files
(tests/golden/ref_<name>, made by ``make_golden.py --ref-configs`` from configs/*.json of the
reference: the cone, file-heightmap and real-DEM lava cases, the classic case, the whole-space MC
cases, and the MC-only config run with --mc-from).  The merged config is the engine's own
config_used.json.  From the reference's step-0 state the oracle's CA run must give its
ca_result.bin byte for byte, its step count, stop reason and per-step histories; its Potts sweeps
must give mc_result.bin, mc_stats.csv and the attempt counters.

CPU only: with tests/test_oracle_pin.py this is what makes the oracle a trustworthy checker.
"""
from __future__ import annotations

import functools
import json
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_pin import STOP_TEXT, check_mc_rows, crystal_bytes, oracle_ca, oracle_mc, sha

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CA_CONFIGS = ["test_2d", "test_3d", "lava_mc_2d", "lava_mc_3d", "heightmap_kaldera", "heightmap_kanion",
              "heightmap_podwojny", "etna_3d", "etna_real", "etna_real_boczna", "wezuwiusz_real", "classic_ref"]


def load(name):
    d = os.path.join(GOLDEN, f"ref_{name}")
    with open(os.path.join(d, "config_used.json")) as f:
        used = json.load(f)
    with open(os.path.join(d, "expect.json")) as f:
        exp = json.load(f)
    return {"_used": used}, exp


def initial(name) -> O.CaState:
    z = np.load(os.path.join(GOLDEN, f"ref_{name}", "initial.npz"))
    nx, ny, nz = (int(v) for v in z["dims"])
    return O.CaState(nx, ny, nz, z["type"].astype(np.uint8), z["flow"].astype(np.int32),
                     z["temp"].astype(np.float32), z["solid"].astype(np.uint16), z["arrival"].astype(np.uint16))


@functools.lru_cache(maxsize=1)
def ca_runs() -> dict:
    """The oracle's CA run of every config, once per session, side by side on the host cores (the
    oracle steps in C with the interpreter lock released; the three 1.6-1.8 M-cell DEM cases take
    half a minute each)."""
    def run(name):
        cfg, _ = load(name)
        return name, oracle_ca(cfg, initial(name))
    O.lib()  # loaded once, before the threads share it
    with ThreadPoolExecutor(max_workers=max(1, min(len(CA_CONFIGS), os.cpu_count() or 1))) as ex:
        return dict(ex.map(run, sorted(CA_CONFIGS, key=lambda n: n.startswith("etna"), reverse=True)))


def check_mc(used, exp, dims, spin, rows, totals, domain):
    assert sha(crystal_bytes(dims, spin)) == exp["files"]["mc_result.bin"]
    check_mc_rows(exp["mc_stats_csv"], rows)
    mc = exp["stats"]["mc"]
    assert [int(t) for t in totals] == [mc["attempts"], mc["accepted"], mc["acceptedUphill"]]
    assert int(domain.sum()) == mc["domainCells"]


def mc_on(used, s: O.CaState):
    dom = O.basalt_domain(s)
    mob = O.mobility_from_cooling(s, dom, used["mc"]["mobilityMin"]) if used["mc"]["mobilityFromCooling"] else None
    return dom, oracle_mc(used["mc"], used, (s.nx, s.ny, s.nz), dom, mob, False)


@pytest.mark.parametrize("name", CA_CONFIGS)
def test_oracle_matches_reference_config(name):
    cfg, exp = load(name)
    s, steps, stop, act, chg = ca_runs()[name]
    st = exp["stats"]
    assert (steps, STOP_TEXT[stop]) == (st["steps"], st["stopReason"])
    assert act == st["activeCells"] and chg == st["changedCells"]
    assert sha(s.to_bytes()) == exp["files"]["ca_result.bin"]
    used = cfg["_used"]
    if used["mc"]["enabled"]:
        dom, (spin, rows, totals) = mc_on(used, s)
        check_mc(used, exp, (s.nx, s.ny, s.nz), spin, rows, totals, dom)


@pytest.mark.parametrize("name", ["mc_full_2d", "mc_full_3d"])
def test_oracle_matches_reference_full_domain_config(name):
    cfg, exp = load(name)
    used = cfg["_used"]
    dims = (used["space"]["nx"], used["space"]["ny"], used["space"]["nz"])
    dom = np.ones(dims[0] * dims[1] * dims[2], np.uint8)
    spin, rows, totals = oracle_mc(used["mc"], used, dims, dom, None, True)
    check_mc(used, exp, dims, spin, rows, totals, dom)


def test_oracle_matches_reference_mc_only_config():
    """configs/mc_basalt.json with --mc-from the lava_mc_3d result: Potts sweeps on the oracle's CA
    result of that config, with the MC config's own neighbourhood, seed and parameters."""
    s, *_ = ca_runs()["lava_mc_3d"]
    cfg, exp = load("mc_basalt")
    used = cfg["_used"]
    dom, (spin, rows, totals) = mc_on(used, s)
    check_mc(used, exp, (s.nx, s.ny, s.nz), spin, rows, totals, dom)
