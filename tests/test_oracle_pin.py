"""Pins the CPU oracle to the reference engine's own outputs (tests/golden, made by
tests/golden/make_golden.py from the reference engine): starting from the reference's initial
state of each case, the oracle's CA run must give the reference's ca_result.bin byte for byte,
the same step count, stop reason and per-step active/changed histories; its Potts sweeps on that
result must give the reference's mc_result.bin, energies (mc_stats.csv) and attempt counters.

CPU only (no GPU): this is what makes the oracle a trustworthy checker for the GPU tests.
"""
from __future__ import annotations

import csv
import hashlib
import io
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STOP_TEXT = {1: "brak płynnej lawy", 2: "brak wolnych komórek (AIR)", 3: "brak zmian w kroku",
             4: "osiągnięto ca.maxSteps"}


def load_case(name):
    with open(os.path.join(GOLDEN, "cases", f"{name}.json")) as f:
        cfg = json.load(f)
    with open(os.path.join(GOLDEN, name, "expect.json")) as f:
        exp = json.load(f)
    return cfg, exp


def initial_state(name) -> O.CaState:
    z = np.load(os.path.join(GOLDEN, name, "initial.npz"))
    nx, ny, nz = (int(v) for v in z["dims"])
    return O.CaState(nx, ny, nz, z["type"].astype(np.uint8), z["flow"].astype(np.int32),
                     z["temp"].astype(np.float32), z["solid"].astype(np.uint16), z["arrival"].astype(np.uint16))


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def crystal_bytes(dims, spin) -> bytes:
    return b"VMC1" + np.array(dims, "<i4").tobytes() + spin.astype("<i4").tobytes()


def ca_params(cfg, s: O.CaState) -> O.CaParams:
    used = cfg["_used"]
    ca, v = used["ca"], used["vents"]
    return O.CaParams(s.nx, s.ny, s.nz, O.NB[used["neighborhood"]], int(used["boundary"] == "periodic"),
                      int(ca["mode"] == "classic"), used["rngSeed"], ca["maxSteps"], v["eruptionSteps"],
                      v["eruptTemp"], ca["solidusTemp"], ca["coolingAmbient"], ca["coolingLateral"],
                      ca["coolingFall"], int(ca["ponding"]))


def oracle_ca(cfg, s0: O.CaState):
    """LavaCA from the initial state: spill levels from the initial terrain, vent table from the seeds."""
    p = ca_params(cfg, s0)
    per = cfg["_used"]["boundary"] == "periodic"
    spill = None
    if not p.classic:
        spill = O.fill_depressions(O.heights_from_state(s0), s0.nx, s0.ny, per and s0.nx > 1, per and s0.ny > 1)
    idx = np.nonzero(s0.type == O.LAVA)[0]
    vents = [(int(i % s0.nx), int((i // s0.nx) % s0.ny), int(i // (s0.nx * s0.ny)), int(s0.flow[i])) for i in idx]
    return O.ca_run(p, s0.copy(), spill, O.vent_table(vents))


def oracle_mc(mc_cfg, used, dims, domain, mobility, full: bool):
    """Checkerboard sweeps with the stats points of McStage::run: energy at MCS 0, every statsEvery
    and at the end; acceptance rate over the sweeps since the previous point."""
    nx, ny, nz = dims
    p = O.mc_params(nx, ny, nz, used["neighborhood"], used["boundary"], full, used["rngSeed"], mc_cfg["Q"],
                    mc_cfg["J"], mc_cfg["kT"])
    spin = O.mc_init(p, domain)
    rows = [(0, O.mc_energy(p, 0, spin), 0.0)]
    totals = np.zeros(3, np.uint64)
    window = np.zeros(3, np.uint64)
    mcs, every = mc_cfg["mcs"], mc_cfg["statsEvery"]
    for k in range(mcs):
        c = O.mc_sweep(p, k, domain, mobility, spin)
        totals += c
        window += c
        if (k + 1) % every == 0 or k + 1 == mcs:
            rate = float(window[1]) / float(window[0]) if window[0] else 0.0
            rows.append((k + 1, O.mc_energy(p, k + 1, spin), rate))
            window[:] = 0
    return spin, rows, totals


def check_mc_rows(exp_csv: str, rows):
    got = list(csv.DictReader(io.StringIO(exp_csv)))
    assert [int(r["mcs"]) for r in got] == [r[0] for r in rows]
    for g, (mcs, energy, rate) in zip(got, rows):
        assert g["energy"] == f"{energy:.3f}", (mcs, g["energy"], energy)
        assert g["acceptRate"] == f"{rate:.6f}", (mcs, g["acceptRate"], rate)


def with_used(name):
    cfg, exp = load_case(name)
    # the reference merges each case over its defaults (engine --print-defaults); the keys the oracle
    # needs are merged here the same way
    cfg["_used"] = merged(cfg)
    return cfg, exp


DEFAULTS = {
    "boundary": "absorbing", "neighborhood": "moore", "rngSeed": 42,
    "vents": {"count": 1, "placement": "crater", "eruptionSteps": 300, "eruptTemp": 1200},
    "ca": {"mode": "lava", "maxSteps": 5000, "coolingAmbient": 0.3, "coolingLateral": 1.5, "coolingFall": 0.1,
           "solidusTemp": 800, "ponding": True},
    "mc": {"enabled": False, "domain": "basalt", "Q": 50, "mcs": 100, "J": 1.0, "kT": 0.0,
           "mobilityFromCooling": True, "mobilityMin": 0.05, "statsEvery": 10},
}


def merged(cfg):
    out = {}
    for k, v in DEFAULTS.items():
        out[k] = dict(v) if isinstance(v, dict) else v
    for k, v in cfg.items():
        if isinstance(v, dict) and isinstance(out.get(k), dict):
            out[k].update(v)
        else:
            out[k] = v
    return out


CA_CASES = ["lava2d_moore", "lava2d_hex_periodic", "lava3d_moore_random", "lava3d_pent_periodic", "lava3d_vn_odd",
            "heightmap_file", "classic3d_moore", "classic2d_vn"]


@pytest.mark.parametrize("name", CA_CASES)
def test_oracle_matches_reference_engine(name):
    cfg, exp = with_used(name)
    s, steps, stop, act, chg = oracle_ca(cfg, initial_state(name))
    st = exp["stats"]
    assert steps == st["steps"]
    assert STOP_TEXT[stop] == st["stopReason"]
    assert act == st["activeCells"]
    assert chg == st["changedCells"]
    if "ca_result.bin" in exp["files"]:
        assert sha(s.to_bytes()) == exp["files"]["ca_result.bin"]
    used = cfg["_used"]
    if used["mc"]["enabled"]:
        dom = O.basalt_domain(s)
        mob = None
        if used["mc"]["mobilityFromCooling"]:
            mob = O.mobility_from_cooling(s, dom, used["mc"]["mobilityMin"])
        spin, rows, totals = oracle_mc(used["mc"], used, (s.nx, s.ny, s.nz), dom, mob, False)
        assert sha(crystal_bytes((s.nx, s.ny, s.nz), spin)) == exp["files"]["mc_result.bin"]
        check_mc_rows(exp["mc_stats_csv"], rows)
        mc = st["mc"]
        assert [int(t) for t in totals] == [mc["attempts"], mc["accepted"], mc["acceptedUphill"]]
        assert int(dom.sum()) == mc["domainCells"]


@pytest.mark.parametrize("name", ["mc_full_3d", "mc_full_2d_hex"])
def test_oracle_full_domain_matches_reference_engine(name):
    cfg, exp = with_used(name)
    used = cfg["_used"]
    sp = cfg["space"]
    dims = (sp["nx"], sp["ny"], sp["nz"])
    dom = np.ones(dims[0] * dims[1] * dims[2], np.uint8)
    spin, rows, totals = oracle_mc(used["mc"], used, dims, dom, None, True)
    assert sha(crystal_bytes(dims, spin)) == exp["files"]["mc_result.bin"]
    check_mc_rows(exp["mc_stats_csv"], rows)
    mc = exp["stats"]["mc"]
    assert [int(t) for t in totals] == [mc["attempts"], mc["accepted"], mc["acceptedUphill"]]
    assert mc["colors"] == O.mc_colors(O.mc_params(*dims, used["neighborhood"], used["boundary"], True,
                                                   used["rngSeed"], 2, 1.0, 0.0))


def test_oracle_mc_from_file_matches_reference_engine():
    """--mc-from: MC on a CA result read back from ca_result.bin (version 2: cooling data included)."""
    src_cfg, _ = with_used("lava2d_moore")
    s, *_ = oracle_ca(src_cfg, initial_state("lava2d_moore"))
    cfg, exp = with_used("mcfrom_lava2d")
    used = cfg["_used"]
    dom = O.basalt_domain(s)
    mob = O.mobility_from_cooling(s, dom, used["mc"]["mobilityMin"])
    spin, rows, totals = oracle_mc(used["mc"], used, (s.nx, s.ny, s.nz), dom, mob, False)
    assert sha(crystal_bytes((s.nx, s.ny, s.nz), spin)) == exp["files"]["mc_result.bin"]
    check_mc_rows(exp["mc_stats_csv"], rows)


def test_oracle_matches_reference_engine_c1_workload():
    """The 512 x 1 x 256 cross-section workload (volcano_ca_mc_b200.workloads.c1) at its full size:
    the oracle's CA run from the heightmap and vents of the workload, and its 50 Potts sweeps, give the
    reference engine's ca_result.bin / mc_result.bin hashes, histories and MC counters
    (tests/golden/c1_large, made by make_golden.py --large c1)."""
    from volcano_ca_mc_b200 import workloads
    from tests import cases as C

    w = workloads.get("c1")
    with open(os.path.join(GOLDEN, "c1_large", "expect.json")) as f:
        exp = json.load(f)
    s0 = C.initial_state(w.nx, w.ny, w.nz, w.heights, w.vent_cells(), 1200.0)
    p = O.CaParams(w.nx, w.ny, w.nz, O.NB[w.neighborhood], int(w.boundary == "periodic"), 0, w.seed, w.max_steps, 300,
                   1200.0, 800.0, 0.3, 1.5, 0.1, 1)
    spill = O.fill_depressions(w.heights, w.nx, w.ny, False, False)
    s, steps, stop, act, chg = O.ca_run(p, s0, spill, O.vent_table(w.vent_cells()))
    assert steps == exp["steps"] and STOP_TEXT[stop] == exp["stopReason"]
    assert act == exp["activeCells"] and chg == exp["changedCells"]
    assert sha(s.to_bytes()) == exp["files"]["ca_result.bin"]
    dom = O.basalt_domain(s)
    mob = O.mobility_from_cooling(s, dom, 0.05)
    used = {"neighborhood": w.neighborhood, "boundary": w.boundary, "rngSeed": w.seed}
    spin, rows, totals = oracle_mc({"Q": w.Q, "J": 1.0, "kT": w.kT, "mcs": w.mcs, "statsEvery": w.mcs}, used,
                                   (w.nx, w.ny, w.nz), dom, mob, False)
    assert sha(crystal_bytes((w.nx, w.ny, w.nz), spin)) == exp["files"]["mc_result.bin"]
    check_mc_rows(exp["mc_stats_csv"], rows)
    mc = exp["mc"]
    assert [int(t) for t in totals] == [mc["attempts"], mc["accepted"], mc["acceptedUphill"]]
    assert int(dom.sum()) == mc["domainCells"]
