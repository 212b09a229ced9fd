"""The benchmark workloads at their full sizes on the GPU against the reference engine's own runs of
the same configs (tests/golden/<name>_large, hashes made by make_golden.py --large):
  c1  512 x 1 x 256 cross-section, Moore, absorbing, 300 steps, 50 Potts sweeps with Q = 64;
  c2  256 x 256 x 128, Moore, periodic, 400 steps, 100 sweeps with Q = 128;
  c3  1024 x 1024 x 256 = 268 M cells, random pentagonal neighbourhood, 800 steps, 200 sweeps with Q = 256.
Checked: the bytes of ca_result.bin and mc_result.bin, every step's active/changed counts, the MC
counters and energies.  The DENSE schedule must give the same bytes as the ACTIVE one."""
from __future__ import annotations

import hashlib
import json
import os
import struct

import numpy as np
import pytest

from volcano_ca_mc_b200 import capi, workloads

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["c1", "c2", "c3"]


def ca_bin_sha(w, planes) -> str:
    h = hashlib.sha256(b"VOLC" + struct.pack("<Iiii", 2, w.nx, w.ny, w.nz))
    for p in planes:
        h.update(memoryview(np.ascontiguousarray(p)).cast("B"))
    return h.hexdigest()


def run_ca(w, sweep):
    ca = capi.LavaCA(capi.CaParams(w.nx, w.ny, w.nz, neighborhood=w.neighborhood, boundary=w.boundary, seed=w.seed,
                                   max_steps=w.max_steps, sweep=sweep))
    ca.apply_terrain(w.heights)
    ca.place_seeds(w.vent_cells())
    ca.run()
    return ca


def expect_of(name):
    with open(os.path.join(GOLDEN, f"{name}_large", "expect.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", NAMES)
def test_large_ca_and_mc_match_reference(name):
    expect, w = expect_of(name), workloads.get(name)
    ca = run_ca(w, capi.SWEEP_ACTIVE)
    info = ca.info()
    assert info.steps == expect["steps"]
    act, chg = ca.history()
    assert act == expect["activeCells"]
    assert chg == expect["changedCells"]
    planes = ca.download()
    assert ca_bin_sha(w, planes) == expect["files"]["ca_result.bin"]
    del planes

    mc = capi.PottsMC(capi.McParams(w.nx, w.ny, w.nz, neighborhood=w.neighborhood, boundary=w.boundary,
                                    seed=w.seed, Q=w.Q, J=1.0, kT=w.kT))
    mc.set_domain_from_ca(ca)
    mc.set_mobility_from_ca(ca, 0.05, True)
    mc.initialize()
    e0 = mc.energy()
    mc.sweep(w.mcs)
    mi = mc.info()
    exp = expect["mc"]
    assert mi.domain_cells == exp["domainCells"]
    assert (mi.attempts, mi.accepted, mi.uphill) == (exp["attempts"], exp["accepted"], exp["acceptedUphill"])
    assert e0 == exp["energyStart"]
    assert mc.energy() == exp["energyEnd"]
    crystals = mc.crystals()
    h = hashlib.sha256(b"VMC1" + struct.pack("<iii", w.nx, w.ny, w.nz))
    h.update(memoryview(crystals).cast("B"))
    assert h.hexdigest() == expect["files"]["mc_result.bin"]
    mc.close()
    ca.close()


@pytest.mark.parametrize("name", NAMES)
def test_large_dense_schedule_same_bytes(name):
    expect, w = expect_of(name), workloads.get(name)
    ca = run_ca(w, capi.SWEEP_DENSE)
    assert ca.info().steps == expect["steps"]
    assert ca_bin_sha(w, ca.download()) == expect["files"]["ca_result.bin"]
    ca.close()
