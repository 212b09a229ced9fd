"""The full-size 3D workload (1024 x 1024 x 256 = 268 M cells, random pentagonal neighbourhood,
800 steps, then 200 Potts sweeps with Q = 256 on its basalt) on the GPU against the reference
engine's own run of the same config (tests/golden/c3_large, hashes made by make_golden.py --large):
the bytes of ca_result.bin and mc_result.bin, every step's active/changed counts, the MC counters
and energies.  The DENSE schedule must give the same bytes as the ACTIVE one."""
from __future__ import annotations

import hashlib
import json
import os
import struct

import numpy as np
import pytest

from volcano_ca_mc_b200 import capi, workloads

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c3_large", "expect.json")


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


@pytest.fixture(scope="module")
def expect():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def c3():
    return workloads.get("c3")


def test_large_ca_and_mc_match_reference(expect, c3):
    ca = run_ca(c3, capi.SWEEP_ACTIVE)
    info = ca.info()
    assert info.steps == expect["steps"]
    act, chg = ca.history()
    assert act == expect["activeCells"]
    assert chg == expect["changedCells"]
    planes = ca.download()
    assert ca_bin_sha(c3, planes) == expect["files"]["ca_result.bin"]
    del planes

    mc = capi.PottsMC(capi.McParams(c3.nx, c3.ny, c3.nz, neighborhood=c3.neighborhood, boundary=c3.boundary,
                                    seed=c3.seed, Q=c3.Q, J=1.0, kT=c3.kT))
    mc.set_domain_from_ca(ca)
    mc.set_mobility_from_ca(ca, 0.05, True)
    mc.initialize()
    e0 = mc.energy()
    mc.sweep(c3.mcs)
    mi = mc.info()
    exp = expect["mc"]
    assert mi.domain_cells == exp["domainCells"]
    assert (mi.attempts, mi.accepted, mi.uphill) == (exp["attempts"], exp["accepted"], exp["acceptedUphill"])
    assert e0 == exp["energyStart"]
    assert mc.energy() == exp["energyEnd"]
    crystals = mc.crystals()
    h = hashlib.sha256(b"VMC1" + struct.pack("<iii", c3.nx, c3.ny, c3.nz))
    h.update(memoryview(crystals).cast("B"))
    assert h.hexdigest() == expect["files"]["mc_result.bin"]
    mc.close()
    ca.close()


def test_large_dense_schedule_same_bytes(expect, c3):
    ca = run_ca(c3, capi.SWEEP_DENSE)
    assert ca.info().steps == expect["steps"]
    assert ca_bin_sha(c3, ca.download()) == expect["files"]["ca_result.bin"]
    ca.close()
