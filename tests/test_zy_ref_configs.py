"""The CUDA path on the reference's own config files (tests/golden/ref_<name>, made by
``make_golden.py --ref-configs`` from configs/*.json of the reference).  From the reference's step-0
state, through the C ABI, the CA run must give the reference engine's ca_result.bin byte for byte,
its step count, stop reason and per-step histories; the Potts sweeps on that result (or on a whole
space) its mc_result.bin, final energy and attempt counters.  The inputs are the oracle's in
tests/test_oracle_ref_configs.py: the spill levels from the state's ROCK columns, the vents from its
LAVA cells, the parameters from the engine's config_used.json (their mapping onto the C ABI is
checked against the oracle's on the CPU).
"""
from __future__ import annotations

import csv
import io

import numpy as np
import pytest

from oracle import oracle as O
from tests import cases as C
from tests.test_oracle_pin import STOP_TEXT, ca_params, crystal_bytes, sha
from tests.test_oracle_ref_configs import CA_CONFIGS, initial, load
from volcano_ca_mc_b200 import capi


def capi_params(used, s: O.CaState) -> capi.CaParams:
    ca, v = used["ca"], used["vents"]
    return capi.CaParams(s.nx, s.ny, s.nz, neighborhood=used["neighborhood"], boundary=used["boundary"],
                         mode=ca["mode"], seed=used["rngSeed"], max_steps=ca["maxSteps"],
                         eruption_steps=v["eruptionSteps"], erupt_temp=v["eruptTemp"], solidus_temp=ca["solidusTemp"],
                         cooling_ambient=ca["coolingAmbient"], cooling_lateral=ca["coolingLateral"],
                         cooling_fall=ca["coolingFall"], ponding=bool(ca["ponding"]))


def spill_and_vents(used, s: O.CaState):
    """The spill levels and vent table the oracle's run takes (tests/test_oracle_pin.py oracle_ca)."""
    per = used["boundary"] == "periodic"
    spill = None
    if used["ca"]["mode"] != "classic":
        spill = O.fill_depressions(O.heights_from_state(s), s.nx, s.ny, per and s.nx > 1, per and s.ny > 1)
    idx = np.nonzero(s.type == O.LAVA)[0]
    vents = [(int(i % s.nx), int((i // s.nx) % s.ny), int(i // (s.nx * s.ny)), int(s.flow[i])) for i in idx]
    return spill, vents


def mc_params(used, dims, full: bool) -> capi.McParams:
    m = used["mc"]
    return capi.McParams(*dims, neighborhood=used["neighborhood"], boundary=used["boundary"], domain_full=full,
                         seed=used["rngSeed"], Q=m["Q"], J=m["J"], kT=m["kT"])


def check_mc(mc: capi.PottsMC, exp, dims):
    assert sha(crystal_bytes(dims, mc.crystals())) == exp["files"]["mc_result.bin"]
    info = mc.info()
    ref = exp["stats"]["mc"]
    assert (info.attempts, info.accepted, info.uphill) == (ref["attempts"], ref["accepted"], ref["acceptedUphill"])
    assert info.domain_cells == ref["domainCells"]
    last = list(csv.DictReader(io.StringIO(exp["mc_stats_csv"])))[-1]
    assert f"{mc.energy():.3f}" == last["energy"]


def ca_run(name):
    cfg, exp = load(name)
    used = cfg["_used"]
    s0 = initial(name)
    spill, vents = spill_and_vents(used, s0)
    ca = capi.LavaCA(capi_params(used, s0))
    ca.set_state(s0.type, s0.flow, s0.temp, s0.solid, s0.arrival, spill, vents, steps_done=0)
    ca.run()
    return ca, used, exp, s0


def mc_after(ca: capi.LavaCA, used, dims) -> capi.PottsMC:
    """McStage on the CA handle: domain and cooling mobility from the device, mcs sweeps."""
    m = used["mc"]
    mc = capi.PottsMC(mc_params(used, dims, False))
    mc.set_domain_from_ca(ca)
    mc.set_mobility_from_ca(ca, m["mobilityMin"], bool(m["mobilityFromCooling"]))
    mc.initialize()
    mc.sweep(m["mcs"])
    return mc


@pytest.mark.parametrize("name", CA_CONFIGS)
def test_capi_params_are_the_oracles(name):
    """CPU: the C ABI parameters built from config_used.json are, field by field, the oracle's."""
    cfg, _ = load(name)
    s0 = initial(name)
    got, want = C.oracle_params(capi_params(cfg["_used"], s0)), ca_params(cfg, s0)
    for field, _ in want._fields_:
        assert getattr(got, field) == getattr(want, field), field


@pytest.mark.gpu
@pytest.mark.parametrize("name", CA_CONFIGS)
def test_cuda_path_matches_reference_config(name):
    ca, used, exp, s0 = ca_run(name)
    info = ca.info()
    st = exp["stats"]
    assert (info.steps, STOP_TEXT[info.stop_reason]) == (st["steps"], st["stopReason"])
    act, chg = ca.history()
    assert act == st["activeCells"] and chg == st["changedCells"]
    planes = ca.download()
    state = O.CaState(s0.nx, s0.ny, s0.nz, *planes)
    assert sha(state.to_bytes()) == exp["files"]["ca_result.bin"]
    if used["mc"]["enabled"]:
        mc = mc_after(ca, used, (s0.nx, s0.ny, s0.nz))
        check_mc(mc, exp, (s0.nx, s0.ny, s0.nz))
        mc.close()
    ca.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["mc_full_2d", "mc_full_3d"])
def test_cuda_path_matches_reference_full_domain_config(name):
    cfg, exp = load(name)
    used = cfg["_used"]
    dims = (used["space"]["nx"], used["space"]["ny"], used["space"]["nz"])
    mc = capi.PottsMC(mc_params(used, dims, True))
    mc.set_domain(None)
    mc.initialize()
    mc.sweep(used["mc"]["mcs"])
    check_mc(mc, exp, dims)
    mc.close()


@pytest.mark.gpu
def test_cuda_path_matches_reference_mc_only_config():
    """configs/mc_basalt.json with --mc-from the lava_mc_3d result: MC with the MC config's own
    neighbourhood, seed and parameters on the CA handle of lava_mc_3d."""
    ca, _, _, s0 = ca_run("lava_mc_3d")
    cfg, exp = load("mc_basalt")
    mc = mc_after(ca, cfg["_used"], (s0.nx, s0.ny, s0.nz))
    check_mc(mc, exp, (s0.nx, s0.ny, s0.nz))
    mc.close()
    ca.close()
