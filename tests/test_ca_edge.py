"""Edge cases of the lava CA rules on the GPU against the CPU oracle, bit for bit, from crafted states.

* Wide votes: CandidateVote (engine/src/ca/CaRules.hpp:127-183) holds any number of flowIds; the
  CUDA path keeps up to four in registers and recounts with room for 26 when a fifth distinct flowId
  shows up.  The states below put AIR cells at junctions of eight or more distinct flows, so every
  such cell takes the wide recount in the first step.
* The end of the step range: ca.maxSteps is at most 65535 (engine/src/io/Config.cpp) and the stamps
  solidStep / arrivalStep are uint16 (LavaCA.hpp:536-546, stamp = min(t, 65535)); a run resumed at
  t = 65525 writes stamps up to 65534 and stops with "ca.maxSteps" at 65535.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import cases as C
from volcano_ca_mc_b200 import capi

pytestmark = pytest.mark.gpu


def junction_state(nx, ny, nz):
    """ROCK floor at z = 0; at z = 1 LAVA everywhere except AIR at (x, y) with x % 3 == 1 and
    y % 3 == 1; at z = 2 LAVA straight above those AIR cells.  Every LAVA cell has its own flowId,
    so each AIR junction cell at z = 1 has eight distinct same-level sources and one falling from above."""
    n = nx * ny * nz
    t = np.zeros((nz, ny, nx), np.uint8)
    f = np.zeros((nz, ny, nx), np.int32)
    te = np.zeros((nz, ny, nx), np.float32)
    t[0] = C.ROCK
    xx, yy = np.meshgrid(np.arange(nx), np.arange(ny))
    hole = (xx % 3 == 1) & (yy % 3 == 1)
    t[1] = np.where(hole, C.AIR, C.LAVA)
    t[2] = np.where(hole, C.LAVA, C.AIR)
    ids = np.arange(1, 2 * nx * ny + 1, dtype=np.int32).reshape(2, ny, nx)
    rng = np.random.default_rng(nx + ny)
    for z in (1, 2):
        lava = t[z] == C.LAVA
        f[z] = np.where(lava, ids[z - 1], 0)
        te[z] = np.where(lava, rng.uniform(900.0, 1250.0, size=(ny, nx)).astype(np.float32), 0.0)
    s = O.CaState(nx, ny, nz, t.reshape(-1).copy(), f.reshape(-1).copy(), te.reshape(-1).copy(),
                  np.zeros(n, np.uint16), np.zeros(n, np.uint16))
    return s, hole


def _distinct_lava_ids_around(s, x, y, z):
    t = s.type.reshape(s.nz, s.ny, s.nx)
    f = s.flow.reshape(s.nz, s.ny, s.nx)
    ids = set()
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                qx, qy, qz = x + dx, y + dy, z + dz
                if 0 <= qx < s.nx and 0 <= qy < s.ny and 0 <= qz < s.nz and t[qz, qy, qx] == C.LAVA:
                    ids.add(int(f[qz, qy, qx]))
    return len(ids)


@pytest.mark.parametrize("sweep", [capi.SWEEP_ACTIVE_LIST, capi.SWEEP_DENSE], ids=["active", "dense"])
@pytest.mark.parametrize("nb", ["moore", "pentagonal"])
def test_wide_vote_junctions_match_oracle(nb, sweep):
    nx, ny, nz = 40, 22, 10
    s, hole = junction_state(nx, ny, nz)
    jy, jx = np.nonzero(hole)
    assert min(_distinct_lava_ids_around(s, int(x), int(y), 1) for x, y in zip(jx, jy)) >= 5
    p = capi.CaParams(nx, ny, nz, neighborhood=nb, boundary="absorbing", seed=31, max_steps=12, eruption_steps=0,
                      erupt_temp=1200.0, solidus_temp=800.0, cooling_ambient=2.0, cooling_lateral=4.0,
                      cooling_fall=2.0, ponding=True, sweep=sweep)
    spill = O.fill_depressions(np.ones(nx * ny, np.int32), nx, ny, False, False)
    op = C.oracle_params(p)
    vt = O.vent_table([])
    ca = capi.LavaCA(p)
    ca.set_state(s.type, s.flow, s.temp, s.solid, s.arrival, spill, [], steps_done=0)
    for t in range(p.max_steps):
        s, counts = O.ca_step(op, t, s, spill, vt)
        stop = O.ca_stop_after(op, t + 1, counts)
        ca.step()
        d = C.state_diff(s, ca.download())
        assert d == "", f"step {t + 1}: {d}"
        assert ca.info().stop_reason == stop
        if stop:
            break
    ca.close()


@pytest.mark.parametrize("sweep", [capi.SWEEP_ACTIVE_LIST, capi.SWEEP_DENSE], ids=["active", "dense"])
def test_last_steps_before_max_steps_limit(sweep):
    nx, ny, nz = 48, 20, 24
    seed = 4242
    p = capi.CaParams(nx, ny, nz, neighborhood="moore", boundary="periodic", seed=seed, max_steps=65535,
                      eruption_steps=65530, erupt_temp=1200.0, solidus_temp=800.0, cooling_ambient=2.0,
                      cooling_lateral=4.0, cooling_fall=2.0, ponding=True, sweep=sweep)
    heights = C.terrain(nx, ny, nz, seed)
    vents = C.pick_vents(heights, nx, ny, nz, 2, seed)
    spill = O.fill_depressions(heights, nx, ny, True, True)
    op = C.oracle_params(p)
    vt = O.vent_table(vents)
    s = C.initial_state(nx, ny, nz, heights, vents, p.erupt_temp)
    for t in range(15):  # a flow with some history
        s, _ = O.ca_step(op, t, s, spill, vt)
    t0 = 65525
    ca = capi.LavaCA(p)
    ca.set_state(s.type, s.flow, s.temp, s.solid, s.arrival, spill, vents, steps_done=t0)
    steps, stop = t0, 0
    while stop == 0:
        s, counts = O.ca_step(op, steps, s, spill, vt)
        steps += 1
        stop = O.ca_stop_after(op, steps, counts)
    ca.run()
    info = ca.info()
    assert (info.steps, info.stop_reason) == (steps, stop)
    assert capi.STOP_NAMES[stop] == "max steps" and steps == 65535
    assert C.state_diff(s, ca.download()) == ""
    assert max(int(s.arrival.max()), int(s.solid.max())) > t0  # stamps of the resumed steps were written
    ca.close()
