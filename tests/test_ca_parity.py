"""CUDA lava CA (libvca.so through the C ABI) against the CPU oracle, bit for bit.

Every case runs step by step: after each step the five planes, the step counters and the stop
reason of the CUDA path must equal the oracle's (LavaCA::step, engine/src/ca/LavaCA.hpp:230-247).
Both step schedules (ACTIVE tile skipping and DENSE) are checked.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import cases as C
from volcano_ca_mc_b200 import capi

pytestmark = pytest.mark.gpu

CASES = [
    # nx, ny, nz, neighborhood, boundary, steps, vents
    (64, 1, 48, "moore", "absorbing", 120, 1),
    (63, 1, 40, "moore", "periodic", 120, 2),
    (100, 1, 33, "von_neumann", "absorbing", 100, 2),
    (70, 1, 40, "hexagonal", "periodic", 100, 2),
    (64, 1, 48, "pentagonal", "absorbing", 100, 1),
    (24, 20, 16, "moore", "absorbing", 60, 2),
    (33, 17, 14, "moore", "periodic", 60, 2),
    (30, 30, 18, "von_neumann", "periodic", 60, 2),
    (40, 24, 20, "pentagonal", "absorbing", 60, 3),
    (65, 9, 21, "pentagonal", "periodic", 50, 2),
    # periodic x with nx a multiple of 16: the wrapped frame columns come with the tile's TMA boxes
    (64, 1, 40, "moore", "periodic", 100, 2),         # one tile in x: both ends wrap
    (48, 20, 16, "pentagonal", "periodic", 50, 2),    # padded rows: the copy of x = 0 sits at x = nx
    (128, 12, 12, "moore", "periodic", 50, 3),        # two tiles in x
]


def _params(nx, ny, nz, nb, bc, steps, sweep, seed):
    return capi.CaParams(nx, ny, nz, neighborhood=nb, boundary=bc, seed=seed, max_steps=steps,
                         eruption_steps=steps // 2, erupt_temp=1200.0, solidus_temp=800.0, cooling_ambient=2.0,
                         cooling_lateral=4.0, cooling_fall=2.0, ponding=True, sweep=sweep)


@pytest.mark.parametrize("sweep", [capi.SWEEP_ACTIVE_LIST, capi.SWEEP_DENSE], ids=["active", "dense"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}-{c[3]}-{c[4]}")
def test_lava_steps_match_oracle(case, sweep):
    nx, ny, nz, nb, bc, steps, nv = case
    seed = 1000 + nx * 7 + ny * 13 + nz
    p = _params(nx, ny, nz, nb, bc, steps, sweep, seed)
    heights = C.terrain(nx, ny, nz, seed)
    vents = C.pick_vents(heights, nx, ny, nz, nv, seed)
    op = C.oracle_params(p)
    per = bc == "periodic"
    spill = O.fill_depressions(heights, nx, ny, per and nx > 1, per and ny > 1)
    vt = O.vent_table(vents)
    s = C.initial_state(nx, ny, nz, heights, vents, p.erupt_temp)

    ca = capi.LavaCA(p)
    ca.apply_terrain(heights)
    ca.place_seeds(vents)
    assert np.array_equal(ca.spill(), spill)
    assert C.state_diff(s, ca.download()) == ""
    act, chg = [], []
    for t in range(steps):
        s, counts = O.ca_step(op, t, s, spill, vt)
        act.append(int(counts[0]))
        chg.append(int(counts[2]))
        stop = O.ca_stop_after(op, t + 1, counts)
        running = ca.step()
        d = C.state_diff(s, ca.download())
        assert d == "", f"step {t + 1}: {d}"
        info = ca.info()
        assert info.steps == t + 1
        assert info.stop_reason == stop, f"step {t + 1}: stop {info.stop_reason} vs {stop}"
        assert running == (stop == 0)
        if stop:
            break
    ha, hc = ca.history()
    assert ha == act and hc == chg
    ca.close()


@pytest.mark.parametrize("case", [(48, 1, 40, "moore", "periodic"), (20, 16, 12, "pentagonal", "absorbing"),
                                  (30, 1, 30, "hexagonal", "absorbing"), (16, 16, 10, "von_neumann", "periodic")])
def test_classic_steps_match_oracle(case):
    nx, ny, nz, nb, bc = case
    seed = 77 + nx
    p = capi.CaParams(nx, ny, nz, neighborhood=nb, boundary=bc, mode="classic", seed=seed, max_steps=80)
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    idx = rng.choice(n, size=6, replace=False)
    vents = [(int(i % nx), int((i // nx) % ny), int(i // (nx * ny)), k + 1) for k, i in enumerate(idx)]
    s = C.initial_state(nx, ny, nz, None, vents, 0.0, classic=True)
    op = C.oracle_params(p)
    vt = O.vent_table(vents)
    ca = capi.LavaCA(p)
    ca.place_seeds(vents)
    for t in range(80):
        s, counts = O.ca_step(op, t, s, None, vt)
        stop = O.ca_stop_after(op, t + 1, counts)
        ca.step()
        d = C.state_diff(s, ca.download())
        assert d == "", f"step {t + 1}: {d}"
        assert ca.info().stop_reason == stop
        if stop:
            break
    ca.close()


def test_run_to_stop_matches_stepwise():
    """vca_ca_run (chunked device-side stop test) ends on the same step and state as the oracle."""
    nx, ny, nz = 96, 1, 64
    p = _params(nx, ny, nz, "moore", "absorbing", 5000, capi.SWEEP_ACTIVE, 5)
    p.eruption_steps = 40
    heights = C.terrain(nx, ny, nz, 5)
    vents = C.pick_vents(heights, nx, ny, nz, 1, 5)
    spill = O.fill_depressions(heights, nx, ny, False, False)
    s0 = C.initial_state(nx, ny, nz, heights, vents, p.erupt_temp)
    s, steps, stop, act, chg = O.ca_run(C.oracle_params(p), s0, spill, O.vent_table(vents))
    for sweep in (capi.SWEEP_ACTIVE, capi.SWEEP_ACTIVE_LIST, capi.SWEEP_DENSE):
        p.sweep = sweep
        ca = capi.LavaCA(p)
        ca.apply_terrain(heights)
        ca.place_seeds(vents)
        ca.run()
        info = ca.info()
        assert (info.steps, info.stop_reason) == (steps, stop)
        assert C.state_diff(s, ca.download()) == ""
        assert ca.history() == (act, chg)
        ca.close()


def test_set_state_resumes():
    """A state uploaded mid-run (steps_done = k) continues exactly like the uninterrupted run."""
    nx, ny, nz = 40, 12, 24
    p = _params(nx, ny, nz, "moore", "periodic", 60, capi.SWEEP_ACTIVE_LIST, 9)
    heights = C.terrain(nx, ny, nz, 9)
    vents = C.pick_vents(heights, nx, ny, nz, 2, 9)
    spill = O.fill_depressions(heights, nx, ny, True, True)
    op = C.oracle_params(p)
    vt = O.vent_table(vents)
    s = C.initial_state(nx, ny, nz, heights, vents, p.erupt_temp)
    for t in range(20):
        s, _ = O.ca_step(op, t, s, spill, vt)
    ca = capi.LavaCA(p)
    ca.set_state(s.type, s.flow, s.temp, s.solid, s.arrival, spill, vents, steps_done=20)
    for t in range(20, 40):
        s, _ = O.ca_step(op, t, s, spill, vt)
        ca.step()
        assert C.state_diff(s, ca.download()) == "", f"step {t + 1}"
    ca.close()


def test_reset_reuses_handle():
    """vca_ca_reset: a handle that ran one job runs the next one (other terrain, other vents) exactly
    like a new handle, and the first job again exactly as before."""
    nx, ny, nz = 40, 24, 20
    jobs = []
    for seed in (7, 8):
        heights = C.terrain(nx, ny, nz, seed)
        vents = C.pick_vents(heights, nx, ny, nz, 2, seed)
        jobs.append((heights, vents))
    p = _params(nx, ny, nz, "moore", "periodic", 5000, capi.SWEEP_ACTIVE, 3)
    p.eruption_steps = 30

    def run(ca, job):
        ca.apply_terrain(job[0])
        ca.place_seeds(job[1])
        ca.run()
        return ca.info().steps, ca.info().stop_reason, ca.history(), ca.download()

    fresh = []
    for job in jobs:
        ca = capi.LavaCA(p)
        fresh.append(run(ca, job))
        ca.close()
    ca = capi.LavaCA(p)
    for n, k in enumerate((0, 1, 0)):
        if n:
            ca.reset()
        got = run(ca, jobs[k])
        assert got[:3] == fresh[k][:3]
        for a, b in zip(got[3], fresh[k][3]):
            assert np.array_equal(a, b)
    ca.close()


def test_reconfigure_runs_other_spaces_exactly():
    """vca_ca_reconfigure: a resident handle created for a large space runs smaller spaces with other
    parameters (2D and 3D, other neighbourhoods and boundaries) exactly like new handles, and refuses
    a space that does not fit."""
    big = _params(64, 40, 32, "moore", "absorbing", 400, capi.SWEEP_ACTIVE, 1)
    jobs = [(40, 24, 20, "pentagonal", "periodic", 7), (96, 1, 40, "hexagonal", "absorbing", 8),
            (33, 17, 14, "von_neumann", "periodic", 9)]
    ca = capi.LavaCA(big)
    for nx, ny, nz, nb, bc, seed in jobs:
        p = _params(nx, ny, nz, nb, bc, 300, capi.SWEEP_ACTIVE, seed)
        p.eruption_steps = 30
        heights = C.terrain(nx, ny, nz, seed)
        vents = C.pick_vents(heights, nx, ny, nz, 2, seed)
        fresh = capi.LavaCA(p)
        fresh.apply_terrain(heights)
        fresh.place_seeds(vents)
        fresh.run()
        want = (fresh.info().steps, fresh.info().stop_reason, fresh.history(), fresh.download())
        fresh.close()
        ca.reconfigure(p)
        ca.apply_terrain(heights)
        ca.place_seeds(vents)
        ca.run()
        got = (ca.info().steps, ca.info().stop_reason, ca.history(), ca.download())
        assert got[:3] == want[:3]
        for a, b in zip(got[3], want[3]):
            assert np.array_equal(a, b)
    assert capi.ca_footprint(big) >= capi.ca_footprint(_params(40, 24, 20, "moore", "absorbing", 300, 0, 1))
    with pytest.raises(capi.VcaError, match="does not fit"):
        ca.reconfigure(_params(128, 40, 32, "moore", "absorbing", 300, capi.SWEEP_ACTIVE, 1))
    ca.close()


TILE_CASES = [
    # nx, ny, nz, neighborhood, boundary, steps
    (70, 22, 27, "moore", "periodic", 60),
    (48, 20, 16, "pentagonal", "periodic", 50),     # periodic x with nx a multiple of 16 (wrapped columns by TMA)
    (65, 17, 21, "von_neumann", "absorbing", 50),
]


@pytest.mark.parametrize("blocks", [0, 1])
@pytest.mark.parametrize("tile", [(4, 4), (2, 8), (8, 2), (1, 16), (16, 1)], ids=lambda t: f"{t[0]}x{t[1]}")
@pytest.mark.parametrize("case", TILE_CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}-{c[3]}-{c[4]}")
def test_tile_shapes_match_oracle(case, tile, blocks):
    """The launch shape (tile 64 x tile_y x tile_z, resident rules blocks per SM) changes nothing in
    the results: every step equals the oracle's, in both schedules."""
    nx, ny, nz, nb, bc, steps = case
    seed = 300 + nx + ny
    heights = C.terrain(nx, ny, nz, seed)
    vents = C.pick_vents(heights, nx, ny, nz, 2, seed)
    per = bc == "periodic"
    spill = O.fill_depressions(heights, nx, ny, per, per)
    for sweep in (capi.SWEEP_ACTIVE_LIST, capi.SWEEP_DENSE):
        p = _params(nx, ny, nz, nb, bc, steps, sweep, seed)
        p.tile_y, p.tile_z, p.rules_blocks_per_sm = tile[0], tile[1], blocks
        op = C.oracle_params(p)
        vt = O.vent_table(vents)
        s = C.initial_state(nx, ny, nz, heights, vents, p.erupt_temp)
        ca = capi.LavaCA(p)
        ca.apply_terrain(heights)
        ca.place_seeds(vents)
        for t in range(steps):
            s, counts = O.ca_step(op, t, s, spill, vt)
            stop = O.ca_stop_after(op, t + 1, counts)
            ca.step()
            d = C.state_diff(s, ca.download())
            assert d == "", f"step {t + 1}: {d}"
            if stop:
                break
        ca.close()

