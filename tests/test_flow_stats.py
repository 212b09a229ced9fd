"""Per-flow sums on the device (vca_ca_flow_stats) against the same sums over the downloaded planes
(Simulation::flowSums, engine/src/app/Simulation.cpp:408-466): LAVA and BASALT cells per flowId and
the largest squared horizontal distance from the flow's vent.  Few flows are summed per block in
shared memory, many (classic grains) with global atomics; both paths are covered."""
import numpy as np
import pytest

from tests import cases as C
from volcano_ca_mc_b200 import capi

pytestmark = pytest.mark.gpu


def _host_sums(planes, nx, ny, nz, vents, flows):
    t, f = planes[0].astype(np.int64), planes[1].astype(np.int64)
    idx = np.arange(nx * ny * nz, dtype=np.int64)
    x, y = idx % nx, (idx // nx) % ny
    sel = ((t == 2) | (t == 3)) & (f > 0) & (f <= flows)
    lava = np.bincount(f[sel & (t == 2)], minlength=flows + 1).astype(np.uint64)
    basalt = np.bincount(f[sel & (t == 3)], minlength=flows + 1).astype(np.uint64)
    vx = np.zeros(flows + 1, np.int64)
    vy = np.zeros(flows + 1, np.int64)
    for (px, py, _pz, fid) in vents:
        if fid <= flows:
            vx[fid], vy[fid] = px, py
    d2 = (x[sel] - vx[f[sel]]) ** 2 + (y[sel] - vy[f[sel]]) ** 2
    reach2 = np.zeros(flows + 1, np.uint64)
    np.maximum.at(reach2, f[sel], d2.astype(np.uint64))
    lava[0] = basalt[0] = reach2[0] = 0
    return lava, basalt, reach2


@pytest.mark.parametrize("case", [(64, 1, 48, "moore", "absorbing", 3), (33, 17, 14, "moore", "periodic", 4),
                                  (40, 24, 20, "pentagonal", "absorbing", 5)])
def test_lava_flow_sums(case):
    nx, ny, nz, nb, bc, nv = case
    seed = 300 + nx
    p = capi.CaParams(nx, ny, nz, neighborhood=nb, boundary=bc, seed=seed, max_steps=90, eruption_steps=45,
                      erupt_temp=1200.0, solidus_temp=800.0, cooling_ambient=2.0, cooling_lateral=4.0,
                      cooling_fall=2.0)
    heights = C.terrain(nx, ny, nz, seed)
    vents = C.pick_vents(heights, nx, ny, nz, nv, seed)
    ca = capi.LavaCA(p)
    ca.apply_terrain(heights)
    ca.place_seeds(vents)
    for steps in (0, 30, 90):
        while ca.info().steps < steps and ca.step():
            pass
        got = ca.flow_stats(len(vents))
        want = _host_sums(ca.download(), nx, ny, nz, vents, len(vents))
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
    ca.close()


def test_classic_many_flows():
    """More flows than the shared-memory path holds: global atomics."""
    nx, ny, nz = 60, 40, 20
    p = capi.CaParams(nx, ny, nz, neighborhood="moore", boundary="periodic", mode="classic", seed=5, max_steps=3)
    rng = np.random.default_rng(5)
    idx = rng.choice(nx * ny * nz, size=3000, replace=False)
    vents = [(int(i % nx), int((i // nx) % ny), int(i // (nx * ny)), k + 1) for k, i in enumerate(idx)]
    ca = capi.LavaCA(p)
    ca.place_seeds(vents)
    ca.run()
    got = ca.flow_stats(len(vents))
    want = _host_sums(ca.download(), nx, ny, nz, vents, len(vents))
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    # fewer flows than ids present: ids above the count are left out
    got = ca.flow_stats(100)
    want = _host_sums(ca.download(), nx, ny, nz, vents, 100)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    ca.close()
