"""CUDA Potts checkerboard MC (libvca.so through the C ABI) against the CPU oracle, bit for bit:
orientations after every sweep, attempts / accepted / uphill counters and the energy
(PottsMC::sweep / totalEnergy, engine/src/mc/PottsMC.cpp:516-664)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import cases as C
from volcano_ca_mc_b200 import capi

pytestmark = pytest.mark.gpu


def _ca_result(nx, ny, nz, nb, bc, seed, steps=80):
    """A basalt field from an oracle CA run (the MC domain of McStage::run)."""
    p = capi.CaParams(nx, ny, nz, neighborhood=nb, boundary=bc, seed=seed, max_steps=steps, eruption_steps=steps // 3,
                      cooling_ambient=3.0, cooling_lateral=4.0, cooling_fall=2.0)
    heights = C.terrain(nx, ny, nz, seed)
    vents = C.pick_vents(heights, nx, ny, nz, 2, seed)
    per = bc == "periodic"
    spill = O.fill_depressions(heights, nx, ny, per and nx > 1, per and ny > 1)
    s0 = C.initial_state(nx, ny, nz, heights, vents, p.erupt_temp)
    s, *_ = O.ca_run(C.oracle_params(p), s0, spill, O.vent_table(vents))
    return p, heights, vents, s


MC_CASES = [
    # nx, ny, nz, nb, bc, Q, kT, mobility
    (80, 1, 48, "moore", "absorbing", 50, 0.0, True),
    (63, 1, 40, "hexagonal", "periodic", 32, 0.6, True),
    (70, 1, 40, "von_neumann", "periodic", 64, 0.5, False),
    (28, 22, 18, "moore", "absorbing", 128, 0.6, True),
    (33, 17, 15, "pentagonal", "periodic", 64, 0.5, True),
    (30, 30, 16, "von_neumann", "absorbing", 40, 0.0, False),
]


@pytest.mark.parametrize("case", MC_CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}-{c[3]}-{c[4]}-kT{c[6]}")
def test_basalt_sweeps_match_oracle(case):
    nx, ny, nz, nb, bc, Q, kT, use_mob = case
    seed = 300 + nx + ny
    _, _, _, s = _ca_result(nx, ny, nz, nb, bc, seed)
    domain = O.basalt_domain(s)
    assert domain.sum() > 20
    mob = O.mobility_from_cooling(s, domain, 0.05)
    mp = O.mc_params(nx, ny, nz, nb, bc, False, seed, Q, 1.0, kT)
    spin = O.mc_init(mp, domain)

    mc = capi.PottsMC(capi.McParams(nx, ny, nz, neighborhood=nb, boundary=bc, seed=seed, Q=Q, J=1.0, kT=kT))
    mc.set_domain(domain)
    if use_mob:
        mc.set_mobility(mob)
    mc.initialize()
    info = mc.info()
    assert info.colors == O.mc_colors(mp)
    assert info.domain_cells == int(domain.sum())
    assert np.array_equal(mc.crystals(), spin)
    assert mc.energy() == O.mc_energy(mp, 0, spin)
    tot = np.zeros(3, np.uint64)
    for t in range(12):
        tot += O.mc_sweep(mp, t, domain, mob if use_mob else None, spin)
        acc = mc.sweep(1)
        got = mc.crystals()
        assert np.array_equal(got, spin), f"sweep {t + 1}: {(got != spin).sum()} cells differ"
    info = mc.info()
    assert (info.attempts, info.accepted, info.uphill) == tuple(int(v) for v in tot)
    assert info.sweeps == 12
    assert mc.energy() == O.mc_energy(mp, 12, spin)
    mc.close()


FULL_CASES = [
    # nb, bc, dims, Q, mobility
    ("moore", "periodic", (25, 1, 31), 20, False),
    ("von_neumann", "periodic", (24, 20, 1), 20, False),
    ("pentagonal", "periodic", (15, 13, 11), 20, False),
    ("von_neumann", "periodic", (9, 10, 7), 20, False),
    ("moore", "absorbing", (14, 12, 10), 256, False),
    ("moore", "periodic", (16, 10, 12), 256, True),
    ("hexagonal", "periodic", (21, 17, 1), 64, True),
    ("von_neumann", "absorbing", (11, 9, 7), 40, True),
    ("pentagonal", "absorbing", (12, 1, 13), 300, False),
]


@pytest.mark.parametrize("nb,bc,dims,Q,use_mob", FULL_CASES,
                         ids=lambda c: str(c) if not isinstance(c, tuple) else "x".join(map(str, c)))
def test_full_domain_sweeps_match_oracle(nb, bc, dims, Q, use_mob):
    """mc.domain = full: odd periodic axes give 3 classes (PottsMC.cpp:145-193).  Q <= 256 runs the
    whole-space sweeps on the byte copy of the orientations, Q = 300 the list sweeps."""
    nx, ny, nz = dims
    seed = 11 + nx
    mp = O.mc_params(nx, ny, nz, nb, bc, True, seed, Q, 1.0, 0.4)
    domain = np.ones(nx * ny * nz, np.uint8)
    spin = O.mc_init(mp, domain)
    mob = None
    if use_mob:
        mob = np.random.default_rng(seed).uniform(0.05, 1.0, nx * ny * nz).astype(np.float32)
    mc = capi.PottsMC(capi.McParams(nx, ny, nz, neighborhood=nb, boundary=bc, domain_full=True, seed=seed, Q=Q,
                                    kT=0.4))
    mc.set_domain(None)
    if use_mob:
        mc.set_mobility(mob)
    mc.initialize()
    assert mc.info().colors == O.mc_colors(mp)
    tot = np.zeros(3, np.uint64)
    for t in range(8):
        tot += O.mc_sweep(mp, t, domain, mob, spin)
        mc.sweep(1)
        assert np.array_equal(mc.crystals(), spin), f"sweep {t + 1}"
    # several sweeps in one call
    for t in range(8, 11):
        tot += O.mc_sweep(mp, t, domain, mob, spin)
    mc.sweep(3)
    assert np.array_equal(mc.crystals(), spin), "sweeps 9-11"
    info = mc.info()
    assert (info.attempts, info.accepted, info.uphill) == tuple(int(v) for v in tot)
    assert mc.energy() == O.mc_energy(mp, 11, spin)
    mc.close()


def test_domain_and_mobility_from_ca_on_device():
    """vca_mc_set_domain_from_ca / set_mobility_from_ca equal CoolingMobility on the host."""
    nx, ny, nz = 40, 18, 20
    p, heights, vents, s = _ca_result(nx, ny, nz, "moore", "absorbing", 21, steps=5000)
    ca = capi.LavaCA(p)
    ca.set_state(s.type, s.flow, s.temp, s.solid, s.arrival, None, vents, steps_done=0)
    domain = O.basalt_domain(s)
    mob = O.mobility_from_cooling(s, domain, 0.05)
    mc = capi.PottsMC(capi.McParams(nx, ny, nz, seed=21, Q=64, kT=0.6))
    mc.set_domain_from_ca(ca)
    mc.set_mobility_from_ca(ca, 0.05, True)
    got = mc.mobility()
    assert np.array_equal(got.view(np.uint32), mob.view(np.uint32))
    mc.initialize()
    assert mc.info().domain_cells == int(domain.sum())
    mp = O.mc_params(nx, ny, nz, "moore", "absorbing", False, 21, 64, 1.0, 0.6)
    spin = O.mc_init(mp, domain)
    for t in range(5):
        O.mc_sweep(mp, t, domain, mob, spin)
    mc.sweep(5)
    assert np.array_equal(mc.crystals(), spin)
    mc.close()
    ca.close()


def _grains_host(spins, dims, moore, periodic, mob=None, thr=0.5):
    """labelGrains (engine/src/mc/Grains.cpp:33-150) and the majority classes of McStage
    (engine/src/app/McStage.cpp:38-66), restated with a plain union-find for the check."""
    nx, ny, nz = dims
    n = nx * ny * nz
    parent = list(range(n))

    def find(i):
        while parent[i] != i:
            parent[i] = parent[parent[i]]
            i = parent[i]
        return i

    offs = [(dx, dy, dz) for dz in (0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
            if (dz > 0 or (dz == 0 and (dy > 0 or (dy == 0 and dx > 0))))
            and not ((nx == 1 and dx) or (ny == 1 and dy) or (nz == 1 and dz))
            and (moore or abs(dx) + abs(dy) + abs(dz) == 1)]
    for i in range(n):
        s = spins[i]
        if s <= 0:
            continue
        x, y, z = i % nx, (i // nx) % ny, i // (nx * ny)
        for dx, dy, dz in offs:
            q = []
            for v, d, size, per in ((x, dx, nx, periodic[0]), (y, dy, ny, periodic[1]), (z, dz, nz, periodic[2])):
                w = v + d
                if 0 <= w < size:
                    q.append(w)
                elif per and size > 1:
                    q.append(w % size)
                else:
                    q = None
                    break
            if q is None:
                continue
            j = q[0] + nx * (q[1] + ny * q[2])
            if spins[j] == s:
                a, b = find(i), find(j)
                if a != b:
                    parent[max(a, b)] = min(a, b)
    size, high = {}, {}
    for i in range(n):
        if spins[i] > 0:
            r = find(i)
            size[r] = size.get(r, 0) + 1
            if mob is not None and float(mob[i]) >= thr:
                high[r] = high.get(r, 0) + 1
    hi = [s for r, s in size.items() if 2 * high.get(r, 0) >= s]
    lo = [s for r, s in size.items() if 2 * high.get(r, 0) < s]
    hc = sum(1 for i in range(n) if spins[i] > 0 and mob is not None and float(mob[i]) >= thr)
    return (len(size), sum(size.values()), max(size.values(), default=0), hc, len(hi), sum(hi), max(hi, default=0),
            len(lo), sum(lo), max(lo, default=0))


@pytest.mark.parametrize("case", [(20, 16, 12, "moore", "periodic", True), (24, 1, 30, "von_neumann", "absorbing", False),
                                  (18, 14, 10, "pentagonal", "periodic", False), (32, 1, 20, "hexagonal", "periodic", True)])
def test_device_grains_match_host_labelling(case):
    nx, ny, nz, nb, bc, full = case
    rng = np.random.default_rng(4)
    mc = capi.PottsMC(capi.McParams(nx, ny, nz, neighborhood=nb, boundary=bc, domain_full=full, seed=9, Q=4, kT=0.2))
    dom = None if full else (rng.random(nx * ny * nz) < 0.7).astype(np.uint8)
    mc.set_domain(dom)
    mob = rng.random(nx * ny * nz).astype(np.float32)
    mc.set_mobility(mob)
    mc.initialize()
    for _ in range(3):
        mc.sweep(2)
        g = mc.grains(moore=nb != "von_neumann", threshold=0.5)
        spins = mc.crystals()
        per = bc == "periodic"
        want = _grains_host(spins.tolist(), (nx, ny, nz), nb != "von_neumann",
                            (per and nx > 1, per and ny > 1, per and full and nz > 1), mob)
        got = (g.grains, g.cells, g.largest, g.high_cells, g.high_grains, g.high_grain_cells, g.high_largest,
               g.low_grains, g.low_grain_cells, g.low_largest)
        assert got == want
    mc.close()


def test_mc_reconfigure_runs_other_spaces_exactly():
    """vca_mc_reconfigure: one handle, spaces of fewer cells and other parameters, same results as
    new handles; a larger space is refused."""
    mc = capi.PottsMC(capi.McParams(40, 30, 20, neighborhood="moore", boundary="periodic", domain_full=True, seed=1, Q=8))
    rng = np.random.default_rng(3)
    for nx, ny, nz, nb, bc, full, Q, kT in [(20, 16, 12, "pentagonal", "periodic", False, 16, 0.4),
                                            (48, 1, 30, "hexagonal", "absorbing", True, 5, 0.0),
                                            (17, 13, 9, "von_neumann", "periodic", True, 32, 1.0)]:
        p = capi.McParams(nx, ny, nz, neighborhood=nb, boundary=bc, domain_full=full, seed=5, Q=Q, kT=kT)
        dom = None if full else (rng.random(nx * ny * nz) < 0.6).astype(np.uint8)
        fresh = capi.PottsMC(p)
        fresh.set_domain(dom)
        fresh.initialize()
        fresh.sweep(4)
        want = (fresh.crystals(), fresh.energy(), fresh.info().attempts)
        fresh.close()
        mc.reconfigure(p)
        mc.set_domain(dom)
        mc.initialize()
        mc.sweep(4)
        got = (mc.crystals(), mc.energy(), mc.info().attempts)
        assert np.array_equal(got[0], want[0]) and got[1:] == want[1:]
    with pytest.raises(capi.VcaError, match="does not fit"):
        mc.reconfigure(capi.McParams(41, 30, 20, neighborhood="moore", boundary="periodic", domain_full=True, Q=8))
    mc.close()
