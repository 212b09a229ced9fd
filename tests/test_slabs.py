"""z slabs of one lava grid (volcano_ca_mc_b200.slabs, the reference's strips): the partition, the
halo plan, and the step loop with its count sums and halo exchange.

CPU part: the step loop runs on slabs whose step is the oracle's strip step (a test backend), in one
process and as two gloo ranks of torch.distributed; the assembled owned layers, step count, stop
reason and histories must equal the single-grid oracle run bit for bit.  GPU part: the same loop on
vca_ca slab handles, several slabs on one GPU, against the single-grid run."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import cases as C
from volcano_ca_mc_b200 import capi, slabs


def test_partition_and_plan():
    lays = slabs.partition(100, 3)
    assert [(l.z0, l.z1) for l in lays] == [(0, 34), (34, 67), (67, 100)]
    assert [(l.lo, l.hi) for l in lays] == [(0, 35), (17, 68), (50, 100)]
    p0, p1, p2 = (slabs.message_plan(l) for l in lays)
    assert set(p0) == {"send_up", "recv_up"} and set(p2) == {"send_down", "recv_down"} and len(p1) == 4
    # rank 0's up message lands exactly in rank 1's halo below, rank 1's down message in rank 0's halo above
    z0, n, full = p0["send_up"]
    rz0, rn, rfull = p1["recv_down"]
    assert (z0 + lays[0].lo, n, full + lays[0].lo) == (rz0 + lays[1].lo, rn, rfull + lays[1].lo)
    assert p1["send_down"][0] + lays[1].lo == p0["recv_up"][0] + lays[0].lo
    with pytest.raises(ValueError):
        slabs.partition(30, 2)


class OracleSlab:
    """A slab whose step is the oracle's strip step (test backend of the slab loop)."""

    def __init__(self, p, lay, s_full, spill, vents):
        self.lay, self.p = lay, p
        n = p.nx * p.ny
        lo, hi = lay.lo, lay.hi
        self.s = O.CaState(p.nx, p.ny, lay.nz_local, *(a[lo * n:hi * n].copy() for a in
                                                       (s_full.type, s_full.flow, s_full.temp, s_full.solid,
                                                        s_full.arrival)))
        self.op = C.oracle_params(capi.CaParams(**{**p.__dict__, "nz": lay.nz_local}))
        self.spill = (spill - lo).astype(np.int32)
        self.vt = O.vent_table(slabs.local_vents(vents, lay))
        self.layer_cells = n
        self.t = 0

    def step(self):
        o0, o1 = self.lay.own
        self.s, c = O.ca_step_strip(self.op, self.t, self.p.nx * self.p.ny * self.lay.lo, o0, o1, self.s, self.spill,
                                    self.vt)
        self.t += 1
        return int(c[0]), int(c[2])

    def stop(self, reason):
        pass

    def _views(self, z0, types, full, buf):
        b = np.asarray(buf).view(np.uint8)
        L = self.layer_cells
        out = [(self.s.type[z0 * L:(z0 + types) * L], b[:types * L])]
        if full >= 0:
            at = types * L
            for plane, w in ((self.s.flow, 4), (self.s.temp, 4), (self.s.solid, 2), (self.s.arrival, 2)):
                out.append((plane[full * L:(full + 1) * L].view(np.uint8), b[at:at + w * L]))
                at += w * L
        return out

    def pack(self, z0, types, full, buf):
        for src, dst in self._views(z0, types, full, buf):
            dst[:] = src

    def unpack(self, z0, types, full, buf):
        for dst, src in self._views(z0, types, full, buf):
            dst[:] = src

    def owned_planes(self):
        o0, o1 = self.lay.own
        n = self.layer_cells
        return [a[o0 * n:o1 * n] for a in (self.s.type, self.s.flow, self.s.temp, self.s.solid, self.s.arrival)]


def case(nb, seed=12):
    nx, ny, nz = 40, 24, 60
    p = capi.CaParams(nx, ny, nz, neighborhood=nb, boundary="periodic", seed=seed, max_steps=70, eruption_steps=35,
                      cooling_ambient=2.0, cooling_lateral=4.0, cooling_fall=2.0, sweep=capi.SWEEP_DENSE)
    heights = C.terrain(nx, ny, nz, seed)
    vents = C.pick_vents(heights, nx, ny, nz, 3, seed)
    spill = O.fill_depressions(heights, nx, ny, True, True)
    s0 = C.initial_state(nx, ny, nz, heights, vents, p.erupt_temp)
    want = O.ca_run(C.oracle_params(p), s0.copy(), spill, O.vent_table(vents))
    return p, heights, vents, spill, s0, want


@pytest.mark.parametrize("nb,world", [("moore", 2), ("pentagonal", 3)])
def test_slab_loop_in_one_process_equals_single_grid(nb, world):
    p, heights, vents, spill, s0, (s, steps, stop, act, chg) = case(nb)
    parts = [OracleSlab(p, lay, s0, spill, vents) for lay in slabs.partition(p.nz, world)]
    got = slabs.run_local(parts, p.max_steps, nb == "pentagonal", len(vents), lambda n: np.zeros(n, np.uint8))
    assert got == (steps, stop, act, chg)
    planes = slabs.assemble([x.owned_planes() for x in parts])
    assert C.state_diff(s, planes) == ""


def _gloo_rank(rank, world, port, nb, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p, heights, vents, spill, s0, _ = case(nb)
        lay = slabs.partition(p.nz, world)[rank]
        slab = OracleSlab(p, lay, s0, spill, vents)
        res = slabs.run_distributed(slab, slabs.TorchComm("cpu"), p.max_steps, nb == "pentagonal", len(vents))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), *slab.owned_planes(), res=np.array(res[:2]),
                 act=np.array(res[2], np.int64), chg=np.array(res[3], np.int64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nb", ["moore", "pentagonal"])
def test_slab_loop_over_two_gloo_ranks_equals_single_grid(nb, tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_gloo_rank, args=(2, port, nb, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    p, heights, vents, spill, s0, (s, steps, stop, act, chg) = case(nb)
    parts = []
    for r in range(2):
        z = np.load(tmp_path / f"rank{r}.npz")
        assert tuple(z["res"]) == (steps, stop)
        assert z["act"].tolist() == act and z["chg"].tolist() == chg
        parts.append([z[f"arr_{i}"] for i in range(5)])
    assert C.state_diff(s, slabs.assemble(parts)) == ""


@pytest.mark.gpu
@pytest.mark.parametrize("nb,world", [("moore", 2), ("pentagonal", 3)])
def test_gpu_slabs_on_one_gpu_equal_single_grid(nb, world):
    import torch
    p, heights, vents, spill, s0, (s, steps, stop, act, chg) = case(nb)
    parts = [slabs.GpuSlab(p, lay, heights, vents) for lay in slabs.partition(p.nz, world)]
    got = slabs.run_local(parts, p.max_steps, nb == "pentagonal", len(vents),
                          lambda n: torch.empty(n, dtype=torch.uint8, device="cuda"))
    assert got == (steps, stop, act, chg)
    planes = slabs.assemble([x.owned_planes() for x in parts])
    assert C.state_diff(s, planes) == ""
    for x in parts:
        x.close()


# ------------------------------------------------------------------------------------------
# MC stage over slabs
# ------------------------------------------------------------------------------------------
class OracleMcSlab:
    """An MC slab whose colour pass is the oracle's strip pass (test backend of the MC slab loop)."""

    def __init__(self, mp_global, lay, spin0, domain, mobility):
        lo, hi = slabs.mc_layout(lay)
        self.lay, self.lo, self.hi = lay, lo, hi
        self.L = mp_global.nx * mp_global.ny
        self.mp = O.McParams(**{f: getattr(mp_global, f) for f, _ in O.McParams._fields_})
        self.mp.nz = hi - lo
        own = slice((lay.z0 - lo) * self.L, (lay.z1 - lo) * self.L)
        glob = slice(lay.z0 * self.L, lay.z1 * self.L)
        n = (hi - lo) * self.L
        self.spin = np.zeros(n, np.int32)
        self.dom = np.zeros(n, np.uint8)
        self.mob = np.zeros(n, np.float32)
        self.spin[own], self.dom[own], self.mob[own] = spin0[glob], domain[glob], mobility[glob]
        self.colors = O.mc_colors(mp_global)
        self.t = 0
        self.cnt = np.zeros(3, np.uint64)

    plan = slabs.McSlab.plan

    def color_pass(self, c):
        self.cnt += O.mc_color_strip(self.mp, self.t, c, self.L * self.lo, self.lo, self.dom, self.mob, self.spin)
        if c == self.colors - 1:
            self.t += 1

    def pack(self, z, buf):
        np.asarray(buf).view(np.int32)[:] = self.spin[z * self.L:(z + 1) * self.L]

    def unpack(self, z, buf):
        self.spin[z * self.L:(z + 1) * self.L] = np.asarray(buf).view(np.int32)

    def counters(self):
        return tuple(int(v) for v in self.cnt)

    def owned_spins(self):
        return self.spin[(self.lay.z0 - self.lo) * self.L:(self.lay.z1 - self.lo) * self.L]


def mc_case(nb, sweeps=6):
    p, heights, vents, spill, s0, (s, *_r) = case(nb)
    mp = O.mc_params(p.nx, p.ny, p.nz, nb, "periodic", False, p.seed, 24, 1.0, 0.5)
    dom = O.basalt_domain(s)
    mob = O.mobility_from_cooling(s, dom, 0.05)
    spin0 = O.mc_init(mp, dom)
    spin = spin0.copy()
    cnt = np.zeros(3, np.uint64)
    for t in range(sweeps):
        cnt += O.mc_sweep(mp, t, dom, mob, spin)
    return p, s, mp, dom, mob, spin0, spin, [int(v) for v in cnt], sweeps


@pytest.mark.parametrize("nb,world", [("moore", 2), ("pentagonal", 3)])
def test_mc_slabs_in_one_process_equal_single_grid(nb, world):
    p, s, mp, dom, mob, spin0, want, cnt, sweeps = mc_case(nb)
    parts = [OracleMcSlab(mp, lay, spin0, dom, mob) for lay in slabs.partition(p.nz, world)]
    slabs.run_mc_local(parts, sweeps, lambda n: np.zeros(n, np.uint8))
    assert np.array_equal(np.concatenate([x.owned_spins() for x in parts]), want)
    assert [sum(x.counters()[i] for x in parts) for i in range(3)] == cnt


def _gloo_mc_rank(rank, world, port, nb, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p, s, mp, dom, mob, spin0, _, _, sweeps = mc_case(nb)
        x = OracleMcSlab(mp, slabs.partition(p.nz, world)[rank], spin0, dom, mob)
        slabs.run_mc_distributed(x, slabs.TorchComm("cpu"), sweeps)
        np.savez(os.path.join(out_dir, f"mc{rank}.npz"), spin=x.owned_spins(), cnt=np.array(x.counters(), np.int64))
    finally:
        dist.destroy_process_group()


def test_mc_slabs_over_two_gloo_ranks_equal_single_grid(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_gloo_mc_rank, args=(2, port, "pentagonal", str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    _, _, _, _, _, _, want, cnt, _ = mc_case("pentagonal")
    z = [np.load(tmp_path / f"mc{r}.npz") for r in range(2)]
    assert np.array_equal(np.concatenate([q["spin"] for q in z]), want)
    assert (z[0]["cnt"] + z[1]["cnt"]).tolist() == cnt


def test_mobility_terms_equal_the_whole_domain():
    """The slab mobility (end step and liquid-time range reduced over the slabs, then normalised per
    slab) equals CoolingMobility::fromCooling of the whole grid."""
    p, s, mp, dom, mob, *_ = mc_case("moore")
    lays = slabs.partition(p.nz, 3)
    n = p.nx * p.ny
    planes = [[a[l.z0 * n:l.z1 * n] for a in (s.type, s.flow, s.temp, s.solid, s.arrival)] for l in lays]
    end, tmin, tmax = slabs.mobility_terms(planes)
    got = np.concatenate([slabs.normalize(slabs.liquid_time(pl, end), slabs.basalt_domain(pl[0]), tmin, tmax, 0.05)
                          for pl in planes])
    assert np.array_equal(got.view(np.uint32), mob.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("nb,world", [("moore", 2), ("pentagonal", 3)])
def test_gpu_mc_slabs_on_one_gpu_equal_single_grid(nb, world):
    import torch
    p, heights, vents, spill, s0, _ = case(nb)
    # single grid on the GPU: CA, then MC with the device-built domain and cooling mobility
    ca = capi.LavaCA(p)
    ca.apply_terrain(heights)
    ca.place_seeds(vents)
    ca.run()
    mcp = capi.McParams(p.nx, p.ny, p.nz, neighborhood=nb, boundary="periodic", seed=p.seed, Q=24, J=1.0, kT=0.5)
    mc = capi.PottsMC(mcp)
    mc.set_domain_from_ca(ca)
    mc.set_mobility_from_ca(ca, 0.05, True)
    mc.initialize()
    mc.sweep(5)
    want, info = mc.crystals(), mc.info()
    mc.close()
    whole = ca.download()
    ca.close()
    # MC slabs on the owned layers of the same CA end state (the CA slabs have their own test)
    lays = slabs.partition(p.nz, world)
    n = p.nx * p.ny
    planes = [[a[lay.z0 * n:lay.z1 * n] for a in whole] for lay in lays]
    buf = lambda n: torch.empty(n, dtype=torch.uint8, device="cuda")
    terms = slabs.mobility_terms(planes)
    ms = [slabs.McSlab(mcp, lay, pl, terms, 0.05) for lay, pl in zip(lays, planes)]
    slabs.run_mc_local(ms, 5, buf)
    assert np.array_equal(np.concatenate([m.owned_spins() for m in ms]), want)
    assert [sum(m.counters()[i] for m in ms) for i in range(3)] == [info.attempts, info.accepted, info.uphill]
    for x in ms:
        x.close()
