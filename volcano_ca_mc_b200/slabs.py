"""z slabs of one lava grid over several GPUs: the reference's strips (engine/src/parallel/Strip.hpp:1-25,
engine/src/mpi/MpiSimulation.cpp, MpiHalo.cpp) on the device.

Each rank owns the global layers [z0, z1) and holds them with 17 halo layers below (dropDepth looks 17
cells down, LavaCA.hpp:404-414 with kMaxDrop = 16) and 1 above.  A step of the whole grid is:

1. every rank steps its slab (vca_ca_slab_step: DENSE schedule, hashRand on global indices, counts of
   the owned layers only);
2. the three counts of the step -- LAVA cells, changed cells -- are summed over the ranks and the stop
   rule of finishStep (LavaCA.hpp:1206-1229) is applied to the sums (the reference sums the same
   counters over its strips, LavaCA.hpp:1207-1211);
3. halo exchange: rank r sends rank r+1 the types of its top 17 owned layers and the full state of the
   topmost one (rank r+1's halo below), and rank r-1 the full state of its lowest owned layer (rank
   r-1's halo above).  Deeper halo layers carry types only, as the reference's strips.

Halo cells are stepped too but their results are overwritten by the exchange before anyone reads
them; every owned cell reads only owned or freshly exchanged cells, so the assembled result is the
single-grid result bit for bit.

The driver is independent of where a slab lives: a backend steps one slab and packs / unpacks its
halo messages (``GpuSlab``: a vca_ca handle on this process's GPU), and a communicator sums counts
and moves messages (``TorchComm``: torch.distributed send / recv and all-reduce, NCCL between GPUs).
``run_local`` drives several slabs in one process (one GPU holding every slab; no kernel waits on
another, the host orders the steps and the copies).

The MC stage splits the same way (PottsMC.cpp:451-460): each slab holds its owned layers and one
halo layer on each side, its domain is the basalt of its owned layers, and after every colour of
every MCS the slabs exchange their boundary layers of orientations.  The cooling mobility needs the
end step and the liquid-time range of the whole domain: those three numbers are reduced over the
slabs (min / max), then each slab normalises its own cells (CoolingMobility::fromCooling,
engine/src/mc/CoolingMobility.cpp:16-83).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import capi

HALO_BELOW = 17  # drop depths read types 17 layers down
HALO_ABOVE = 1   # sources one layer up
STOP_NO_LAVA, STOP_NO_CHANGE, STOP_MAX_STEPS = 1, 3, 4


@dataclass
class SlabLayout:
    """Global layers of one rank's slab: it owns [z0, z1) and holds [lo, hi)."""
    rank: int
    world: int
    nz: int
    z0: int
    z1: int
    lo: int
    hi: int

    @property
    def own(self) -> tuple[int, int]:
        """Owned layers in local z."""
        return self.z0 - self.lo, self.z1 - self.lo

    @property
    def nz_local(self) -> int:
        return self.hi - self.lo


def partition(nz: int, world: int) -> list[SlabLayout]:
    """Equal z slabs (the first nz % world ranks one layer taller).  Every slab must hold at least
    HALO_BELOW + 1 layers, so that a halo comes from one neighbour only."""
    base, extra = divmod(nz, world)
    if base < HALO_BELOW + 1:
        raise ValueError(f"{nz} layers over {world} slabs leaves fewer than {HALO_BELOW + 1} layers per slab")
    out, z = [], 0
    for r in range(world):
        h = base + (1 if r < extra else 0)
        lo, hi = max(0, z - HALO_BELOW), min(nz, z + h + HALO_ABOVE)
        out.append(SlabLayout(r, world, nz, z, z + h, lo, hi))
        z += h
    return out


def message_plan(lay: SlabLayout) -> dict:
    """The halo messages of a rank after a step, in local z of the sender / receiver:
    up: to rank + 1, types of the top HALO_BELOW owned layers + full state of the topmost;
    down: to rank - 1, full state of the lowest owned layer."""
    o0, o1 = lay.own
    plan = {}
    if lay.rank + 1 < lay.world:
        plan["send_up"] = (o1 - HALO_BELOW, HALO_BELOW, o1 - 1)  # (z0, type layers, full layer)
        plan["recv_up"] = (o1, 1, o1)                            # halo above from rank + 1
    if lay.rank > 0:
        plan["send_down"] = (o0, 1, o0)
        plan["recv_down"] = (o0 - HALO_BELOW, HALO_BELOW, o0 - 1)
    return plan


def message_bytes(types: int, full: int, layer_cells: int) -> int:
    return (types + (12 if full >= 0 else 0)) * layer_cells


def finish(steps: int, active: int, changed: int, max_steps: int, random_nb: bool) -> int:
    """finishStep's stop rule on counts summed over all slabs (LavaCA.hpp:1216-1228), lava mode."""
    if active == 0:
        return STOP_NO_LAVA
    if changed == 0 and not random_nb:
        return STOP_NO_CHANGE
    if steps >= max_steps:
        return STOP_MAX_STEPS
    return 0


def local_vents(vents, lay: SlabLayout):
    """Vents (global x, y, z, flowId) inside the slab's held layers, in local z."""
    return [(x, y, z - lay.lo, f) for (x, y, z, f) in vents if lay.lo <= z < lay.hi]


class GpuSlab:
    """One slab on this process's GPU: a vca_ca handle of nx x ny x (held layers), set as a slab."""

    def __init__(self, params: "capi.CaParams", lay: SlabLayout, heights, vents):
        p = capi.CaParams(**{**params.__dict__, "nz": lay.nz_local, "sweep": capi.SWEEP_DENSE})
        self.lay = lay
        self.ca = capi.LavaCA(p)
        o0, o1 = lay.own
        self.ca.set_slab(lay.lo, o0, o1)
        self.ca.apply_terrain(heights)  # the whole grid's heights; the handle shifts them to its layers
        self.ca.place_seeds(local_vents(vents, lay))
        self.layer_cells = self.ca.layers()[1]

    def step(self) -> tuple[int, int]:
        return self.ca.slab_step()

    def stop(self, reason: int) -> None:
        self.ca.slab_stop(reason)

    def pack(self, z0: int, types: int, full: int, buf) -> None:
        self.ca.pack_layers(z0, types, full, buf.data_ptr())

    def unpack(self, z0: int, types: int, full: int, buf) -> None:
        self.ca.unpack_layers(z0, types, full, buf.data_ptr())

    def owned_planes(self):
        """The owned layers of the five planes (host arrays, globalIndex order of the slab)."""
        t, f, te, so, ar = self.ca.download()
        o0, o1 = self.lay.own
        n = self.ca.params.nx * self.ca.params.ny
        return [a[o0 * n:o1 * n] for a in (t, f, te, so, ar)]

    def close(self):
        self.ca.close()


class TorchComm:
    """Counts and halo messages over torch.distributed (NCCL for CUDA buffers, gloo for CPU ones)."""

    def __init__(self, device):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.device = dist, torch, device

    def allreduce(self, values, op: str = "sum"):
        t = self.torch.tensor(values, dtype=self.torch.int64, device=self.device)
        red = {"sum": self.dist.ReduceOp.SUM, "min": self.dist.ReduceOp.MIN, "max": self.dist.ReduceOp.MAX}[op]
        self.dist.all_reduce(t, op=red)
        return [int(v) for v in t.tolist()]

    def buffer(self, nbytes: int):
        return self.torch.empty(nbytes, dtype=self.torch.uint8, device=self.device)

    def exchange(self, sends: dict, recvs: dict) -> None:
        """sends / recvs: peer rank -> buffer; all transfers of a step go out together."""
        ops = [self.dist.P2POp(self.dist.isend, b, peer) for peer, b in sends.items()]
        ops += [self.dist.P2POp(self.dist.irecv, b, peer) for peer, b in recvs.items()]
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()


def run_distributed(slab, comm, max_steps: int, random_nb: bool, initial_lava: int):
    """The step loop of one rank: step, sum the counts over the ranks, stop rule, halo exchange.
    Returns (steps, stop, active history, changed history), identical on every rank."""
    lay = slab.lay
    plan = message_plan(lay)
    L = slab.layer_cells
    bufs = {k: comm.buffer(message_bytes(v[1], v[2], L)) for k, v in plan.items()}
    stop = STOP_NO_LAVA if initial_lava == 0 else (STOP_MAX_STEPS if max_steps <= 0 else 0)
    steps, act, chg = 0, [], []
    while stop == 0:
        a, c = slab.step()
        a, c = comm.allreduce([a, c])
        steps += 1
        act.append(a)
        chg.append(c)
        stop = finish(steps, a, c, max_steps, random_nb)
        if stop:
            slab.stop(stop)
            break
        for key in ("send_up", "send_down"):
            if key in plan:
                slab.pack(*plan[key], bufs[key])
        sends = {lay.rank + 1: bufs["send_up"]} if "send_up" in plan else {}
        if "send_down" in plan:
            sends[lay.rank - 1] = bufs["send_down"]
        recvs = {lay.rank + 1: bufs["recv_up"]} if "recv_up" in plan else {}
        if "recv_down" in plan:
            recvs[lay.rank - 1] = bufs["recv_down"]
        comm.exchange(sends, recvs)
        for key in ("recv_up", "recv_down"):
            if key in plan:
                slab.unpack(*plan[key], bufs[key])
    return steps, stop, act, chg


def run_local(slabs: list, max_steps: int, random_nb: bool, initial_lava: int, buffer):
    """The same loop for every slab held by this process (e.g. several slabs on one GPU): the host
    steps them one after another, sums the counts, and moves each halo message through a buffer made
    by buffer(nbytes).  Returns (steps, stop, active history, changed history)."""
    plans = [message_plan(s.lay) for s in slabs]
    stop = STOP_NO_LAVA if initial_lava == 0 else (STOP_MAX_STEPS if max_steps <= 0 else 0)
    steps, act, chg = 0, [], []
    while stop == 0:
        a = c = 0
        for s in slabs:
            sa, sc = s.step()
            a += sa
            c += sc
        steps += 1
        act.append(a)
        chg.append(c)
        stop = finish(steps, a, c, max_steps, random_nb)
        if stop:
            for s in slabs:
                s.stop(stop)
            break
        for r, (s, plan) in enumerate(zip(slabs, plans)):
            for key, peer, into in (("send_up", r + 1, "recv_down"), ("send_down", r - 1, "recv_up")):
                if key not in plan:
                    continue
                z0, types, full = plan[key]
                buf = buffer(message_bytes(types, full, s.layer_cells))
                s.pack(z0, types, full, buf)
                slabs[peer].unpack(*plans[peer][into], buf)
    return steps, stop, act, chg


def assemble(parts: list) -> list:
    """The whole grid's five planes from the owned planes of every slab, bottom slab first."""
    return [np.concatenate([p[i] for p in parts]) for i in range(5)]


# ------------------------------------------------------------------------------------------
# MC stage over slabs
# ------------------------------------------------------------------------------------------
LAVA, BASALT = 2, 3


def mc_layout(lay: SlabLayout) -> tuple[int, int]:
    """Global layers [lo, hi) an MC slab holds: its owned layers and one halo layer on each side."""
    return max(0, lay.z0 - 1), min(lay.nz, lay.z1 + 1)


def basalt_domain(types) -> np.ndarray:
    """CoolingMobility::basaltDomain (CoolingMobility.cpp:8-14): BASALT or LAVA cells."""
    return ((types == BASALT) | (types == LAVA)).astype(np.uint8)


def local_end(planes) -> int:
    """This slab's share of CoolingMobility::endStep (CoolingMobility.cpp:16-25): the largest stamp
    of its owned domain cells (max-reduced over the slabs)."""
    t, _, _, so, ar = planes
    dom = basalt_domain(t) > 0
    return int(np.maximum(so[dom], ar[dom]).max()) if dom.any() else 0


def liquid_time(planes, end: int) -> np.ndarray:
    """CoolingMobility::liquidTime (CoolingMobility.cpp:31-45) of the owned cells, 0 outside the domain."""
    t, _, _, so, ar = planes
    dom = basalt_domain(t) > 0
    sol = np.where(t == BASALT, so.astype(np.int64), end)
    return np.where(dom, np.maximum(sol - ar.astype(np.int64), 0), 0)


def local_time_range(planes, end: int) -> tuple[int, int]:
    """This slab's (min, max) liquid time over its domain (min- / max-reduced over the slabs)."""
    dom = basalt_domain(planes[0]) > 0
    if not dom.any():
        return np.iinfo(np.int64).max, -1
    tm = liquid_time(planes, end)[dom]
    return int(tm.min()), int(tm.max())


def normalize(time, domain, tmin: int, tmax: int, mobility_min: float) -> np.ndarray:
    """CoolingMobility::normalize (CoolingMobility.cpp:62-77): double steps rounded one by one, then
    to float."""
    dom = domain.astype(bool)
    mob = np.zeros(len(domain), np.float32)
    if tmax < 0:
        return mob
    if tmax == tmin:
        mob[dom] = 1.0
        return mob
    norm = (time[dom] - tmin).astype(np.float64) / float(tmax - tmin)
    mob[dom] = (mobility_min + (1.0 - mobility_min) * norm).astype(np.float32)
    return mob


def mobility_terms(planes_of_slabs, reduce=None):
    """(end, tmin, tmax) of the whole domain: from the owned planes of every slab of this process,
    reduced further over the ranks by reduce(values, op) when given."""
    end = max(local_end(p) for p in planes_of_slabs)
    if reduce:
        end = reduce([end], "max")[0]
    ranges = [local_time_range(p, end) for p in planes_of_slabs]
    tmin, tmax = min(r[0] for r in ranges), max(r[1] for r in ranges)
    if reduce:
        tmin, tmax = reduce([tmin], "min")[0], reduce([tmax], "max")[0]
    return end, tmin, tmax


class McSlab:
    """One slab of the MC stage on this process's GPU (a vca_mc handle of nx x ny x held layers): the
    basalt of its owned layers, the cooling mobility from the whole domain's (end, tmin, tmax)."""

    def __init__(self, mcp: "capi.McParams", lay: SlabLayout, owned_planes, terms, mobility_min: float,
                 use_mobility: bool = True):
        lo, hi = mc_layout(lay)
        self.lay, self.lo, self.hi = lay, lo, hi
        self.L = mcp.nx * mcp.ny
        end, tmin, tmax = terms
        own_dom = basalt_domain(owned_planes[0])
        mob_own = normalize(liquid_time(owned_planes, end), own_dom, tmin, tmax, mobility_min)
        held = hi - lo
        dom = np.zeros(held * self.L, np.uint8)
        mob = np.zeros(held * self.L, np.float32)
        a, b = (lay.z0 - lo) * self.L, (lay.z1 - lo) * self.L
        dom[a:b] = own_dom
        mob[a:b] = mob_own
        self.mc = capi.PottsMC(capi.McParams(**{**mcp.__dict__, "nz": held}))
        self.mc.set_slab(lo)
        self.mc.set_domain(dom)
        self.mc.set_mobility(mob if use_mobility else None)
        self.mc.initialize()
        self.colors = self.mc.info().colors

    def plan(self) -> dict:
        """Halo layers in local z: up (to rank + 1) the top owned layer into its lower halo, down (to
        rank - 1) the lowest owned layer into its upper halo."""
        lay, lo = self.lay, self.lo
        p = {}
        if lay.rank + 1 < lay.world:
            p["send_up"] = lay.z1 - 1 - lo
            p["recv_up"] = lay.z1 - lo
        if lay.rank > 0:
            p["send_down"] = lay.z0 - lo
            p["recv_down"] = lay.z0 - 1 - lo
        return p

    def color_pass(self, c: int) -> None:
        self.mc.color_pass(c)

    def pack(self, z, buf):
        self.mc.pack_spins(z, 1, buf.data_ptr())

    def unpack(self, z, buf):
        self.mc.unpack_spins(z, 1, buf.data_ptr())

    def counters(self) -> tuple[int, int, int]:
        i = self.mc.info()
        return i.attempts, i.accepted, i.uphill

    def owned_spins(self) -> np.ndarray:
        c = self.mc.crystals()
        return c[(self.lay.z0 - self.lo) * self.L:(self.lay.z1 - self.lo) * self.L]

    def close(self):
        self.mc.close()


def run_mc_local(mslabs: list, sweeps: int, buffer) -> None:
    """`sweeps` checkerboard MCS on the MC slabs of this process: each colour on every slab, then the
    boundary layers of orientations move to the neighbours' halos (an exchange also comes first,
    so the halos hold the initial orientations)."""
    def exchange():
        for r, s in enumerate(mslabs):
            p = s.plan()
            for key, peer, into in (("send_up", r + 1, "recv_down"), ("send_down", r - 1, "recv_up")):
                if key in p:
                    buf = buffer(4 * s.L)
                    s.pack(p[key], buf)
                    mslabs[peer].unpack(mslabs[peer].plan()[into], buf)
    exchange()
    colors = mslabs[0].colors
    for _ in range(sweeps):
        for c in range(colors):
            for s in mslabs:
                s.color_pass(c)
            exchange()


def run_mc_distributed(mslab, comm, sweeps: int) -> None:
    """The same loop on one rank; halo layers over comm (torch.distributed)."""
    p = mslab.plan()
    bufs = {k: comm.buffer(4 * mslab.L) for k in p}
    lay = mslab.lay

    def exchange():
        for key in ("send_up", "send_down"):
            if key in p:
                mslab.pack(p[key], bufs[key])
        sends = {}
        recvs = {}
        if "send_up" in p:
            sends[lay.rank + 1] = bufs["send_up"]
            recvs[lay.rank + 1] = bufs["recv_up"]
        if "send_down" in p:
            sends[lay.rank - 1] = bufs["send_down"]
            recvs[lay.rank - 1] = bufs["recv_down"]
        comm.exchange(sends, recvs)
        for key in ("recv_up", "recv_down"):
            if key in p:
                mslab.unpack(p[key], bufs[key])
    exchange()
    for _ in range(sweeps):
        for c in range(mslab.colors):
            mslab.color_pass(c)
            exchange()
