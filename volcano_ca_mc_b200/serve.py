"""Batched and served execution of many independent lava CA + Potts MC jobs on one GPU.

The reference runs one job per engine process (its batch runner starts the engine once per config,
engine/src/app/Batch.cpp:147-246; its GUI queues jobs one after the other).  Here a job server keeps
a fixed number of worker slots, each with a resident CA handle and a resident MC handle on its own
CUDA streams, sized once for the largest job of the mix:

* a job is admitted when a slot is free and the device bytes of the running jobs plus its own
  (``vca_ca_footprint`` + ``vca_mc_footprint``) stay within the HBM budget;
* an admitted job reconfigures its slot's handles to its space and parameters
  (``vca_ca_reconfigure`` / ``vca_mc_reconfigure``: no allocation), runs the CA to its stop rule,
  crystallises the basalt, computes the grain statistics on the device and returns its planes;
* jobs that arrive while others run are admitted as slots free up, so the short, latency-bound
  launches of many small grids overlap on the GPU (continuous batching).

``run(jobs, slots=1)`` is the one-at-a-time baseline on the same trace.  Every job's result is a
pure function of its spec, so a job's result hash is the same alone and in the mix (checked by
``compare``).

The mixes follow the batched/served benchmark definitions: 2D x-z sections with sides drawn
log-uniformly from 128 to 2048, 3D grids with sides from 64 to 256 and z = side / 2, all four
neighbourhoods (hexagonal in 2D only), both boundaries, 1-8 vents on Gaussian-cone terrain, Q in
{32, 64, 128}, 200-600 CA steps and 20-100 MC sweeps, drawn from a recorded master seed.
"""
from __future__ import annotations

import hashlib
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .workloads import _finish, value_noise


@dataclass
class JobSpec:
    job_id: int
    nx: int
    ny: int
    nz: int
    neighborhood: str
    boundary: str
    seed: int
    max_steps: int
    n_vents: int
    Q: int
    kT: float
    mcs: int
    arrival_s: float = 0.0
    _terrain: tuple | None = field(default=None, repr=False)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def ca_params(self, device: int = 0) -> capi.CaParams:
        return capi.CaParams(self.nx, self.ny, self.nz, neighborhood=self.neighborhood, boundary=self.boundary,
                             seed=self.seed, max_steps=self.max_steps, eruption_steps=self.max_steps // 2,
                             cooling_ambient=2.0, cooling_lateral=4.0, cooling_fall=2.0, device=device)

    def mc_params(self, device: int = 0) -> capi.McParams:
        return capi.McParams(self.nx, self.ny, self.nz, neighborhood=self.neighborhood, boundary=self.boundary,
                             seed=self.seed, Q=self.Q, J=1.0, kT=self.kT, device=device)

    def terrain(self):
        """Heights (int32, nx*ny) and vents [(x, y, z, flowId)]: 1-3 Gaussian cones with value noise,
        vents near the cone summits on columns with room above the terrain."""
        if self._terrain is None:
            rng = np.random.default_rng(self.seed)
            nx, ny, nz = self.nx, self.ny, self.nz
            x = np.arange(nx)[None, :]
            y = np.arange(ny)[:, None]
            h = np.zeros((ny, nx))
            centres = []
            for _ in range(int(rng.integers(1, 4))):
                cx, cy = rng.uniform(0.2, 0.8) * nx, (rng.uniform(0.2, 0.8) * ny if ny > 1 else 0.0)
                peak = rng.uniform(0.3, 0.7) * nz
                sig = rng.uniform(0.12, 0.3) * max(nx, ny)
                h += peak * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sig * sig))
                centres.append((cx, cy))
            h += 0.02 * nz * value_noise(nx, ny, self.seed)
            heights = _finish(h, nz)
            hm = heights.reshape(ny, nx)
            vents, used = [], set()
            for i in range(self.n_vents):
                cx, cy = centres[i % len(centres)]
                for _ in range(64):
                    vx = int(np.clip(cx + rng.normal(0, 3), 0, nx - 1))
                    vy = int(np.clip(cy + rng.normal(0, 3), 0, ny - 1)) if ny > 1 else 0
                    if (vx, vy) not in used and hm[vy, vx] < nz:
                        break
                used.add((vx, vy))
                vents.append((vx, vy, int(hm[vy, vx]), i + 1))
            vents = [v for v in vents if v[2] < nz]
            self._terrain = (heights, vents)
        return self._terrain

    def footprint(self) -> int:
        return capi.ca_footprint(self.ca_params()) + capi.mc_footprint(self.mc_params())


def make_mix(n: int, master_seed: int, share_3d: float = 0.3, rate_hz: float | None = None, side_2d=(128, 2048),
             side_3d=(64, 256), steps=(200, 600), mcs=(20, 100)) -> list[JobSpec]:
    """n jobs drawn from the batched-benchmark distribution (the size ranges can be narrowed for
    tests); with rate_hz, Poisson arrival times."""
    rng = np.random.default_rng(master_seed)
    jobs, t = [], 0.0
    for j in range(n):
        three_d = rng.random() < share_3d
        if three_d:
            s = int(round(np.exp(rng.uniform(np.log(side_3d[0]), np.log(side_3d[1])))))
            nx, ny, nz = s, s, max(8, s // 2)
            nb = ["von_neumann", "moore", "pentagonal"][int(rng.integers(0, 3))]
        else:
            nx = int(round(np.exp(rng.uniform(np.log(side_2d[0]), np.log(side_2d[1])))))
            nz = int(round(np.exp(rng.uniform(np.log(side_2d[0]), np.log(side_2d[1])))))
            ny = 1
            nb = ["von_neumann", "moore", "pentagonal", "hexagonal"][int(rng.integers(0, 4))]
        if rate_hz:
            t += float(rng.exponential(1.0 / rate_hz))
        jobs.append(JobSpec(job_id=j, nx=nx, ny=ny, nz=nz, neighborhood=nb,
                            boundary=["absorbing", "periodic"][int(rng.integers(0, 2))],
                            seed=int(rng.integers(1, 2**31)), max_steps=int(rng.integers(steps[0], steps[1] + 1)),
                            n_vents=int(rng.integers(1, 9)), Q=int(rng.choice([32, 64, 128])),
                            kT=float(rng.choice([0.0, 0.3, 0.6])), mcs=int(rng.integers(mcs[0], mcs[1] + 1)),
                            arrival_s=t))
    return jobs


class ResultBuffers:
    """Pinned host buffers that jobs' results are downloaded into and handed to the consumer in.
    A slot takes a free buffer set for each job and is released as soon as the result is in it; the
    consumer (here the result hash) returns the set when it is done, so a slow consumer holds back
    new jobs only when every set is taken."""

    def __init__(self, cap_cells: int, count: int):
        import torch
        pin = lambda dt: torch.empty(cap_cells, dtype=dt, pin_memory=True).numpy()
        self.free: queue.Queue = queue.Queue()
        for _ in range(count):
            self.free.put((pin(torch.uint8), pin(torch.int32), pin(torch.float32), pin(torch.int16).view("uint16"),
                           pin(torch.int16).view("uint16"), pin(torch.int32)))

    def get(self):
        return self.free.get()

    def put(self, bufs):
        self.free.put(bufs)


class Slot:
    """A worker's resident CA and MC handles, sized for the largest job it may get."""

    def __init__(self, cap: JobSpec, device: int):
        self.device = device
        self.ca = capi.LavaCA(cap.ca_params(device))
        self.mc = capi.PottsMC(cap.mc_params(device))
        # one small job first: the handles' set-up buffers are allocated on first use, sized for the
        # capacity, so no job of the trace waits on a device-wide allocation
        three_d = cap.ny > 1
        self.run(JobSpec(job_id=-2, nx=32 if three_d else 64, ny=32 if three_d else 1, nz=16 if three_d else 64,
                         neighborhood="moore", boundary="absorbing", seed=1, max_steps=8, n_vents=1, Q=32, kT=0.0,
                         mcs=1))

    def run(self, job: JobSpec, bufs=None) -> tuple[dict, tuple]:
        """Runs the job; returns its record and its result arrays (the five CA planes and the crystal
        orientations, views of ``bufs`` when given)."""
        t = [time.perf_counter()]
        heights, vents = job.terrain()
        self.ca.reconfigure(job.ca_params(self.device))
        self.ca.apply_terrain(heights)
        self.ca.place_seeds(vents)
        t.append(time.perf_counter())
        self.ca.run()
        info = self.ca.info()
        lava, basalt, reach2 = self.ca.flow_stats(len(vents))
        t.append(time.perf_counter())
        n = job.cells
        planes = self.ca.download(None if bufs is None else tuple(a[:n] for a in bufs[:5]))
        t.append(time.perf_counter())
        self.mc.reconfigure(job.mc_params(self.device))
        self.mc.set_domain_from_ca(self.ca)
        self.mc.set_mobility_from_ca(self.ca, 0.05, True)
        self.mc.initialize()
        self.mc.sweep(job.mcs)
        g = self.mc.grains(moore=job.neighborhood != "von_neumann")
        crystals = self.mc.crystals(None if bufs is None else bufs[5][:n])
        mi = self.mc.info()
        energy = self.mc.energy()
        t.append(time.perf_counter())
        rec = {"job": job.job_id, "steps": info.steps, "stop": info.stop_reason, "energy": energy, "grains": g.grains,
               "lava_volume": int(lava.sum() + basalt.sum()), "max_reach": round(float(np.sqrt(reach2.max())), 2),
               "attempts": mi.attempts, "cell_updates": job.cells * info.steps, "done": t[-1],
               "phases_ms": {k: round((t[i + 1] - t[i]) * 1e3, 3)
                             for i, k in enumerate(("setup", "ca", "download", "mc"))}}
        return rec, (*planes, crystals)

    def close(self):
        self.mc.close()
        self.ca.close()


def result_hash(arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(memoryview(np.ascontiguousarray(a)).cast("B"))
    return h.hexdigest()[:24]


def capacity(jobs: list[JobSpec]) -> JobSpec:
    """A spec whose handles hold every job of the list (all 2D or all 3D): the largest size on each
    axis and the longest step history; the buffer sizes grow with each axis, so every job fits."""
    return JobSpec(job_id=-1, nx=max(j.nx for j in jobs), ny=max(j.ny for j in jobs), nz=max(j.nz for j in jobs),
                   neighborhood="moore", boundary="absorbing", seed=1, max_steps=65535, n_vents=1, Q=2, kT=0.0, mcs=0)


def run(jobs: list[JobSpec], slots: int = 8, budget_bytes: int = 120 << 30, realtime: bool = False,
        device: int = 0) -> dict:
    """Run the jobs on `slots` workers with footprint admission; realtime replays the arrival times.
    Returns per-job records (arrival, start, end in seconds from the trace start, result) and totals."""
    by_dim = {"2d": [j for j in jobs if j.ny == 1], "3d": [j for j in jobs if j.ny > 1]}
    caps = {k: capacity(v) for k, v in by_dim.items() if v}
    per_slot = sum(capi.ca_footprint(c.ca_params()) + capi.mc_footprint(c.mc_params()) for c in caps.values())
    slots = max(1, min(slots, budget_bytes // max(1, per_slot)))
    pool: queue.Queue = queue.Queue()
    for _ in range(slots):
        pool.put({k: Slot(c, device) for k, c in caps.items()})
    results = {k: ResultBuffers(c.cells, slots + 4) for k, c in caps.items()}
    lock = threading.Condition()
    in_use = [0]
    records: dict[int, dict] = {}
    errors: list[BaseException] = []
    order = sorted(jobs, key=lambda j: j.arrival_s)
    for j in order:  # host-side set-up outside the trace (terrain synthesis)
        j.terrain()
    t0 = time.perf_counter()

    def worker(job: JobSpec, slot_set: dict, start: float, fp: int):
        dim = "3d" if job.ny > 1 else "2d"
        bufs = results[dim].get()
        rec = None
        try:
            rec, arrays = slot_set[dim].run(job, bufs)
        except BaseException as e:  # reported after the run
            errors.append(e)
        finally:  # the slot is free once the result is in host memory
            pool.put(slot_set)
            with lock:
                in_use[0] -= fp
                lock.notify_all()
        try:  # the consumer: checks the result, then gives the buffers back
            if rec is not None:
                rec["sha"] = result_hash(arrays)
                records[job.job_id] = {"arrival": job.arrival_s, "start": start, "end": rec.pop("done") - t0, **rec}
        except BaseException as e:
            errors.append(e)
        finally:
            results[dim].put(bufs)

    threads = []
    for job in order:
        if realtime:
            delay = job.arrival_s - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
        fp = job.footprint()
        slot_set = pool.get()  # a free slot
        with lock:
            while in_use[0] + fp > budget_bytes and in_use[0] > 0:
                lock.wait(timeout=1.0)
            in_use[0] += fp
        th = threading.Thread(target=worker, args=(job, slot_set, time.perf_counter() - t0, fp), daemon=True)
        th.start()
        threads.append(th)
    for th in threads:
        th.join()
    while not pool.empty():
        for s in pool.get().values():
            s.close()
    if errors:
        raise errors[0]
    makespan = max((r["end"] for r in records.values()), default=0.0)  # the last result in host memory
    lat = np.array([r["end"] - (r["arrival"] if realtime else 0.0) for r in records.values()])
    busy = sum(r["end"] - r["start"] for r in records.values())
    phases = {}
    for r in records.values():
        for k, v in r["phases_ms"].items():
            phases[k] = phases.get(k, 0.0) + v
    return {"records": records, "slots": slots, "makespan_s": makespan, "jobs": len(records),
            "mean_concurrency": busy / makespan if makespan > 0 else 0.0,
            "phase_ms_total": {k: round(v, 1) for k, v in phases.items()},
            "jobs_per_s": len(records) / makespan if makespan > 0 else 0.0,
            "cell_updates_per_s": sum(r["cell_updates"] for r in records.values()) / makespan if makespan > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else 0.0,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else 0.0,
            "per_slot_bytes": per_slot, "budget_bytes": budget_bytes}


def compare(a: dict, b: dict) -> int:
    """Number of jobs whose results differ between two runs of the same jobs."""
    ra, rb = a["records"], b["records"]
    return sum(1 for k in ra if ra[k]["sha"] != rb.get(k, {}).get("sha"))
