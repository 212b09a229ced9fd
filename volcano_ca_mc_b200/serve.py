"""Batched and served execution of many independent lava CA + Potts MC jobs on one GPU, through the
job server of the engine command (``engine --serve``, volcano_ca_mc_b200/csrc/engine/serve.cpp).

The reference runs one job per engine process (its batch runner starts the engine once per config,
engine/src/app/Batch.cpp:147-246; its GUI queue, gui/jobs.py, starts one job after another).  Here
the jobs are engine configs in the reference's schema, sent to one server process as they arrive:

* each job is a config object (space, boundary, neighbourhood, seed, a CSV heightmap of Gaussian
  cones with value noise, vents at given columns, ca.* and mc.* parameters) with ``output.format``
  none: the server answers with digests of its ca_result.bin / mc_result.bin bytes;
* the server admits a job when a worker is free and its resident device handles fit the HBM budget,
  steps the CA grids of all running jobs together in one batch, and runs each job's MC stage and
  statistics on the worker's own streams;
* ``run(..., slots=1, batched=False)`` is the one-at-a-time plain GPU path on the same trace
  (vca_ca_run per job, no overlap), the baseline of the jobs/s and latency figures.

Every job's result is a pure function of its config, so its digests are the same alone and in the
mix (``compare``).

The mixes follow the batched/served benchmark definitions: 2D x-z sections with sides drawn
log-uniformly from 128 to 2048, 3D grids with sides from 64 to 256 and z = side / 2, all four
neighbourhoods (hexagonal in 2D only), both boundaries, 1-8 vents on Gaussian-cone terrain, Q in
{32, 64, 128}, 200-600 CA steps and 20-100 MC sweeps, drawn from a recorded master seed.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile
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
            if not vents:  # every pick landed on a full column: the lowest column instead
                y0, x0 = np.unravel_index(int(np.argmin(hm)), hm.shape)
                vents = [(int(x0), int(y0), int(hm[y0, x0]), 1)]
            self._terrain = (heights, vents)
        return self._terrain

    def footprint(self) -> int:
        return capi.ca_footprint(self.ca_params()) + capi.mc_footprint(self.mc_params())

    def config(self, folder: str) -> dict:
        """The job as an engine config in the reference's schema (engine/src/io/Config.cpp:153-176):
        its heightmap written as a CSV file into folder (terrain.type = "file"), vents at its columns."""
        heights, vents = self.terrain()
        csv = os.path.join(folder, f"job{self.job_id}_heightmap.csv")
        if not os.path.exists(csv):
            with open(csv, "w") as f:
                for row in heights.reshape(self.ny, self.nx):
                    f.write(",".join(str(int(v)) for v in row) + "\n")
        return {
            "space": {"nx": self.nx, "ny": self.ny, "nz": self.nz}, "boundary": self.boundary,
            "neighborhood": self.neighborhood, "rngSeed": self.seed,
            "terrain": {"type": "file", "file": csv},
            "vents": {"count": len(vents), "placement": "positions", "positions": [[v[0], v[1]] for v in vents],
                      "eruptionSteps": self.max_steps // 2, "eruptTemp": 1200},
            "ca": {"mode": "lava", "maxSteps": self.max_steps, "coolingAmbient": 2.0, "coolingLateral": 4.0,
                   "coolingFall": 2.0, "solidusTemp": 800, "ponding": True, "sweep": "front"},
            "mc": {"enabled": True, "domain": "basalt", "Q": self.Q, "mcs": self.mcs, "J": 1.0, "kT": self.kT,
                   "mobilityFromCooling": True, "statsEvery": max(1, self.mcs), "update": "checkerboard"},
            "output": {"format": "none"},
        }


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



class EngineServer:
    """One ``engine --serve`` process: requests go to its standard input as JSON lines, its answers
    are collected by a reader thread."""

    def __init__(self, slots: int = 16, batched: bool = True, budget_gb: float = 120.0, device: int = 0):
        args = [capi.ENGINE_PATH, "--serve", "--slots", str(slots), "--budget-gb", f"{budget_gb:g}"]
        if not batched:
            args.append("--no-batch")
        if not os.path.exists(capi.ENGINE_PATH):
            raise capi.VcaError(f"{capi.ENGINE_PATH} is missing: the engine has not been built")
        self.proc = subprocess.Popen(args, stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                     text=True, bufsize=1, env=dict(os.environ, VCA_DEVICE=str(device)))
        self.answers: dict[str, dict] = {}
        self.summary: dict | None = None
        self._err: list[str] = []
        self._reader = threading.Thread(target=self._read, daemon=True)
        self._reader.start()
        self._err_reader = threading.Thread(target=lambda: self._err.extend(self.proc.stderr), daemon=True)
        self._err_reader.start()

    def _read(self):
        for line in self.proc.stdout:
            d = json.loads(line)
            if "summary" in d:
                self.summary = d["summary"]
            else:
                self.answers[str(d["id"])] = d

    def submit(self, request: dict) -> None:
        self.proc.stdin.write(json.dumps(request) + "\n")
        self.proc.stdin.flush()

    def close(self, timeout: float = 3600.0) -> int:
        self.proc.stdin.close()
        rc = self.proc.wait(timeout=timeout)
        self._reader.join(timeout=10)
        self._err_reader.join(timeout=10)
        return rc

    def stderr(self) -> str:
        return "".join(self._err)


def run(jobs: list[JobSpec], slots: int = 16, batched: bool = True, budget_gb: float = 120.0, realtime: bool = False,
        device: int = 0, folder: str | None = None) -> dict:
    """Sends the jobs to a job server (at their arrival times when realtime, else all at once) and
    returns per-job records and totals: jobs/s over the makespan (first arrival to last completion),
    cell-updates/s, p50 / p99 of completion - arrival, mean concurrency."""
    tmp = None
    if folder is None:
        tmp = tempfile.TemporaryDirectory(prefix="vca_serve_")
        folder = tmp.name
    try:
        order = sorted(jobs, key=lambda j: j.arrival_s)
        configs = {j.job_id: j.config(folder) for j in order}  # terrains and heightmaps before the trace
        srv = EngineServer(slots=slots, batched=batched, budget_gb=budget_gb, device=device)
        t0 = time.perf_counter()
        for j in order:
            if realtime:
                delay = j.arrival_s - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            srv.submit({"id": str(j.job_id), "json": configs[j.job_id]})
        rc = srv.close()
        if rc != 0 or srv.summary is None:
            raise RuntimeError(f"engine --serve ended with {rc}: {srv.stderr()[-2000:]} "
                               f"{[a for a in srv.answers.values() if a.get('status') != 'ok'][:3]}")
    finally:
        if tmp is not None:
            tmp.cleanup()
    recs = {int(k): v for k, v in srv.answers.items()}
    first = min(r["arrival_ms"] for r in recs.values())
    last = max(r["done_ms"] for r in recs.values())
    makespan = (last - first) / 1e3
    lat = np.array([r["latency_ms"] / 1e3 for r in recs.values()])
    busy = sum(r["done_ms"] - r["admitted_ms"] for r in recs.values()) / 1e3
    phases = phase_sums(recs.values())
    return {"records": recs, "slots": slots, "batched": batched, "jobs": len(recs), "makespan_s": makespan,
            "jobs_per_s": len(recs) / makespan if makespan > 0 else 0.0,
            "cell_updates_per_s": sum(r["cell_updates"] for r in recs.values()) / makespan if makespan > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_concurrency": busy / makespan if makespan > 0 else 0.0, "server": srv.summary,
            "phases_ms": phases}


def phase_sums(records) -> dict[str, float]:
    """The per-section times of the answers (`times_ms`: times.json sections, MC set-up details,
    digest) summed over the jobs, in ms."""
    sums: dict[str, float] = {}
    for r in records:
        for k, v in r.get("times_ms", {}).items():
            sums[k] = sums.get(k, 0.0) + float(v)
    return {k: round(v, 3) for k, v in sums.items()}


def compare(a: dict, b: dict) -> int:
    """Number of jobs whose results (digests of ca_result.bin and mc_result.bin) differ between two
    runs of the same jobs."""
    ra, rb = a["records"], b["records"]
    return sum(1 for k in ra if ra[k]["digest"] != rb.get(k, {}).get("digest"))
