#!/usr/bin/env python
"""Benchmark of the lava-CA + Potts-MC hot paths on B200 (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3] [--impl ours|reference]

A step is one job of the workload: the lava CA run from the seeded terrain to its stop rule (for
c3, 800 steps of a 1024 x 1024 x 256 grid, random pentagonal neighbourhood) followed by the Potts
checkerboard crystallisation of the basalt it left (200 MCS).  The jobs run on resident handles:
terrain and vents are in HBM when a job's timed region starts; L2 is flushed before every CA run
and MC run, outside their device events (c3's 7 GB of state is far larger than L2 anyway).

  value          CA cell-updates/s = cells x CA steps / CA device time (ACTIVE schedule), all ranks.
  parity         the last timed job's ca_result.bin / mc_result.bin bytes (SHA-256) against the reference
                 engine's run of the same config (tests/golden/<workload>_large), computed after timing.
  mc             MC trials/s and attempts/s of the same jobs (attempts exclude mobility skips).
  dense          the same job with the DENSE schedule (every cell every step).
  roofline       the rules kernel of the DENSE job: 26 B per cell (13 B state read + 13 B written) over
                 its CUDA-event launch time, against the measured HBM copy bandwidth; traffic = ncu DRAM
                 bytes per cell of the same kernel on the c3q case (profiles/), times the cells of a launch.
  kernels_ms     device time per step of the drop-depth, rules and candidate kernels.
  e2e            the same metric through the C ABI with host buffers: reset, terrain and vents from host
                 memory, run, all five planes back into pinned host memory, host wall clock over a run of
                 jobs with two in flight (one computing, the other's planes copying); one_at_a_time beside it.
  cpu_baseline   the reference engine (oracle/_ref/engine, --threads = host cores) on one full job.
  c2             the 256 x 256 x 128 workload: ACTIVE / DENSE figures and its parity.
  batched/served many small independent jobs through the job server (volcano_ca_mc_b200.serve).

With --impl reference the reference engine itself is timed on the host cores (rank 0 only).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import struct
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0
BYTES_PER_CELL_UPDATE = 26   # 13 B state read + 13 B next state written
BYTES_PER_TRIAL = 12         # spin read + spin write + mobility read
# The reference arm's bounded sample: the first REF_SAMPLE_STEPS CA steps of the workload's job (its
# front sweep runs from step 0 only: the reference engine has no resume), MC off.
REF_SAMPLE_STEPS = {"c1": 300, "c2": 400, "c3": 300, "c3q": 300}
# jobs in flight in the e2e measurement: one computing while the other's planes travel
E2E_INFLIGHT = 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c2", action="store_true", help="skip the 256x256x128 sub-benchmark")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched job-mix sub-benchmark")
    ap.add_argument("--no-served", action="store_true", help="skip the served (Poisson arrivals) sub-benchmark")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="length of the served arrival trace")
    ap.add_argument("--slots", type=int, default=16, help="workers of the job server in the batched and served runs")
    ap.add_argument("--serve-rates", type=float, nargs="*", default=[20.0, 60.0, 120.0, 240.0],
                    help="arrival rates [jobs/s] of the served sweep")
    ap.add_argument("--sweep-seconds", type=float, default=4.0, help="length of each trace of the served sweep")
    ap.add_argument("--profile-job", choices=["active", "dense", "mc", "mcfull"], default=None,
                    help="run exactly one CA job with this schedule (no warm-up, no MC), or with mc one ACTIVE "
                         "CA job and its MC stage, or with mcfull the whole-space MC case (--max-steps sweeps), "
                         "and exit: the case ncu captures")
    ap.add_argument("--max-steps", type=int, default=None, help="with --profile-job: stop the CA after this many steps")
    ap.add_argument("--slabs", action="store_true",
                    help="with --gpus N > 1: one grid of the workload split into N z slabs (strong scaling, halo "
                         "exchange over NCCL) instead of N independent replicas")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(values, device, world):
    """Element-wise maximum of per-rank timings over all ranks (the job is as slow as its slowest
    replica); a no-op for one rank.  The process group must be initialised when world > 1."""
    if world <= 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def ncu_traffic_per_cell(kernel: str, workload: str, schedule: str):
    """DRAM bytes per processed cell of a kernel launch from the committed ncu summaries (profiles/*.md
    lines `traffic: kernel=<k> workload=<w> schedule=<s> bytes_per_launch=<n> cells_per_launch=<c>`),
    or None."""
    import glob
    import re
    pat = re.compile(r"traffic:\s*kernel=(\S+)\s+workload=(\S+)\s+schedule=(\S+)\s+bytes_per_launch=(\d+)"
                     r"\s+cells_per_launch=(\d+)")
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for line in f:
                m = pat.search(line)
                if m and m.group(1) == kernel and m.group(2) == workload and m.group(3) == schedule:
                    return int(m.group(4)) / int(m.group(5)), m.group(2)
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def config_of(w) -> dict:
    """The workload as both arms name it (identical keys and values in the two JSON lines)."""
    return {"workload": f"{w.name}: {w.description}", "grid": [w.nx, w.ny, w.nz], "neighborhood": w.neighborhood,
            "boundary": w.boundary, "ca_max_steps": w.max_steps,
            "mc": f"Q={w.Q} kT={w.kT} {w.mcs} MCS checkerboard, cooling mobility",
            "step": "one job: the CA run to its stop rule, then the MC crystallisation of its basalt",
            "inputs": "seeded synthetic terrain written as the reference's CSV heightmap"}


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------
def ca_params(w, sweep, device):
    from volcano_ca_mc_b200 import capi
    return capi.CaParams(w.nx, w.ny, w.nz, neighborhood=w.neighborhood, boundary=w.boundary, seed=w.seed,
                         max_steps=w.max_steps, sweep=sweep, device=device)


def mc_params(w, device):
    from volcano_ca_mc_b200 import capi
    return capi.McParams(w.nx, w.ny, w.nz, neighborhood=w.neighborhood, boundary=w.boundary, seed=w.seed, Q=w.Q,
                         J=1.0, kT=w.kT, device=device)


class L2Flush:
    """Writes a buffer larger than L2 (126 MB) between runs."""

    def __init__(self, device):
        import torch
        self.buf = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{device}")

    def __call__(self):
        import torch
        self.buf.fill_(1)
        torch.cuda.synchronize()


class Resident:
    """One CA handle and one MC handle of a workload, kept for job after job (vca_ca_reset /
    vca_mc_reconfigure between jobs: nothing is allocated per job).  run() does one job and returns
    its device-timed figures: CA time from the handle's CUDA events around its step launches, MC time
    likewise, launch counts and trial counters as deltas."""

    def __init__(self, w, sweep, device, profile=False):
        from volcano_ca_mc_b200 import capi
        self.w, self.device = w, device
        if profile:
            os.environ["VCA_PROFILE_KERNELS"] = "1"
        try:
            self.ca = capi.LavaCA(ca_params(w, sweep, device))
        finally:
            os.environ.pop("VCA_PROFILE_KERNELS", None)
        self.mc = None
        self.fresh = True

    def run(self, flush, mc=True):
        w, ca = self.w, self.ca
        if not self.fresh:
            ca.reset()
        self.fresh = False
        ca.apply_terrain(w.heights)
        ca.place_seeds(w.vent_cells())
        t0, _, _ = ca.timing()
        l0 = ca.info().kernel_launches
        flush()
        ca.run()
        t1, rules_ms, rules_n = ca.timing()
        info = ca.info()
        out = {"ca_ms": t1 - t0, "steps": info.steps, "stop": info.stop_reason, "launches": info.kernel_launches - l0,
               "tiles": info.tiles_processed, "cells_per_tile": info.cells_per_tile, "tiles_total": info.tiles_total,
               "rules_ms": rules_ms, "rules_n": rules_n, "mc": None}
        if mc:
            from volcano_ca_mc_b200 import capi
            if self.mc is None:
                self.mc = capi.PottsMC(mc_params(w, self.device))
            else:
                self.mc.reconfigure(mc_params(w, self.device))
            m = self.mc
            m.set_domain_from_ca(ca)
            m.set_mobility_from_ca(ca, 0.05, True)
            m.initialize()
            a0, l0m = m.info().attempts, m.info().kernel_launches
            m0, _, _ = m.timing()
            flush()
            m.sweep(w.mcs)
            mi = m.info()
            m1, _, _ = m.timing()
            out["mc"] = {"ms": m1 - m0, "trials": mi.domain_cells * w.mcs, "attempts": mi.attempts - a0,
                         "launches": mi.kernel_launches - l0m, "domain_cells": mi.domain_cells}
        return out

    def parity(self):
        """SHA-256 of this job's ca_result.bin and mc_result.bin bytes (ResultWriter.cpp:155-167,
        204-213) against the reference engine's run of the same config, when a golden exists."""
        import numpy as np
        w = self.w
        gold = os.path.join(ROOT, "tests", "golden", f"{w.name}_large", "expect.json")
        if not os.path.exists(gold):
            return {"checked": False, "reason": f"no golden for {w.name}"}
        with open(gold) as f:
            exp = json.load(f)
        h = hashlib.sha256(b"VOLC" + struct.pack("<Iiii", 2, w.nx, w.ny, w.nz))
        for plane in self.ca.download():
            h.update(memoryview(np.ascontiguousarray(plane)).cast("B"))
        ca_ok = h.hexdigest() == exp["files"]["ca_result.bin"]
        act, chg = self.ca.history()
        hist_ok = act == exp["activeCells"] and chg == exp["changedCells"]
        mc_ok = None
        if self.mc is not None:
            hm = hashlib.sha256(b"VMC1" + struct.pack("<iii", w.nx, w.ny, w.nz))
            hm.update(memoryview(self.mc.crystals()).cast("B"))
            mc_ok = hm.hexdigest() == exp["files"]["mc_result.bin"]
        return {"checked": True, "golden": f"tests/golden/{w.name}_large (reference engine, same config)",
                "ca_result.bin": "match" if ca_ok else "MISMATCH", "histories": "match" if hist_ok else "MISMATCH",
                "mc_result.bin": None if mc_ok is None else ("match" if mc_ok else "MISMATCH"),
                "ok": bool(ca_ok and hist_ok and mc_ok is not False)}

    def close(self):
        if self.mc is not None:
            self.mc.close()
        self.ca.close()


class E2E:
    """The call sequence of a job through the C ABI: reset, terrain and vents from host memory, run to
    the stop rule, all five planes back into pinned host memory.  Jobs go through `inflight` resident
    handles, each driven by a host thread of its own; a lock admits one vca_ca_run at a time, so every
    job computes with the whole GPU to itself while the previous job's planes travel back to the host
    and the next job's terrain goes up (the job server's form).  With inflight = 1 this is the plain
    one-at-a-time sequence.  Handles and pinned buffers are set up once, outside the timed jobs."""

    def __init__(self, w, device, inflight=1):
        import torch
        from volcano_ca_mc_b200 import capi
        self.w = w
        n = w.cells
        pin = lambda dt: torch.empty(n, dtype=dt, pin_memory=True).numpy()
        self.slots = []
        for _ in range(inflight):
            ca = capi.LavaCA(ca_params(w, capi.SWEEP_ACTIVE, device))
            out = (pin(torch.uint8), pin(torch.int32), pin(torch.float32), pin(torch.int16).view("uint16"),
                   pin(torch.int16).view("uint16"))
            self.slots.append((ca, out))
        self.heights = torch.from_numpy(w.heights.copy()).pin_memory().numpy()
        self.vents = w.vent_cells()

    def jobs(self, count):
        """`count` jobs; returns (wall ms of all of them, CA steps summed, per-phase medians in ms)."""
        run_lock, take_lock = threading.Lock(), threading.Lock()
        todo = [count]
        phases, steps, errors = [], [], []

        def worker(ca, out):
            try:
                while True:
                    with take_lock:
                        if todo[0] == 0:
                            return
                        todo[0] -= 1
                    t0 = time.perf_counter()
                    ca.reset()
                    ca.apply_terrain(self.heights)
                    ca.place_seeds(self.vents)
                    t1 = time.perf_counter()
                    with run_lock:
                        t2 = time.perf_counter()
                        ca.run()
                        t3 = time.perf_counter()
                    ca.download(out)
                    t4 = time.perf_counter()
                    steps.append(ca.info().steps)
                    phases.append((t1 - t0, t3 - t2, t4 - t3))
            except Exception as e:  # noqa: BLE001
                errors.append(e)

        threads = [threading.Thread(target=worker, args=s) for s in self.slots]
        t0 = time.perf_counter()
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        wall = (time.perf_counter() - t0) * 1e3
        if errors:
            raise errors[0]
        med = {k: round(statistics.median(p[i] for p in phases) * 1e3, 2)
               for i, k in enumerate(("prep_ms", "run_ms", "download_ms"))}
        return wall, sum(steps), med

    def bytes(self):
        return self.heights.nbytes + 16 * len(self.w.vents), sum(int(a.nbytes) for a in self.slots[0][1])

    def close(self):
        for ca, _ in self.slots:
            ca.close()


def roofline(p, w, schedule, peak, peak_kind):
    """Rules-kernel roofline of a profiled job p (per-launch CUDA events): 26 B per cell of the tiles
    a launch processed, over its average duration."""
    cells = p["tiles"] * p["cells_per_tile"] / max(1, p["rules_n"])
    bytes_per_launch = BYTES_PER_CELL_UPDATE * cells
    ach = bytes_per_launch / (p["rules_ms"] * 1e-3) / 1e9 if p["rules_ms"] > 0 else 0.0
    # DENSE over at least 64 tiles per rules block (4 per SM) runs the run-time hand-out form
    import torch
    blocks = 4 * torch.cuda.get_device_properties(0).multi_processor_count
    kernel = "ca_rules_dyn_kernel" if schedule == "dense" and p["tiles_total"] >= 64 * blocks else "ca_rules_kernel"
    traffic, src = None, None
    t = ncu_traffic_per_cell(kernel, "c3q" if w.name == "c3" else w.name, schedule)
    if t is not None:
        traffic, src = int(round(t[0] * cells)), t[1]
    return {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
            "traffic": traffic, "kernel": kernel, "schedule": schedule,
            "launch_ms": round(p["rules_ms"], 5), "bytes_per_launch": int(bytes_per_launch), "launches": p["rules_n"],
            "peak_kind": peak_kind,
            "traffic_ratio": round(traffic / bytes_per_launch, 3) if traffic else None,
            "note": "26 B per cell of the processed tiles (13 B state read + 13 B written); frac of the "
                    f"{peak_kind} HBM copy bandwidth; traffic = ncu dram bytes read+write per cell of this kernel on "
                    f"the {src or '-'} case (profiles/), times the cells of one launch"}


def workload_block(w, device, flush, peak, peak_kind, jobs=2):
    """ACTIVE jobs, a DENSE job, a profiled DENSE job (rules-kernel roofline) and the parity of the
    last ACTIVE job, for a sub-benchmark."""
    from volcano_ca_mc_b200 import capi
    r = Resident(w, capi.SWEEP_ACTIVE, device)
    runs = [r.run(flush) for _ in range(jobs)]
    par = r.parity()
    r.close()
    d = Resident(w, capi.SWEEP_DENSE, device)
    dj = d.run(flush, mc=False)
    d.close()
    pd = Resident(w, capi.SWEEP_DENSE, device, profile=True)
    pj = pd.run(flush, mc=False)
    pj["kernels"] = pd.ca.kernel_times()
    pd.close()
    ca_ms = sum(j["ca_ms"] for j in runs)
    mc_ms = sum(j["mc"]["ms"] for j in runs)
    return {"workload": f"{w.name}: {w.description}", "grid": [w.nx, w.ny, w.nz], "ca_steps": runs[0]["steps"],
            "value": w.cells * sum(j["steps"] for j in runs) / (ca_ms * 1e-3), "unit": "cell-updates/s",
            "ms_per_job": ca_ms / len(runs),
            "dense": {"value": w.cells * dj["steps"] / (dj["ca_ms"] * 1e-3), "ms_per_job": dj["ca_ms"]},
            "roofline": roofline(pj, w, "dense", peak, peak_kind), "kernels_dense_ms": pj["kernels"],
            "mc": {"attempts_per_s": sum(j["mc"]["attempts"] for j in runs) / (mc_ms * 1e-3),
                   "trials_per_s": sum(j["mc"]["trials"] for j in runs) / (mc_ms * 1e-3), "ms_per_job": mc_ms / len(runs)},
            "parity": par}


def mc_full_block(device, flush, peak, peak_kind, sweeps=20):
    """Potts sweeps on a whole 3D space (mc.domain = full, as the reference's configs/mc_full_3d.json,
    scaled up): 512 x 512 x 256 = 67 M cells, Moore, periodic, Q = 64, kT = 0.5, no mobility.  Every
    cell is a trial every MCS: 12 B per trial (spin read + write + the trial's share of a mobility
    read, counted as in the basalt case) against the HBM copy bandwidth."""
    from volcano_ca_mc_b200 import capi
    nx, ny, nz = 512, 512, 256
    mc = capi.PottsMC(capi.McParams(nx, ny, nz, neighborhood="moore", boundary="periodic", domain_full=True, seed=9,
                                    Q=64, J=1.0, kT=0.5, device=device))
    mc.set_domain(None)
    mc.initialize()
    mc.sweep(2)  # warm-up
    flush()
    t0 = mc.timing()[0]
    mc.sweep(sweeps)
    ms = mc.timing()[0] - t0
    info = mc.info()
    mc.close()
    trials = nx * ny * nz * sweeps
    gbs = BYTES_PER_TRIAL * trials / (ms * 1e-3) / 1e9
    return {"space": [nx, ny, nz], "neighborhood": "moore", "boundary": "periodic", "Q": 64, "kT": 0.5,
            "sweeps": sweeps, "colors": info.colors, "ms_per_sweep": ms / sweeps,
            "trials_per_s": trials / (ms * 1e-3), "achieved_gbs_12B_per_trial": round(gbs, 1),
            "hbm_frac": round(gbs / peak, 4), "peak_kind": peak_kind}


def job_mixes(args, device):
    """Many small independent jobs on one GPU through the engine's job server (engine --serve: engine
    configs in, resident handles admitted against the HBM budget, all running CA grids stepped in one
    batch), against the one-at-a-time plain path on the same jobs (one worker, vca_ca_run per job):
    a batch of 96 jobs drawn from master seed 2026 sent at once, a Poisson trace at 20 jobs/s (master
    seed 77) replayed in real time, and a sweep of arrival rates.  Every job's result digests must
    agree between the two modes."""
    from volcano_ca_mc_b200 import serve

    keys = ("slots", "jobs", "makespan_s", "jobs_per_s", "cell_updates_per_s", "p50_s", "p99_s", "mean_concurrency",
            "phases_ms")
    pick = lambda r: {k: (round(r[k], 4) if isinstance(r[k], float) else r[k]) for k in keys}
    out = {}
    # a whole mix takes one to three seconds and varies by up to a third from run to run (host
    # threads of the server against the GPU): each mode runs twice, the faster run is reported
    def best(**kw):
        runs = [serve.run(device=device, **kw) for _ in range(2)]
        return max(runs, key=lambda r: r["jobs_per_s"])

    if not args.no_batched:
        jobs = serve.make_mix(96, 2026)
        many = best(jobs=jobs, slots=args.slots, batched=True)
        one = best(jobs=jobs, slots=1, batched=False)
        streams = best(jobs=jobs, slots=args.slots, batched=False)
        out["batched"] = {"mix": "96 jobs, master seed 2026: 2D sides 128-2048, 3D sides 64-256 (z = side/2), "
                                 "200-600 CA steps, 20-100 MCS, sent at once; each mode the faster of two runs",
                          "cells": sum(j.cells for j in jobs), **pick(many), "server": many["server"],
                          "one_at_a_time": pick(one), "independent_streams": pick(streams),
                          "mismatches": serve.compare(many, one) + serve.compare(streams, one)}
    if not args.no_served:
        rate = 20.0
        trace = serve.make_mix(max(1, int(rate * args.serve_seconds)), 77, rate_hz=rate)
        many = serve.run(trace, slots=args.slots, batched=True, realtime=True, device=device)
        one = serve.run(trace, slots=1, batched=False, realtime=True, device=device)
        out["served"] = {"trace": f"{len(trace)} jobs, Poisson arrivals at {rate:g} jobs/s, master seed 77, "
                                  "replayed in real time; latency = completion - arrival",
                         **pick(many), "server": many["server"], "one_at_a_time": pick(one),
                         "mismatches": serve.compare(many, one)}
        sweep = []
        for lam in args.serve_rates:
            n = max(1, int(lam * args.sweep_seconds))
            tr = serve.make_mix(n, 1000 + int(lam), rate_hz=lam)
            m = serve.run(tr, slots=args.slots, batched=True, realtime=True, device=device)
            o = serve.run(tr, slots=1, batched=False, realtime=True, device=device)
            sweep.append({"rate_hz": lam, "jobs": n, "batched": pick(m), "one_at_a_time": pick(o),
                          "mismatches": serve.compare(m, o)})
        out["served"]["rate_sweep"] = sweep
    return out


def reference_job(w, threads, timeout, **over):
    """The reference engine on the workload's config (with overrides); its times.json and stats.json."""
    from oracle import oracle as O
    over.setdefault("output.format", "none")  # no result files: a c3 job would write 4.5 GB
    with tempfile.TemporaryDirectory() as d:
        cfg = w.write(d, **over)
        out = os.path.join(d, "out")
        subprocess.run([O.REF_ENGINE, "--config", cfg, "--out", out, "--threads", str(threads)], check=True,
                       capture_output=True, timeout=timeout)
        with open(os.path.join(out, "times.json")) as f:
            t = json.load(f)
        with open(os.path.join(out, "stats.json")) as f:
            st = json.load(f)
    return t, st


def cpu_baseline(w):
    """The reference engine on one full job of the workload, all host threads."""
    from oracle import oracle as O
    if not os.path.exists(O.REF_ENGINE):
        return None
    cores = os.cpu_count() or 1
    try:
        t, st = reference_job(w, cores, 1800)
    except Exception:
        return None
    cu = w.cells * int(t["steps"])
    return {"value": cu / (t["caSim"] * 1e-3), "unit": "cell-updates/s", "cores": cores, "kind": "reference",
            "sample": f"one full {w.name} job ({t['steps']} CA steps, ca.sweep=front, caSim {t['caSim']:.0f} ms; "
                      f"MC {w.mcs} MCS, mcSim {t['mcSim']:.0f} ms; no result files written)",
            "mc_attempts_per_s": st["mc"]["attempts"] / (t["mcSim"] * 1e-3)}


def engine_cli(w):
    """The engine command (volcano_ca_mc_b200/bin/engine) on one job of the workload, from the same
    config file the reference engine runs; its times.json sections as the reference writes them."""
    from volcano_ca_mc_b200 import capi
    if not os.path.exists(capi.ENGINE_PATH):
        return None
    with tempfile.TemporaryDirectory() as d:
        cfg = w.write(d, **{"output.format": "none"})
        out = os.path.join(d, "out")
        r = subprocess.run([capi.ENGINE_PATH, "--config", cfg, "--out", out, "--timing-detail"], capture_output=True,
                           text=True, timeout=900)
        if r.returncode != 0:
            return {"error": r.stderr.strip()[-300:]}
        with open(os.path.join(out, "times.json")) as f:
            t = json.load(f)
    keys = ("readConfig", "allocate", "terrain", "vents", "caSim", "save", "caStats", "mcInit", "mcSim", "mcStats",
            "mcSave", "total")
    return {"times_ms": {k: t[k] for k in keys if k in t}, "detail_ms": t.get("detail"), "steps": t.get("steps"),
            "cell_updates_per_s_caSim": w.cells * int(t["steps"]) / (t["caSim"] * 1e-3)}


def ours(args):
    import torch
    import torch.distributed as dist
    from volcano_ca_mc_b200 import capi, workloads

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    w = workloads.get(args.workload)
    flush = L2Flush(local)
    peak, peak_kind = measured_peaks()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    job = Resident(w, capi.SWEEP_ACTIVE, local)
    for _ in range(args.warmup):
        job.run(flush)

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    wall0 = time.perf_counter()
    jobs = [job.run(flush) for _ in range(args.steps)]
    barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()
    parity = job.parity()  # the last timed job's bytes, after the timed region
    job.close()

    ca_ms = sum(j["ca_ms"] for j in jobs)
    mc_ms = sum(j["mc"]["ms"] for j in jobs)
    cell_updates = sum(w.cells * j["steps"] for j in jobs)
    trials = sum(j["mc"]["trials"] for j in jobs)
    attempts = sum(j["mc"]["attempts"] for j in jobs)
    launches = sum(j["launches"] + j["mc"]["launches"] for j in jobs)

    # the same job with the DENSE schedule, and profiled jobs (per-kernel CUDA events) of both schedules
    dense = Resident(w, capi.SWEEP_DENSE, local)
    dj = dense.run(flush, mc=False)
    dense.close()
    profs = {}
    for name, sweep in (("active", capi.SWEEP_ACTIVE), ("dense", capi.SWEEP_DENSE)):
        pr = Resident(w, sweep, local, profile=True)
        pj = pr.run(flush, mc=False)
        pj["kernels"] = pr.ca.kernel_times()
        pr.close()
        profs[name] = pj
    roof_dense = roofline(profs["dense"], w, "dense", peak, peak_kind)
    roof_active = roofline(profs["active"], w, "active", peak, peak_kind)

    # e2e through the C ABI with host buffers on resident handles: two jobs in flight (one computing,
    # one copying), and one at a time
    e2e = E2E(w, local, inflight=E2E_INFLIGHT)
    e2e.jobs(E2E_INFLIGHT)  # warm-up: one job per handle
    e2e_jobs = max(2 * E2E_INFLIGHT, min(4 * E2E_INFLIGHT, args.steps))
    e2e_ms, e2e_steps, e2e_phases = e2e.jobs(e2e_jobs)
    e2e_h2d, e2e_d2h = e2e.bytes()
    e2e.close()
    del e2e  # its pinned buffers go back to torch's pinned-memory cache, which the next pass reuses
    e1 = E2E(w, local, inflight=1)
    e1.jobs(1)
    e1_jobs = max(1, min(3, args.steps))
    e1_ms, e1_steps, e1_phases = e1.jobs(e1_jobs)
    e1.close()

    ca_ms, mc_ms, dense_ms, e2e_ms, e1_ms, wall_ms = max_over_ranks(
        [ca_ms, mc_ms, dj["ca_ms"], e2e_ms, e1_ms, wall * 1e3], f"cuda:{local}", world)
    extra = {}
    cpu = None
    if rank == 0 and world == 1:
        # the side measurements report their own failure; the headline line prints either way
        def side(name, fn):
            try:
                return fn()
            except Exception as e:  # noqa: BLE001
                print(f"bench: {name} failed: {type(e).__name__}: {e}", file=sys.stderr, flush=True)
                return {"failed": f"{type(e).__name__}: {str(e)[:300]}"}

        if not args.no_c2 and w.name != "c2":
            extra["c2"] = side("c2", lambda: workload_block(workloads.get("c2"), local, flush, peak, peak_kind))
        extra["mc_full"] = side("mc_full", lambda: mc_full_block(local, flush, peak, peak_kind))
        mixes = side("job_mixes", lambda: job_mixes(args, local))
        extra.update(mixes if "failed" not in mixes else {"job_mixes": mixes})
        eng = side("engine_cli", lambda: engine_cli(w))
        if eng is not None:
            extra["engine_cli"] = eng
        if not args.no_cpu_baseline:
            cpu = side("cpu_baseline", lambda: cpu_baseline(w))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    value = world * cell_updates / (ca_ms * 1e-3)
    line = {
        "metric": "CA cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ca_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8+i32+f32 (integer rules, f32 temperatures)",
        "data": "synthetic (seeded Gaussian-cone terrain written as the reference's CSV heightmap)",
        "config": config_of(w),
        "method": {"schedule": "ACTIVE (tile skipping, bit-identical to DENSE)",
                   "l2": "flushed (256 MiB write) before every CA run and MC run, outside their device events; "
                         "the state (13 B x 2 buffers per cell) is far larger than L2",
                   "timing": "CUDA events on the handle's stream around the step launches of each job",
                   "parallelism": f"{world} independent replicas (weak scaling)", "ca_steps": jobs[0]["steps"]},
        "parity": parity,
        "mc": {"metric": "MC attempts/s", "attempts_per_s": world * attempts / (mc_ms * 1e-3),
               "trials_per_s": world * trials / (mc_ms * 1e-3), "ms_per_job": mc_ms / args.steps,
               "domain_cells": jobs[0]["mc"]["domain_cells"],
               "hbm_frac_12B_per_trial": round(BYTES_PER_TRIAL * trials / (mc_ms * 1e-3) / 1e9 / peak, 4)},
        "dense": {"value": world * w.cells * dj["steps"] / (dense_ms * 1e-3), "ms_per_step": dense_ms},
        "roofline": roof_dense,
        "roofline_active": roof_active,
        "kernels_ms": {"active": profs["active"]["kernels"], "dense": profs["dense"]["kernels"]},
        "active_tiles_frac": round(profs["active"]["tiles"] / max(1, profs["active"]["tiles_total"] *
                                                                   profs["active"]["steps"]), 4),
        "e2e": {"value": world * w.cells * e2e_steps / (e2e_ms * 1e-3), "unit": "cell-updates/s",
                "h2d_bytes_per_step": e2e_h2d, "d2h_bytes_per_step": e2e_d2h, "ms_per_step": e2e_ms / e2e_jobs,
                "jobs": e2e_jobs, "jobs_in_flight": E2E_INFLIGHT, "phases_median": e2e_phases,
                "path": "per job: vca_ca_reset + apply_terrain (host priority flood + upload) + place_seeds + run + "
                        "download of the five planes into pinned memory; resident handles each driven by a host "
                        "thread, one run at a time (a job's download and the next job's upload overlap the running "
                        "job); host wall clock over all jobs, first job's upload and last job's download included",
                "one_at_a_time": {"value": world * w.cells * e1_steps / (e1_ms * 1e-3), "ms_per_step": e1_ms / e1_jobs,
                                  "jobs": e1_jobs, "phases_median": e1_phases}},
        "gpu_launches": launches,
        "clocks": clocks,
        "wall_s_timed_loop": round(wall_ms / 1e3, 3),
    }
    line.update(extra)
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# reference arm: the reference engine's own CPU implementation on the host cores
# ------------------------------------------------------------------------------------------
def reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    from volcano_ca_mc_b200 import workloads
    if not os.path.exists(O.REF_ENGINE):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/engine was not built (reference sources absent "
                                                              "when build() ran)"}))
        return
    w = workloads.get(args.workload)
    cores = os.cpu_count() or 1
    sample_steps = min(w.max_steps, REF_SAMPLE_STEPS.get(w.name, w.max_steps))
    ca_ms, cu, runs = 0.0, 0, 0
    for i in range(args.warmup + args.steps):
        t, _ = reference_job(w, cores, 1800, **{"ca.maxSteps": sample_steps, "mc.enabled": False})
        if i < args.warmup:
            continue
        ca_ms += t["caSim"]
        cu += w.cells * int(t["steps"])
        runs += 1
    value = cu / (ca_ms * 1e-3)
    if sample_steps < w.max_steps:
        sample = (f"the first {sample_steps} of the job's {w.max_steps} CA steps (ca.maxSteps={sample_steps}, MC off), "
                  "caSim from the engine's times.json; the reference engine cannot resume a run, and its front sweep "
                  "costs less per step while the lava front is small, so this sample's rate is above the full job's")
    else:
        sample = f"the job's full CA run ({w.max_steps} steps at most, MC off), caSim from the engine's times.json"
    line = {"impl": "reference", "metric": "CA cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ca_ms / runs,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8+i32+f32 (integer rules, f32 temperatures)", "data": "synthetic",
            "config": config_of(w),
            "method": {"engine": "oracle/_ref/engine (reference sources, g++ -O3 -fopenmp)",
                       "ca.sweep": "front (the reference default, its fastest path)", "threads": cores},
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_job(args):
    """One CA job of the workload, nothing else: a bounded case for ncu."""
    from volcano_ca_mc_b200 import capi, workloads
    if args.profile_job == "mcfull":
        nx, ny, nz = 512, 512, 256
        sweeps = args.max_steps or 4
        mc = capi.PottsMC(capi.McParams(nx, ny, nz, neighborhood="moore", boundary="periodic", domain_full=True,
                                        seed=9, Q=64, J=1.0, kT=0.5, device=0))
        mc.set_domain(None)
        mc.initialize()
        mc.sweep(sweeps)
        mi = mc.info()
        print(json.dumps({"profile_job": "mcfull", "space": [nx, ny, nz], "sweeps": mi.sweeps,
                          "ms": mc.timing()[0]}))
        mc.close()
        return
    w = workloads.get(args.workload)
    if args.max_steps is not None:
        w.max_steps = args.max_steps
    sweep = capi.SWEEP_DENSE if args.profile_job == "dense" else capi.SWEEP_ACTIVE
    ca = capi.LavaCA(ca_params(w, sweep, 0))
    ca.apply_terrain(w.heights)
    ca.place_seeds(w.vent_cells())
    ca.run()
    info = ca.info()
    ms, _, _ = ca.timing()
    out = {"profile_job": args.profile_job, "workload": w.name, "steps": info.steps,
           "tiles_processed": info.tiles_processed, "cells_per_tile": info.cells_per_tile, "ms": ms}
    if args.profile_job == "mc":
        mc = capi.PottsMC(mc_params(w, 0))
        mc.set_domain_from_ca(ca)
        mc.set_mobility_from_ca(ca, 0.05, True)
        mc.initialize()
        mc.sweep(w.mcs)
        mi = mc.info()
        out["mc"] = {"sweeps": mi.sweeps, "domain_cells": mi.domain_cells, "ms": mc.timing()[0]}
        mc.close()
    print(json.dumps(out))
    ca.close()


def slab_arm(args):
    """One CA run of the workload split into z slabs, one per rank (volcano_ca_mc_b200.slabs): each
    rank steps its slab, the step counts are summed over NCCL, halos move by NCCL send / receive.
    CA time = CUDA events around the whole loop on each rank, max over ranks."""
    import torch
    import torch.distributed as dist
    from volcano_ca_mc_b200 import capi, slabs, workloads
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    w = workloads.get(args.workload)
    p = ca_params(w, capi.SWEEP_DENSE, local)
    lay = slabs.partition(w.nz, world)[rank]
    comm = slabs.TorchComm(f"cuda:{local}")
    random_nb = w.neighborhood in ("pentagonal", "hexagonal")
    times = []
    for it in range(args.warmup + args.steps):
        slab = slabs.GpuSlab(p, lay, w.heights, w.vent_cells())
        dist.barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        steps, stop, _, _ = slabs.run_distributed(slab, comm, w.max_steps, random_nb, len(w.vents))
        b.record()
        torch.cuda.synchronize()
        if it >= args.warmup:
            times.append(a.elapsed_time(b))
        slab.close()
    ms = max_over_ranks([sum(times)], f"cuda:{local}", world)[0]
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        value = w.cells * steps * args.steps / (ms * 1e-3)
        print(json.dumps({"metric": "CA cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                          "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                          "dtype": "u8+i32+f32 (integer rules, f32 temperatures)", "data": "synthetic",
                          "config": config_of(w),
                          "method": {"parallelism": f"{world} z slabs of one grid (DENSE schedule, halo exchange and "
                                                    "count sums over NCCL every step)", "ca_steps": steps}}),
              flush=True)


def main():
    args = parse()
    if args.slabs and args.impl == "ours" and dist_env()[1] > 1:
        slab_arm(args)
        return
    if args.profile_job:
        profile_job(args)
    elif args.impl == "reference":
        reference(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
