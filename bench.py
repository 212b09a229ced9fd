#!/usr/bin/env python
"""Benchmark of the lava-CA + Potts-MC hot paths on B200 (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2] [--impl ours|reference]

A step is one job of the workload: the lava CA run from the seeded terrain to its stop rule (for
c2, 400 steps of a 256 x 256 x 128 grid) followed by the Potts checkerboard crystallisation of
the basalt it left (100 MCS).  Inputs are resident in HBM when the timed region starts (each job's
handle is set up beforehand); L2 is flushed before every job outside the job's device events.

  value          CA cell-updates/s = cells x CA steps / CA device time (ACTIVE schedule, the
                 default), whole job over all ranks.
  mc             MC trials/s and attempts/s of the same jobs (attempts exclude mobility skips).
  dense          the same jobs with the DENSE schedule (every cell every step).
  roofline       the rules kernel of the DENSE jobs: 26 B per cell (13 B state read + 13 B written)
                 over its CUDA-event launch time, against the measured HBM copy bandwidth; traffic =
                 the ncu DRAM bytes per launch recorded in profiles/.  roofline_active: the same for
                 the ACTIVE jobs (26 B per cell of the processed tiles).
  kernels_ms     device time per step of the drop-depth, rules and candidate kernels.
  large          the full-size workload c3 (1024 x 1024 x 256, random pentagonal, 800 steps, 200 MCS):
                 one ACTIVE job with its MC, one DENSE job, the DENSE rules-kernel roofline.
  e2e            CA cell-updates/s through the C ABI on one resident handle: reset, terrain and vents
                 from host memory, run, the five planes back into pinned host memory.
  engine_cli     the engine command on one job of the workload, its times.json sections.
  cpu_baseline   the reference engine (oracle/_ref/engine, --threads = host cores) on one job.

With --impl reference the reference engine itself is timed on the host cores (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-large", action="store_true", help="skip the full-size 1024x1024x256 sub-benchmark")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched job-mix sub-benchmark")
    ap.add_argument("--no-served", action="store_true", help="skip the served (Poisson arrivals) sub-benchmark")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="length of the served arrival trace")
    ap.add_argument("--slots", type=int, default=16, help="worker slots of the batched and served runs")
    ap.add_argument("--profile-job", choices=["active", "dense", "mc"], default=None,
                    help="run exactly one CA job with this schedule (no warm-up, no MC), or with mc one ACTIVE "
                         "CA job and its MC stage, and exit: the case ncu captures")
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


def ncu_traffic(kernel: str, workload: str, schedule: str):
    """DRAM bytes per launch of a kernel from the committed ncu summaries (profiles/*.md lines
    `traffic: kernel=<k> workload=<w> schedule=<s> bytes_per_launch=<n>`), or None."""
    import glob
    import re
    pat = re.compile(r"traffic:\s*kernel=(\S+)\s+workload=(\S+)\s+schedule=(\S+)\s+bytes_per_launch=(\d+)")
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for line in f:
                m = pat.search(line)
                if m and m.group(1) == kernel and m.group(2) == workload and m.group(3) == schedule:
                    return int(m.group(4))
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
    """Writes a buffer larger than L2 (126 MB) between jobs."""

    def __init__(self, device):
        import torch
        self.buf = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{device}")

    def __call__(self):
        import torch
        self.buf.fill_(1)
        torch.cuda.synchronize()


def run_job(w, sweep, device, flush, profile=False, mc=True):
    """One job with resident inputs; returns device-timed figures."""
    from volcano_ca_mc_b200 import capi
    if profile:
        os.environ["VCA_PROFILE_KERNELS"] = "1"
    try:
        ca = capi.LavaCA(ca_params(w, sweep, device))
        ca.apply_terrain(w.heights)
        ca.place_seeds(w.vent_cells())
    finally:
        os.environ.pop("VCA_PROFILE_KERNELS", None)
    flush()
    ca.run()
    ca_ms, rules_ms, rules_n = ca.timing()
    info = ca.info()
    mc_out = None
    if not profile and mc:
        mc = capi.PottsMC(mc_params(w, device))
        mc.set_domain_from_ca(ca)
        mc.set_mobility_from_ca(ca, 0.05, True)
        mc.initialize()
        flush()
        mc.sweep(w.mcs)
        mi = mc.info()
        mc_ms, _, _ = mc.timing()
        mc_out = {"ms": mc_ms, "trials": mi.domain_cells * w.mcs, "attempts": mi.attempts,
                  "launches": mi.kernel_launches, "domain_cells": mi.domain_cells}
        mc.close()
    out = {"ca_ms": ca_ms, "steps": info.steps, "stop": info.stop_reason, "tiles": info.tiles_processed,
           "cells_per_tile": info.cells_per_tile, "tiles_total": info.tiles_total, "launches": info.kernel_launches,
           "rules_ms": rules_ms, "rules_n": rules_n, "mc": mc_out}
    if profile:
        out["kernels"] = ca.kernel_times()
    ca.close()
    return out


class E2E:
    """The call sequence of a job through the C ABI on one resident handle: reset, terrain and vents
    from host memory, run to the stop rule, all five planes back into pinned host memory.  The handle
    and the pinned buffers are set up once, outside the timed steps."""

    def __init__(self, w, device):
        import torch
        from volcano_ca_mc_b200 import capi
        self.w = w
        self.ca = capi.LavaCA(ca_params(w, capi.SWEEP_ACTIVE, device))
        n = w.cells
        pin = lambda dt: torch.empty(n, dtype=dt, pin_memory=True).numpy()
        self.out = (pin(torch.uint8), pin(torch.int32), pin(torch.float32), pin(torch.int16).view("uint16"),
                    pin(torch.int16).view("uint16"))
        self.heights = torch.from_numpy(w.heights.copy()).pin_memory().numpy()

    def step(self):
        """One job; returns (ms, steps)."""
        t0 = time.perf_counter()
        self.ca.reset()
        self.ca.apply_terrain(self.heights)
        self.ca.place_seeds(self.w.vent_cells())
        self.ca.run()
        self.ca.download(self.out)
        steps = self.ca.info().steps
        return (time.perf_counter() - t0) * 1e3, steps

    def bytes(self):
        return self.heights.nbytes + 16 * len(self.w.vents), sum(int(a.nbytes) for a in self.out)

    def close(self):
        self.ca.close()


def job_mixes(args, device):
    """Many small independent jobs on one GPU through the job server (resident handles, footprint
    admission): a batch of 96 jobs drawn from master seed 2026, run on `slots` workers and one at a
    time, and a Poisson trace (20 jobs/s, master seed 77) replayed in real time the same two ways.
    Every job's result hash must agree between the two runs."""
    from volcano_ca_mc_b200 import serve

    keys = ("slots", "jobs", "makespan_s", "jobs_per_s", "cell_updates_per_s", "p50_s", "p99_s", "mean_concurrency")
    out = {}
    if not args.no_batched:
        jobs = serve.make_mix(96, 2026)
        many = serve.run(jobs, slots=args.slots, device=device)
        one = serve.run(jobs, slots=1, device=device)
        out["batched"] = {"mix": "96 jobs, master seed 2026: 2D sides 128-2048, 3D sides 64-256 (z = side/2), "
                                 "200-600 CA steps, 20-100 MCS",
                          "cells": sum(j.cells for j in jobs), **{k: many[k] for k in keys},
                          "phase_ms_total": many["phase_ms_total"],
                          "one_at_a_time": {k: one[k] for k in keys}, "mismatches": serve.compare(many, one)}
    if not args.no_served:
        rate = 20.0
        trace = serve.make_mix(max(1, int(rate * args.serve_seconds)), 77, rate_hz=rate)
        many = serve.run(trace, slots=args.slots, realtime=True, device=device)
        one = serve.run(trace, slots=1, realtime=True, device=device)
        out["served"] = {"trace": f"{len(trace)} jobs, Poisson arrivals at {rate:g} jobs/s, master seed 77, "
                                  "replayed in real time; latency = completion - arrival",
                         **{k: many[k] for k in keys}, "phase_ms_total": many["phase_ms_total"],
                         "one_at_a_time": {k: one[k] for k in keys}, "mismatches": serve.compare(many, one)}
    return out


def cpu_baseline(w):
    """The reference engine on one job of the workload, all host threads."""
    from oracle import oracle as O
    if not os.path.exists(O.REF_ENGINE):
        return None
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        cfg = w.write(d)
        out = os.path.join(d, "out")
        r = subprocess.run([O.REF_ENGINE, "--config", cfg, "--out", out, "--threads", str(cores)],
                           capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            return None
        t = json.load(open(os.path.join(out, "times.json")))
        st = json.load(open(os.path.join(out, "stats.json")))
    cu = w.cells * int(t["steps"])
    return {"value": cu / (t["caSim"] * 1e-3), "unit": "cell-updates/s", "cores": cores, "kind": "reference",
            "sample": f"one full {w.name} job ({t['steps']} CA steps, ca.sweep=front, caSim {t['caSim']:.0f} ms; "
                      f"MC {w.mcs} MCS mcSim {t['mcSim']:.0f} ms)",
            "mc_attempts_per_s": st["mc"]["attempts"] / (t["mcSim"] * 1e-3)}


def engine_cli(w):
    """The engine command (volcano_ca_mc_b200/bin/engine) on one job of the workload, from the same
    config file the reference engine runs; its times.json sections as the reference writes them."""
    from volcano_ca_mc_b200 import capi
    if not os.path.exists(capi.ENGINE_PATH):
        return None
    with tempfile.TemporaryDirectory() as d:
        cfg = w.write(d)
        out = os.path.join(d, "out")
        r = subprocess.run([capi.ENGINE_PATH, "--config", cfg, "--out", out, "--timing-detail"], capture_output=True,
                           text=True, timeout=900)
        if r.returncode != 0:
            return {"error": r.stderr.strip()[-300:]}
        t = json.load(open(os.path.join(out, "times.json")))
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

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        run_job(w, capi.SWEEP_ACTIVE, local, flush)

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    wall0 = time.perf_counter()
    jobs = [run_job(w, capi.SWEEP_ACTIVE, local, flush) for _ in range(args.steps)]
    barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()

    ca_ms = sum(j["ca_ms"] for j in jobs)
    mc_ms = sum(j["mc"]["ms"] for j in jobs)
    cell_updates = sum(w.cells * j["steps"] for j in jobs)
    trials = sum(j["mc"]["trials"] for j in jobs)
    attempts = sum(j["mc"]["attempts"] for j in jobs)
    launches = sum(j["launches"] + j["mc"]["launches"] for j in jobs)

    # dense schedule, same jobs (like-for-like with a full sweep)
    dense = [run_job(w, capi.SWEEP_DENSE, local, flush) for _ in range(max(1, min(2, args.steps)))]
    dense_ms = sum(j["ca_ms"] for j in dense)
    dense_cu = sum(w.cells * j["steps"] for j in dense)

    # rules-kernel roofline: per-launch CUDA events on the handle's stream
    prof = run_job(w, capi.SWEEP_ACTIVE, local, flush, profile=True)
    prof_dense = run_job(w, capi.SWEEP_DENSE, local, flush, profile=True)
    peak, peak_kind = measured_peaks()

    def roof(p, wl_name, schedule):
        cells = p["tiles"] * p["cells_per_tile"] / max(1, p["rules_n"])
        bytes_per_launch = BYTES_PER_CELL_UPDATE * cells
        ach = bytes_per_launch / (p["rules_ms"] * 1e-3) / 1e9 if p["rules_ms"] > 0 else 0.0
        return {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
                "traffic": ncu_traffic("ca_rules_kernel", wl_name, schedule), "kernel": "ca_rules_kernel",
                "schedule": schedule, "launch_ms": round(p["rules_ms"], 5), "bytes_per_launch": int(bytes_per_launch),
                "launches": p["rules_n"], "peak_kind": peak_kind,
                "note": "26 B per cell of the processed tiles (13 B state read + 13 B written); frac of measured HBM copy "
                        "bandwidth; traffic = ncu dram bytes read+write per launch (profiles/)"}

    roof_active, roof_dense = roof(prof, w.name, "active"), roof(prof_dense, w.name, "dense")

    # the full-size 3D workload: one ACTIVE job (CA + MC), one DENSE job, one DENSE job with per-kernel events
    large = None
    if not args.no_large:
        wl3 = workloads.get("c3")
        j3 = run_job(wl3, capi.SWEEP_ACTIVE, local, flush)
        d3 = run_job(wl3, capi.SWEEP_DENSE, local, flush, mc=False)
        p3 = run_job(wl3, capi.SWEEP_DENSE, local, flush, profile=True)
        m3 = j3["mc"]
        large = {"workload": f"{wl3.name}: {wl3.description}", "grid": [wl3.nx, wl3.ny, wl3.nz], "ca_steps": j3["steps"],
                 "value": wl3.cells * j3["steps"] / (j3["ca_ms"] * 1e-3), "unit": "cell-updates/s",
                 "ms_per_job": j3["ca_ms"],
                 "dense": {"value": wl3.cells * d3["steps"] / (d3["ca_ms"] * 1e-3), "ms_per_job": d3["ca_ms"]},
                 "roofline": roof(p3, wl3.name, "dense"), "kernels_dense_ms": p3["kernels"],
                 "mc": {"attempts_per_s": m3["attempts"] / (m3["ms"] * 1e-3), "trials_per_s": m3["trials"] / (m3["ms"] * 1e-3),
                        "ms_per_job": m3["ms"], "domain_cells": m3["domain_cells"],
                        "hbm_frac_12B_per_trial": round(BYTES_PER_TRIAL * m3["trials"] / (m3["ms"] * 1e-3) / 1e9 / peak, 4)}}

    # e2e through the C ABI with host buffers, on a resident handle
    e2e = E2E(w, local)
    e2e.step()  # warm-up
    e2e_runs = [e2e.step() for _ in range(max(1, min(3, args.steps)))]
    e2e_ms = sum(r[0] for r in e2e_runs)
    e2e_cu = sum(r[1] * w.cells for r in e2e_runs)
    e2e_h2d, e2e_d2h = e2e.bytes()
    e2e.close()

    ca_ms, mc_ms, dense_ms, e2e_ms, wall_ms = max_over_ranks([ca_ms, mc_ms, dense_ms, e2e_ms, wall * 1e3],
                                                             f"cuda:{local}", world)
    cpu = None
    eng = None
    mixes = {}
    if rank == 0 and world == 1:
        mixes = job_mixes(args, local)
        eng = engine_cli(w)
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(w)
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
        "config": {"workload": f"{w.name}: {w.description}", "grid": [w.nx, w.ny, w.nz],
                   "neighborhood": w.neighborhood, "boundary": w.boundary, "ca_steps": jobs[0]["steps"],
                   "mc": f"Q={w.Q} kT={w.kT} {w.mcs} MCS checkerboard, cooling mobility",
                   "schedule": "ACTIVE (tile skipping, bit-identical to DENSE)",
                   "l2": "flushed (256 MiB write) before every CA run and MC run, outside their device events",
                   "step": "one job: CA run to the stop rule + MC crystallisation of its basalt",
                   "parallelism": f"{world} independent replicas (weak scaling)"},
        "mc": {"metric": "MC attempts/s", "attempts_per_s": world * attempts / (mc_ms * 1e-3),
               "trials_per_s": world * trials / (mc_ms * 1e-3), "ms_per_job": mc_ms / args.steps,
               "domain_cells": jobs[0]["mc"]["domain_cells"],
               "hbm_frac_12B_per_trial": round(BYTES_PER_TRIAL * trials / (mc_ms * 1e-3) / 1e9 / peak, 4)},
        "dense": {"value": world * dense_cu / (dense_ms * 1e-3), "ms_per_step": dense_ms / len(dense)},
        "roofline": roof_dense,
        "roofline_active": roof_active,
        "kernels_ms": {"active": prof["kernels"], "dense": prof_dense["kernels"]},
        "active_tiles_frac": round(prof["tiles"] / max(1, prof["tiles_total"] * prof["steps"]), 4),
        "e2e": {"value": world * e2e_cu / (e2e_ms * 1e-3), "unit": "cell-updates/s",
                "h2d_bytes_per_step": e2e_h2d, "d2h_bytes_per_step": e2e_d2h, "ms_per_step": e2e_ms / len(e2e_runs),
                "path": "vca_ca_reset + apply_terrain (host priority flood + upload) + place_seeds + run + download of "
                        "the five planes into pinned memory, one resident handle, host wall clock"},
        "gpu_launches": launches,
        "clocks": clocks,
        "wall_s_timed_loop": round(wall_ms / 1e3, 3),
    }
    if large is not None:
        line["large"] = large
    line.update(mixes)
    if eng is not None:
        line["engine_cli"] = eng
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
    ca_ms, mc_ms, cu, att, runs = 0.0, 0.0, 0, 0, 0
    with tempfile.TemporaryDirectory() as d:
        cfg = w.write(d)
        for i in range(args.warmup + args.steps):
            out = os.path.join(d, f"out{i}")
            subprocess.run([O.REF_ENGINE, "--config", cfg, "--out", out, "--threads", str(cores)], check=True,
                           capture_output=True, timeout=900)
            if i < args.warmup:
                continue
            t = json.load(open(os.path.join(out, "times.json")))
            st = json.load(open(os.path.join(out, "stats.json")))
            ca_ms += t["caSim"]
            mc_ms += t["mcSim"]
            cu += w.cells * int(t["steps"])
            att += st["mc"]["attempts"]
            runs += 1
    value = cu / (ca_ms * 1e-3)
    line = {"impl": "reference", "metric": "CA cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ca_ms / runs,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8+i32+f32 (integer rules, f32 temperatures)", "data": "synthetic",
            "config": {"workload": f"{w.name}: {w.description}", "grid": [w.nx, w.ny, w.nz],
                       "engine": "oracle/_ref/engine (reference sources, g++ -O3 -fopenmp)",
                       "ca.sweep": "front (the reference default, its fastest path)", "threads": cores},
            "mc": {"metric": "MC attempts/s", "attempts_per_s": att / (mc_ms * 1e-3)},
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": "reference",
                             "sample": f"{runs} full {w.name} jobs, caSim from times.json"},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_job(args):
    """One CA job of the workload, nothing else: a bounded case for ncu."""
    from volcano_ca_mc_b200 import capi, workloads
    w = workloads.get(args.workload)
    sweep = capi.SWEEP_DENSE if args.profile_job == "dense" else capi.SWEEP_ACTIVE
    ca = capi.LavaCA(ca_params(w, sweep, 0))
    ca.apply_terrain(w.heights)
    ca.place_seeds(w.vent_cells())
    ca.run()
    info = ca.info()
    ms, _, _ = ca.timing()
    out = {"profile_job": args.profile_job, "workload": w.name, "steps": info.steps,
           "tiles_processed": info.tiles_processed, "ms": ms}
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


def main():
    args = parse()
    if args.profile_job:
        profile_job(args)
    elif args.impl == "reference":
        reference(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
