"""Seeded synthetic workloads: Gaussian-cone terrains with craters and value noise, written as the
reference engine's own inputs (a CSV heightmap for terrain.type = "file" and vents.positions),
so that the same files drive both this engine and the reference engine.

The reference generates only a single cone itself (engine/src/terrain/TerrainGenerator.cpp:61-84),
so multi-cone terrains are produced here and loaded through HeightmapLoader::loadCsv
(engine/src/terrain/HeightmapLoader.cpp:37-83: ROCK count = ceil(value), clamped to nz).  Heights
are written as integers, so both engines read identical columns.

Workloads (sizes from the benchmark definitions):
  c1  2D cross-section 512 x 1 x 256, one cone, 2 vents, Moore, absorbing, 300 steps, MC Q=64 kT=0.6 50 MCS
  c2  3D 256 x 256 x 128, two cones + crater, 3 vents, Moore, periodic, 400 steps, MC Q=128 kT=0.6 100 MCS
  c3  3D 1024 x 1024 x 256, six cones, 8 vents, pentagonal, absorbing, 800 steps, MC Q=256 kT=0.5 200 MCS
  c3q the c3 family on 512 x 512 x 256 (a bounded profiling case)
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np


def value_noise(nx: int, ny: int, seed: int) -> np.ndarray:
    """Smooth value noise in [-1, 1] (3 octaves, spacing 16/8/4, smoothstep interpolation) on an
    (ny, nx) grid, from a seeded lattice of uniform values."""
    rng = np.random.default_rng(seed)
    out = np.zeros((ny, nx))
    weights = ((16, 1.0), (8, 0.5), (4, 0.25))
    for spacing, w in weights:
        gx, gy = nx // spacing + 2, max(1, ny // spacing) + 2
        lat = rng.uniform(-1.0, 1.0, size=(gy, gx))
        x = np.arange(nx)
        y = np.arange(ny)
        i, fx = x // spacing, (x % spacing) / spacing
        j, fy = y // spacing, (y % spacing) / spacing
        sx = fx * fx * (3 - 2 * fx)
        sy = fy * fy * (3 - 2 * fy)
        v00 = lat[j][:, i]
        v10 = lat[j][:, i + 1]
        v01 = lat[j + 1][:, i]
        v11 = lat[j + 1][:, i + 1]
        a = v00 + (v10 - v00) * sx[None, :]
        b = v01 + (v11 - v01) * sx[None, :]
        out += w * (a + (b - a) * sy[:, None])
    return out / sum(w for _, w in weights)


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    neighborhood: str
    boundary: str
    seed: int
    max_steps: int
    heights: np.ndarray              # int32, nx*ny, x fastest
    vents: list                      # [(x, y)] columns; z = height (first AIR cell)
    Q: int
    kT: float
    mcs: int
    ca: dict = field(default_factory=dict)   # ca.* overrides
    description: str = ""

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def vent_cells(self):
        """(x, y, z, flowId) of each vent: the first AIR cell of its column (VentPlacer::placeAt,
        engine/src/terrain/VentPlacer.cpp:60-81)."""
        h = self.heights.reshape(self.ny, self.nx)
        return [(x, y, int(h[y, x]), i + 1) for i, (x, y) in enumerate(self.vents)]

    def config(self, heightmap_file: str, **over) -> dict:
        """Reference-engine JSON config (engine/src/io/Config.cpp:153-176 keys)."""
        c = {
            "space": {"nx": self.nx, "ny": self.ny, "nz": self.nz},
            "boundary": self.boundary,
            "neighborhood": self.neighborhood,
            "rngSeed": self.seed,
            "terrain": {"type": "file", "file": heightmap_file},
            "vents": {"count": len(self.vents), "placement": "positions",
                      "positions": [[int(x), int(y)] for (x, y) in self.vents]},
            "ca": {"mode": "lava", "maxSteps": self.max_steps, "sweep": "front", **self.ca},
            "mc": {"enabled": True, "domain": "basalt", "Q": self.Q, "mcs": self.mcs, "J": 1.0, "kT": self.kT,
                   "mobilityFromCooling": True, "update": "checkerboard", "statsEvery": max(1, self.mcs)},
            "output": {"format": "bin"},
        }
        for k, v in over.items():
            sect, _, key = k.partition(".")
            if key:
                c.setdefault(sect, {})[key] = v
            else:
                c[sect] = v
        return c

    def write(self, folder: str, **over) -> str:
        """Write <name>_heightmap.csv and <name>.json into folder; returns the config path."""
        os.makedirs(folder, exist_ok=True)
        csv = os.path.join(folder, f"{self.name}_heightmap.csv")
        h = self.heights.reshape(self.ny, self.nx)
        with open(csv, "w") as f:
            for row in h:
                f.write(",".join(str(int(v)) for v in row) + "\n")
        path = os.path.join(folder, f"{self.name}.json")
        with open(path, "w") as f:
            json.dump(self.config(os.path.basename(csv), **over), f, indent=2)
        return path


def _finish(h: np.ndarray, nz: int) -> np.ndarray:
    return np.clip(np.ceil(h), 0, nz).astype(np.int32).reshape(-1)


def c1() -> Workload:
    nx, ny, nz = 512, 1, 256
    x = np.arange(nx)
    h = 180.0 * np.exp(-((x - 256.0) ** 2) / (2 * 100.0 ** 2))[None, :] + 4.0 * value_noise(nx, ny, 1)
    hh = _finish(h, nz)
    return Workload("c1", nx, ny, nz, "moore", "absorbing", 1, 300, hh, [(236, 0), (276, 0)], 64, 0.6, 50,
                    description="2D cross-section 512x1x256, Gaussian cone peak 180 sigma 100, noise 4, 2 vents")


def c2() -> Workload:
    nx, ny, nz = 256, 256, 128
    x = np.arange(nx)[None, :]
    y = np.arange(ny)[:, None]
    ax, ay, bx, by = 100.0, 128.0, 170.0, 128.0
    ra = np.sqrt((x - ax) ** 2 + (y - ay) ** 2)
    rb = np.sqrt((x - bx) ** 2 + (y - by) ** 2)
    h = np.maximum(90.0 * np.exp(-ra ** 2 / (2 * 50.0 ** 2)), 60.0 * np.exp(-rb ** 2 / (2 * 35.0 ** 2)))
    h = np.where(ra < 10.0, h - 6.0, h)   # 6-cell-deep crater of radius 10 on the higher cone
    h = h + 2.0 * value_noise(nx, ny, 2)
    hh = _finish(h, nz)
    return Workload("c2", nx, ny, nz, "moore", "periodic", 2, 400, hh, [(100, 128), (96, 124), (104, 131)], 128, 0.6,
                    100, description="3D 256x256x128, cones (90, s50) + (60, s35), crater r10 d6, noise 2, 3 vents")


def c3(nx: int = 1024, ny: int = 1024, nz: int = 256, name: str = "c3") -> Workload:
    rng = np.random.default_rng(3)
    x = np.arange(nx)[None, :]
    y = np.arange(ny)[:, None]
    h = np.zeros((ny, nx))
    centers = []
    for _ in range(6):
        cx, cy = rng.uniform(150, nx - 150), rng.uniform(150, ny - 150)
        peak, sigma = rng.uniform(40, 200), rng.uniform(60, 250)
        h = np.maximum(h, peak * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sigma ** 2)))
        centers.append((cx, cy))
    h = h + 3.0 * value_noise(nx, ny, 3)
    hh = _finish(h, nz)
    vents = []
    for k in range(8):
        cx, cy = centers[k % 6]
        vents.append((int(cx) + 3 * (k // 6), int(cy)))
    return Workload(name, nx, ny, nz, "pentagonal", "absorbing", 3, 800, hh, vents, 256, 0.5, 200,
                    description=f"3D {nx}x{ny}x{nz}, six cones peak U[40,200] sigma U[60,250], noise 3, 8 vents")


def c3q() -> Workload:
    """The c3 family at a quarter of its cells (512 x 512 x 256, 67 M cells, 3.5 GB of state): the
    bounded case on which a profiler captures the c3 kernels (their DRAM traffic grows with the cells)."""
    return c3(512, 512, 256, "c3q")


WORKLOADS = {"c1": c1, "c2": c2, "c3": c3, "c3q": c3q}


def get(name: str) -> Workload:
    return WORKLOADS[name]()
