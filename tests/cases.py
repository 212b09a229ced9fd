"""Seeded CA / MC cases shared by the parity tests: terrain, vents, initial states, and helpers
that run the same case through the CUDA path (libvca.so) and through the CPU oracle."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

ROCK, LAVA, AIR = 1, 2, 0


def terrain(nx: int, ny: int, nz: int, seed: int, crater: bool = True) -> np.ndarray:
    """Cone(s) plus noise, ceil'd and clamped to [0, nz]; heights as int32 nx*ny (x fastest)."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx)[None, :]
    y = np.arange(ny)[:, None]
    h = np.zeros((ny, nx))
    for _ in range(2):
        cx, cy = rng.uniform(0.25, 0.75) * nx, rng.uniform(0.25, 0.75) * ny
        peak = rng.uniform(0.35, 0.7) * nz
        sigma = rng.uniform(0.15, 0.3) * max(nx, ny)
        h = np.maximum(h, peak * np.exp(-((x - cx) ** 2 + (y - cy) ** 2 * (ny > 1)) / (2 * sigma ** 2)))
    if crater:
        cx, cy = np.unravel_index(np.argmax(h), h.shape)[::-1]
        r = np.sqrt((x - cx) ** 2 + (y - cy) ** 2 * (ny > 1))
        h = np.where(r < max(2, nx // 16), h - 3, h)
    h = h + rng.uniform(-1.5, 1.5, size=h.shape)
    return np.clip(np.ceil(h), 0, nz).astype(np.int32).reshape(-1)


def pick_vents(heights: np.ndarray, nx: int, ny: int, nz: int, count: int, seed: int):
    rng = np.random.default_rng(seed + 7)
    hh = heights.reshape(ny, nx)
    cols = [(int(x), int(y)) for y in range(ny) for x in range(nx) if hh[y, x] < nz]
    # prefer high columns (near the summit) so lava has somewhere to go
    cols.sort(key=lambda c: -hh[c[1], c[0]])
    top = cols[: max(count * 6, 12)]
    idx = rng.choice(len(top), size=count, replace=False)
    return [(top[i][0], top[i][1], int(hh[top[i][1], top[i][0]]), k + 1) for k, i in enumerate(idx)]


def initial_state(nx, ny, nz, heights, vents, erupt_temp, classic=False) -> O.CaState:
    n = nx * ny * nz
    t = np.zeros((nz, ny, nx), np.uint8)
    if heights is not None:
        hh = heights.reshape(ny, nx)
        z = np.arange(nz)[:, None, None]
        t[z < hh[None, :, :]] = ROCK
    s = O.CaState(nx, ny, nz, t.reshape(-1).copy(), np.zeros(n, np.int32), np.zeros(n, np.float32),
                  np.zeros(n, np.uint16), np.zeros(n, np.uint16))
    for (x, y, zz, f) in vents:
        i = x + nx * (y + ny * zz)
        s.type[i] = LAVA
        s.flow[i] = f
        s.temp[i] = 0.0 if classic else erupt_temp
    return s


def oracle_params(p) -> O.CaParams:
    """capi.CaParams -> oracle CaParams."""
    return O.CaParams(p.nx, p.ny, p.nz, O.NB[p.neighborhood], int(p.boundary == "periodic"), int(p.mode == "classic"),
                      p.seed, p.max_steps, p.eruption_steps, p.erupt_temp, p.solidus_temp, p.cooling_ambient,
                      p.cooling_lateral, p.cooling_fall, int(p.ponding))


def state_diff(a: O.CaState, planes) -> str:
    """Empty when equal bit for bit; otherwise a short description of the first differences."""
    out = []
    for name, got in zip(("type", "flow", "temp", "solid", "arrival"), planes):
        ref = getattr(a, name)
        if ref.dtype == np.float32:
            bad = np.nonzero(ref.view(np.uint32) != np.asarray(got, np.float32).view(np.uint32))[0]
        else:
            bad = np.nonzero(ref != got)[0]
        if len(bad):
            out.append(f"{name}: {len(bad)} cells differ, first {bad[:4].tolist()} ref {ref[bad[:4]].tolist()} "
                       f"got {np.asarray(got)[bad[:4]].tolist()}")
    return "; ".join(out)
