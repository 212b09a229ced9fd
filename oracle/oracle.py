"""ctypes front end of the CPU oracle (oracle/vca_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the CPU leg of
``bench.py`` as the checker, never by the product package.  It restates the reference's lava-CA
step (engine/src/ca/LavaCA.hpp) and Potts checkerboard sweep (engine/src/mc/PottsMC.cpp) in C;
``tests/test_oracle_pin.py`` pins it against outputs of the reference engine itself.

Also holds readers for the reference's result files (engine/src/io/ResultWriter.hpp:4-32), used
to compare outputs.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liboracle.so")
REF_ENGINE = os.path.join(HERE, "_ref", "engine")

AIR, ROCK, LAVA, BASALT, VOID = 0, 1, 2, 3, 255
NB = {"von_neumann": 0, "moore": 1, "pentagonal": 2, "hexagonal": 3}


def build() -> None:
    """Compile the oracle library (and the reference engine when its sources are present)."""
    subprocess.run(["make", "-C", HERE, "-s", "all"], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u64, i32, f32, f64, p = ctypes.c_uint64, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_void_p
        L.vo_splitmix64.restype = u64
        L.vo_splitmix64.argtypes = [u64]
        L.vo_hash_rand.restype = u64
        L.vo_hash_rand.argtypes = [u64, u64, u64, u64]
        L.vo_fill_depressions.argtypes = [p, i32, i32, i32, i32, p]
        L.vo_ca_step.argtypes = [p, i32, p, p, i32, p, p, p, p, p, p, p, p, p, p, p]
        L.vo_ca_step_strip.argtypes = [p, i32, u64, i32, i32, p, p, i32, p, p, p, p, p, p, p, p, p, p, p]
        L.vo_ca_step_strip.restype = None
        L.vo_ca_stop_after.restype = i32
        L.vo_ca_stop_after.argtypes = [p, i32, p]
        L.vo_mc_init.argtypes = [p, p, p]
        L.vo_mc_sweep.argtypes = [p, i32, p, p, p, p]
        L.vo_mc_energy.restype = f64
        L.vo_mc_energy.argtypes = [p, i32, p]
        L.vo_mc_color_strip.argtypes = [p, i32, i32, u64, i32, p, p, p, p]
        L.vo_mc_color_strip.restype = None
        L.vo_mc_colors.restype = i32
        L.vo_mc_colors.argtypes = [p]
        _lib = L
    return _lib


class CaParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("neighborhood", ctypes.c_int), ("periodic", ctypes.c_int), ("classic", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("max_steps", ctypes.c_int), ("eruption_steps", ctypes.c_int),
                ("erupt_temp", ctypes.c_float), ("solidus_temp", ctypes.c_float),
                ("cooling_ambient", ctypes.c_float), ("cooling_lateral", ctypes.c_float),
                ("cooling_fall", ctypes.c_float), ("ponding", ctypes.c_int)]


class McParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("neighborhood", ctypes.c_int), ("periodic", ctypes.c_int * 3),
                ("seed", ctypes.c_uint64), ("Q", ctypes.c_int), ("J", ctypes.c_double), ("kT", ctypes.c_double)]


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


@dataclass
class CaState:
    """Unframed SoA planes in globalIndex order (engine/src/core/Types.hpp:105-134)."""
    nx: int
    ny: int
    nz: int
    type: np.ndarray
    flow: np.ndarray
    temp: np.ndarray
    solid: np.ndarray
    arrival: np.ndarray

    def copy(self) -> "CaState":
        return CaState(self.nx, self.ny, self.nz, self.type.copy(), self.flow.copy(), self.temp.copy(),
                       self.solid.copy(), self.arrival.copy())

    def to_bytes(self) -> bytes:
        """ca_result.bin version 2 bytes (engine/src/io/ResultWriter.cpp:155-167, 204-213)."""
        head = b"VOLC" + struct.pack("<Iiii", 2, self.nx, self.ny, self.nz)
        return head + b"".join(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
                               for a in (self.type, self.flow, self.temp, self.solid, self.arrival))


def read_ca_bin(path: str) -> CaState:
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] != b"VOLC":
        raise ValueError(f"{path}: not a ca_result.bin")
    version, nx, ny, nz = struct.unpack_from("<Iiii", data, 4)
    n = nx * ny * nz
    off = 20
    type_ = np.frombuffer(data, np.uint8, n, off); off += n
    flow = np.frombuffer(data, "<i4", n, off); off += 4 * n
    temp = np.frombuffer(data, "<f4", n, off); off += 4 * n
    solid = np.frombuffer(data, "<u2", n, off); off += 2 * n
    if version >= 2:
        arrival = np.frombuffer(data, "<u2", n, off)
    else:
        arrival = np.zeros(n, np.uint16)
    return CaState(nx, ny, nz, type_.copy(), flow.astype(np.int32), temp.astype(np.float32),
                   solid.astype(np.uint16), arrival.astype(np.uint16))


def read_mc_bin(path: str) -> tuple[tuple[int, int, int], np.ndarray]:
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] != b"VMC1":
        raise ValueError(f"{path}: not a mc_result.bin")
    nx, ny, nz = struct.unpack_from("<iii", data, 4)
    return (nx, ny, nz), np.frombuffer(data, "<i4", nx * ny * nz, 16).astype(np.int32)


def heights_from_state(s: CaState) -> np.ndarray:
    """Terrain heights recovered from an initial state: ROCK fills z < h(x, y) (LavaCA.hpp:185-194)."""
    t = s.type.reshape(s.nz, s.ny, s.nx)
    rock = t == ROCK
    h = np.zeros((s.ny, s.nx), np.int32)
    for z in range(s.nz):
        h = np.where((h == z) & rock[z], z + 1, h)
    return h.reshape(-1)


def fill_depressions(height: np.ndarray, nx: int, ny: int, periodic_x: bool, periodic_y: bool) -> np.ndarray:
    h = np.ascontiguousarray(height, np.int32)
    out = np.empty_like(h)
    lib().vo_fill_depressions(_ptr(h), nx, ny, int(periodic_x), int(periodic_y), _ptr(out))
    return out


def vent_table(vents: list[tuple[int, int, int, int]]) -> np.ndarray:
    """flowId -> vent cell (LavaCA::placeSeeds, LavaCA.hpp:215-227); -1 marks no vent."""
    slots = max([f for (_, _, _, f) in vents], default=0) + 1
    t = np.full((slots, 3), -1, np.int32)
    for (x, y, z, f) in vents:
        t[f] = (x, y, z)
    return t


def ca_step(p: CaParams, t: int, s: CaState, spill: np.ndarray | None, vents: np.ndarray) -> tuple[CaState, np.ndarray]:
    n = s.nx * s.ny * s.nz
    out = CaState(s.nx, s.ny, s.nz, np.empty(n, np.uint8), np.empty(n, np.int32), np.empty(n, np.float32),
                  np.empty(n, np.uint16), np.empty(n, np.uint16))
    counts = np.zeros(3, np.uint64)
    vt = np.ascontiguousarray(vents, np.int32)
    lib().vo_ca_step(ctypes.byref(p), t, None if spill is None else _ptr(spill), _ptr(vt), len(vt),
                     _ptr(s.type), _ptr(s.flow), _ptr(s.temp), _ptr(s.solid), _ptr(s.arrival),
                     _ptr(out.type), _ptr(out.flow), _ptr(out.temp), _ptr(out.solid), _ptr(out.arrival),
                     _ptr(counts))
    return out, counts


def ca_step_strip(p: CaParams, t: int, gidx_base: int, own_z0: int, own_z1: int, s: CaState,
                  spill_local: np.ndarray | None, vents: np.ndarray) -> tuple[CaState, np.ndarray]:
    """One step of a strip of z layers (p.nz = the strip's layers): hashRand on global indices
    (local + gidx_base), counts over layers [own_z0, own_z1); spill levels in local z."""
    n = s.nx * s.ny * s.nz
    out = CaState(s.nx, s.ny, s.nz, np.empty(n, np.uint8), np.empty(n, np.int32), np.empty(n, np.float32),
                  np.empty(n, np.uint16), np.empty(n, np.uint16))
    counts = np.zeros(3, np.uint64)
    vt = np.ascontiguousarray(vents, np.int32)
    lib().vo_ca_step_strip(ctypes.byref(p), t, gidx_base, own_z0, own_z1,
                           None if spill_local is None else _ptr(spill_local), _ptr(vt), len(vt),
                           _ptr(s.type), _ptr(s.flow), _ptr(s.temp), _ptr(s.solid), _ptr(s.arrival),
                           _ptr(out.type), _ptr(out.flow), _ptr(out.temp), _ptr(out.solid), _ptr(out.arrival),
                           _ptr(counts))
    return out, counts


def ca_run(p: CaParams, s: CaState, spill: np.ndarray | None, vents: np.ndarray, initial_lava: int | None = None,
           max_steps: int | None = None):
    """Step loop with the reference stop rule (LavaCA::run/finishStep/countInitialState,
    LavaCA.hpp:253-256, 1206-1280).  Returns (state, steps, stop, active_hist, changed_hist)."""
    if max_steps is None:
        max_steps = p.max_steps
    lava0 = int((s.type == LAVA).sum()) if initial_lava is None else initial_lava
    air0 = int((s.type == AIR).sum())
    stop = 0
    if not p.classic and lava0 == 0:
        stop = 1
    elif p.classic and air0 == 0:
        stop = 2
    elif p.max_steps <= 0:
        stop = 4
    act, chg = [], []
    steps = 0
    while stop == 0 and steps < max_steps:
        s, c = ca_step(p, steps, s, spill, vents)
        steps += 1
        act.append(int(c[0]))
        chg.append(int(c[2]))
        stop = lib().vo_ca_stop_after(ctypes.byref(p), steps, _ptr(c))
    return s, steps, stop, act, chg


def mc_init(p: McParams, domain: np.ndarray) -> np.ndarray:
    spin = np.empty(p.nx * p.ny * p.nz, np.int32)
    d = np.ascontiguousarray(domain, np.uint8)
    lib().vo_mc_init(ctypes.byref(p), _ptr(d), _ptr(spin))
    return spin


def mc_sweep(p: McParams, t: int, domain: np.ndarray, mobility: np.ndarray | None, spin: np.ndarray) -> np.ndarray:
    """In-place sweep number t; returns [attempts, accepted, uphill] of this sweep."""
    out = np.zeros(3, np.uint64)
    d = np.ascontiguousarray(domain, np.uint8)
    m = None if mobility is None else np.ascontiguousarray(mobility, np.float32)
    lib().vo_mc_sweep(ctypes.byref(p), t, _ptr(d), None if m is None else _ptr(m), _ptr(spin), _ptr(out))
    return out


def mc_color_strip(p: McParams, t: int, col: int, gidx_base: int, zoff: int, domain: np.ndarray,
                   mobility: np.ndarray | None, spin: np.ndarray) -> np.ndarray:
    """One colour of MCS t on a strip of z layers (p.nz = the strip's layers), in place; returns
    (attempts, accepted, uphill)."""
    out = np.zeros(3, np.uint64)
    lib().vo_mc_color_strip(ctypes.byref(p), t, col, gidx_base, zoff, _ptr(domain),
                            None if mobility is None else _ptr(mobility), _ptr(spin), _ptr(out))
    return out


def mc_energy(p: McParams, t: int, spin: np.ndarray) -> float:
    return float(lib().vo_mc_energy(ctypes.byref(p), t, _ptr(spin)))


def mc_colors(p: McParams) -> int:
    return int(lib().vo_mc_colors(ctypes.byref(p)))


def basalt_domain(s: CaState) -> np.ndarray:
    """CoolingMobility::basaltDomain (engine/src/mc/CoolingMobility.cpp:8-14)."""
    return ((s.type == BASALT) | (s.type == LAVA)).astype(np.uint8)


def mobility_from_cooling(s: CaState, domain: np.ndarray, mobility_min: float) -> np.ndarray:
    """CoolingMobility::fromCooling (engine/src/mc/CoolingMobility.cpp:16-83), float64 steps rounded
    one by one as in the reference, then to float32."""
    dom = domain.astype(bool)
    mob = np.zeros(len(domain), np.float32)
    if not dom.any():
        return mob
    end = int(np.maximum(s.solid[dom], s.arrival[dom]).max())
    solid = np.where(s.type == BASALT, s.solid.astype(np.int64), end)
    tm = np.where(dom, np.maximum(solid - s.arrival.astype(np.int64), 0), 0)
    tmin, tmax = int(tm[dom].min()), int(tm[dom].max())
    if tmax == tmin:
        mob[dom] = 1.0
        return mob
    norm = (tm[dom] - tmin).astype(np.float64) / float(tmax - tmin)
    mob[dom] = (mobility_min + (1.0 - mobility_min) * norm).astype(np.float32)
    return mob


def mc_params(nx, ny, nz, neighborhood: str, boundary: str, domain_full: bool, seed: int, Q: int, J: float,
              kT: float) -> McParams:
    """PottsMC periodicity from the boundary and the domain mode (PottsMC.cpp:18, McStage.cpp:104-106)."""
    per = boundary == "periodic"
    return McParams(nx, ny, nz, NB[neighborhood], (int(per and nx > 1), int(per and ny > 1),
                                                   int(per and domain_full and nz > 1)), seed, Q, J, kT)


def ca_stop_after(p: CaParams, steps_done: int, counts: np.ndarray) -> int:
    """Stop reason after a step (LavaCA::finishStep, LavaCA.hpp:1206-1229)."""
    c = np.ascontiguousarray(counts, np.uint64)
    return int(lib().vo_ca_stop_after(ctypes.byref(p), steps_done, _ptr(c)))
