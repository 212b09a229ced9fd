"""ctypes binding of libvca.so (include/vca.h) for Python callers: tests, bench and tools.

The CUDA library is the only implementation: if ``lib/libvca.so`` is missing or fails to load,
every call raises ``VcaError`` -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libvca.so")
ENGINE_PATH = os.path.join(PKG_DIR, "bin", "engine")

# enums of include/vca.h
NB = {"von_neumann": 0, "moore": 1, "pentagonal": 2, "hexagonal": 3}
BC = {"absorbing": 0, "periodic": 1}
MODE = {"lava": 0, "classic": 1}
SWEEP_ACTIVE, SWEEP_DENSE, SWEEP_ACTIVE_LIST = 0, 1, 2
STOP_NAMES = {0: "running", 1: "no lava", 2: "no air", 3: "no change", 4: "max steps"}

# Every entry point declared in include/vca.h.
EXPORTS = [
    "vca_ca_create", "vca_ca_footprint", "vca_ca_reconfigure", "vca_ca_reset", "vca_ca_apply_terrain", "vca_ca_place_seeds", "vca_ca_step", "vca_ca_run",
    "vca_ca_get_info", "vca_ca_history", "vca_ca_download", "vca_ca_set_state", "vca_ca_get_spill", "vca_ca_flow_stats",
    "vca_ca_timing", "vca_ca_kernel_times", "vca_ca_destroy",
    "vca_ca_batch_create", "vca_ca_batch_add", "vca_ca_batch_advance", "vca_ca_batch_remove", "vca_ca_batch_info",
    "vca_ca_batch_destroy",
    "vca_ca_set_slab", "vca_ca_slab_step", "vca_ca_slab_stop", "vca_ca_layers", "vca_ca_pack_layers",
    "vca_ca_unpack_layers",
    "vca_mc_create", "vca_mc_footprint", "vca_mc_reconfigure", "vca_mc_set_domain", "vca_mc_set_mobility", "vca_mc_set_domain_from_ca",
    "vca_mc_set_mobility_from_ca", "vca_mc_mobility", "vca_mc_initialize", "vca_mc_sweep", "vca_mc_get_info",
    "vca_mc_energy", "vca_mc_grains", "vca_mc_set_mobility_values", "vca_mc_crystals", "vca_mc_set_spins", "vca_mc_timing", "vca_mc_destroy",
    "vca_mc_set_slab", "vca_mc_color_pass", "vca_mc_pack_spins", "vca_mc_unpack_spins",
    "vca_mc_energy_noalloc",
    "vca_last_error", "vca_version",
]


class VcaError(RuntimeError):
    pass


class CaDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("neighborhood", ctypes.c_int), ("boundary", ctypes.c_int), ("mode", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("max_steps", ctypes.c_int), ("eruption_steps", ctypes.c_int),
                ("erupt_temp", ctypes.c_float), ("solidus_temp", ctypes.c_float),
                ("cooling_ambient", ctypes.c_float), ("cooling_lateral", ctypes.c_float),
                ("cooling_fall", ctypes.c_float), ("ponding", ctypes.c_int), ("sweep", ctypes.c_int),
                ("device", ctypes.c_int), ("tile_y", ctypes.c_int), ("tile_z", ctypes.c_int),
                ("rules_blocks_per_sm", ctypes.c_int)]


class Vent(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int), ("y", ctypes.c_int), ("z", ctypes.c_int), ("flow_id", ctypes.c_int32)]


class CaInfo(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int), ("stop_reason", ctypes.c_int), ("lava_cells", ctypes.c_uint64),
                ("air_cells", ctypes.c_uint64), ("tiles_total", ctypes.c_uint64),
                ("tiles_processed", ctypes.c_uint64), ("cells_per_tile", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64)]


class McDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("neighborhood", ctypes.c_int), ("boundary", ctypes.c_int), ("domain_full", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("Q", ctypes.c_int), ("J", ctypes.c_double), ("kT", ctypes.c_double),
                ("device", ctypes.c_int)]


class GrainStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("grains", "cells", "largest", "high_cells", "high_grains", "high_grain_cells",
                                              "high_largest", "low_grains", "low_grain_cells", "low_largest")]


class McInfo(ctypes.Structure):
    _fields_ = [("sweeps", ctypes.c_int), ("colors", ctypes.c_int), ("domain_cells", ctypes.c_uint64),
                ("attempts", ctypes.c_uint64), ("accepted", ctypes.c_uint64), ("uphill", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libvca.so (raises VcaError when it is absent: build it with __graft_entry__.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise VcaError(f"{LIB_PATH} is missing: the CUDA library has not been built")
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise VcaError(f"cannot load {LIB_PATH}: {e}") from e
    p, i32, u64, f64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_double
    sig = {
        "vca_ca_create": [p, p], "vca_ca_footprint": [p, p], "vca_ca_reconfigure": [p, p], "vca_ca_reset": [p], "vca_ca_apply_terrain": [p, p], "vca_ca_place_seeds": [p, p, i32],
        "vca_ca_step": [p, p], "vca_ca_run": [p], "vca_ca_get_info": [p, p],
        "vca_ca_history": [p, p, p, i32, p], "vca_ca_download": [p, p, p, p, p, p],
        "vca_ca_set_state": [p, p, p, p, p, p, p, p, i32, i32], "vca_ca_get_spill": [p, p], "vca_ca_flow_stats": [p, i32, p, p, p],
        "vca_ca_timing": [p, p, p, p], "vca_ca_kernel_times": [p, p, p, p, p],
        "vca_ca_batch_create": [i32, i32, p], "vca_ca_batch_add": [p, p], "vca_ca_batch_advance": [p, i32, p, i32, p, p],
        "vca_ca_batch_remove": [p, p], "vca_ca_batch_info": [p, p, p, p],
        "vca_ca_set_slab": [p, i32, i32, i32], "vca_ca_slab_step": [p, p, p], "vca_ca_slab_stop": [p, i32],
        "vca_ca_layers": [p, p, p, p, p, p, p], "vca_ca_pack_layers": [p, i32, i32, i32, p],
        "vca_ca_unpack_layers": [p, i32, i32, i32, p],
        "vca_mc_create": [p, p], "vca_mc_footprint": [p, p], "vca_mc_reconfigure": [p, p], "vca_mc_set_domain": [p, p], "vca_mc_set_mobility": [p, p],
        "vca_mc_set_domain_from_ca": [p, p], "vca_mc_set_mobility_from_ca": [p, p, f64, i32],
        "vca_mc_mobility": [p, p], "vca_mc_initialize": [p], "vca_mc_sweep": [p, i32, p],
        "vca_mc_get_info": [p, p], "vca_mc_energy": [p, p], "vca_mc_grains": [p, i32, f64, p],
        "vca_mc_set_mobility_values": [p, p, i32], "vca_mc_crystals": [p, p],
        "vca_mc_set_spins": [p, p], "vca_mc_timing": [p, p, p, p],
        "vca_mc_energy_noalloc": [p, i32, i32, i32, i32, i32, i32, u64, i32, f64, p, p],
        "vca_mc_set_slab": [p, i32], "vca_mc_color_pass": [p, i32], "vca_mc_pack_spins": [p, i32, i32, p],
        "vca_mc_unpack_spins": [p, i32, i32, p],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.vca_ca_destroy.argtypes = [p]
    L.vca_ca_destroy.restype = None
    L.vca_mc_destroy.argtypes = [p]
    L.vca_mc_destroy.restype = None
    L.vca_ca_batch_destroy.argtypes = [p]
    L.vca_ca_batch_destroy.restype = None
    L.vca_last_error.restype = ctypes.c_char_p
    L.vca_version.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(status: int, what: str) -> None:
    if status != 0:
        msg = lib().vca_last_error().decode("utf-8", "replace")
        raise VcaError(f"{what} failed (status {status}): {msg}")


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return ctypes.c_void_p(a.ctypes.data)


@dataclass
class CaParams:
    """CaParams + grid of a lava / classic CA (engine/src/ca/CaRules.hpp:93-105)."""
    nx: int
    ny: int
    nz: int
    neighborhood: str = "moore"
    boundary: str = "absorbing"
    mode: str = "lava"
    seed: int = 42
    max_steps: int = 5000
    eruption_steps: int = 300
    erupt_temp: float = 1200.0
    solidus_temp: float = 800.0
    cooling_ambient: float = 0.3
    cooling_lateral: float = 1.5
    cooling_fall: float = 0.1
    ponding: bool = True
    sweep: int = SWEEP_ACTIVE
    device: int = 0
    tile_y: int = 0              # launch shape (0, 0: the default tile); results do not depend on it
    tile_z: int = 0
    rules_blocks_per_sm: int = 0

    def desc(self) -> CaDesc:
        return CaDesc(self.nx, self.ny, self.nz, NB[self.neighborhood], BC[self.boundary], MODE[self.mode],
                      self.seed, self.max_steps, self.eruption_steps, self.erupt_temp, self.solidus_temp,
                      self.cooling_ambient, self.cooling_lateral, self.cooling_fall, int(self.ponding),
                      self.sweep, self.device, self.tile_y, self.tile_z, self.rules_blocks_per_sm)


def ca_footprint(params: "CaParams") -> int:
    """Device bytes of a CA handle for these parameters."""
    d = params.desc()
    b = ctypes.c_uint64()
    _check(lib().vca_ca_footprint(ctypes.byref(d), ctypes.byref(b)), "vca_ca_footprint")
    return b.value


class LavaCA:
    """Python face of the vca_ca_* handle (the reference's LavaCA, engine/src/ca/LavaCA.hpp)."""

    def __init__(self, params: CaParams):
        self.params = params
        self.n = params.nx * params.ny * params.nz
        h = ctypes.c_void_p()
        d = params.desc()
        _check(lib().vca_ca_create(ctypes.byref(d), ctypes.byref(h)), "vca_ca_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().vca_ca_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reconfigure(self, params: "CaParams") -> None:
        """Another space / parameters on this handle's device memory (must fit), state of a new handle."""
        d = params.desc()
        _check(lib().vca_ca_reconfigure(self.h, ctypes.byref(d)), "vca_ca_reconfigure")
        self.params = params
        self.n = params.nx * params.ny * params.nz

    def reset(self) -> None:
        """All cells AIR, no terrain, no vents, step 0 (device memory kept)."""
        _check(lib().vca_ca_reset(self.h), "vca_ca_reset")

    def apply_terrain(self, heights: np.ndarray) -> None:
        h = np.ascontiguousarray(heights, np.int32)
        _check(lib().vca_ca_apply_terrain(self.h, _ptr(h)), "vca_ca_apply_terrain")

    def place_seeds(self, vents) -> None:
        arr = (Vent * max(1, len(vents)))(*[Vent(int(x), int(y), int(z), int(f)) for (x, y, z, f) in vents])
        _check(lib().vca_ca_place_seeds(self.h, arr, len(vents)), "vca_ca_place_seeds")

    def set_state(self, type_, flow, temp, solid, arrival, spill=None, vents=(), steps_done=0) -> None:
        t = np.ascontiguousarray(type_, np.uint8)
        f = np.ascontiguousarray(flow, np.int32)
        te = np.ascontiguousarray(temp, np.float32)
        s = np.ascontiguousarray(solid, np.uint16)
        a = np.ascontiguousarray(arrival, np.uint16)
        sp = None if spill is None else np.ascontiguousarray(spill, np.int32)
        arr = (Vent * max(1, len(vents)))(*[Vent(int(x), int(y), int(z), int(fi)) for (x, y, z, fi) in vents])
        _check(lib().vca_ca_set_state(self.h, _ptr(t), _ptr(f), _ptr(te), _ptr(s), _ptr(a), _ptr(sp), arr,
                                      len(vents), steps_done), "vca_ca_set_state")

    def step(self) -> bool:
        running = ctypes.c_int()
        _check(lib().vca_ca_step(self.h, ctypes.byref(running)), "vca_ca_step")
        return bool(running.value)

    def run(self) -> None:
        _check(lib().vca_ca_run(self.h), "vca_ca_run")

    def info(self) -> CaInfo:
        out = CaInfo()
        _check(lib().vca_ca_get_info(self.h, ctypes.byref(out)), "vca_ca_get_info")
        return out

    def history(self) -> tuple[list[int], list[int]]:
        steps = self.info().steps
        a = np.zeros(max(steps, 1), np.uint64)
        c = np.zeros(max(steps, 1), np.uint64)
        cnt = ctypes.c_int()
        _check(lib().vca_ca_history(self.h, _ptr(a), _ptr(c), steps, ctypes.byref(cnt)), "vca_ca_history")
        return [int(v) for v in a[:steps]], [int(v) for v in c[:steps]]

    def download(self, out=None):
        """The five planes (type, flowId, temp, solidStep, arrivalStep) in globalIndex order, into new
        arrays or into ``out`` (five C-contiguous arrays of those dtypes, e.g. views of pinned memory)."""
        n = self.n
        if out is None:
            out = (np.empty(n, np.uint8), np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.uint16),
                   np.empty(n, np.uint16))
        t, f, te, s, a = out
        _check(lib().vca_ca_download(self.h, _ptr(t), _ptr(f), _ptr(te), _ptr(s), _ptr(a)), "vca_ca_download")
        return t, f, te, s, a

    def spill(self) -> np.ndarray:
        out = np.empty(self.params.nx * self.params.ny, np.int32)
        _check(lib().vca_ca_get_spill(self.h, _ptr(out)), "vca_ca_get_spill")
        return out

    def flow_stats(self, flows: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Simulation::flowSums on the device: per flowId 0..flows the LAVA cells, the BASALT cells and
        the largest squared horizontal distance from the flow's vent (entry 0 is 0)."""
        lava, basalt, reach2 = (np.zeros(flows + 1, np.uint64) for _ in range(3))
        _check(lib().vca_ca_flow_stats(self.h, flows, _ptr(lava), _ptr(basalt), _ptr(reach2)), "vca_ca_flow_stats")
        return lava, basalt, reach2

    def set_slab(self, z_offset: int, own_z0: int, own_z1: int) -> None:
        """This handle is the slab of a taller grid whose layer 0 is global layer z_offset and which owns
        its layers [own_z0, own_z1) (vca_ca_set_slab)."""
        _check(lib().vca_ca_set_slab(self.h, z_offset, own_z0, own_z1), "vca_ca_set_slab")

    def slab_step(self) -> tuple[int, int]:
        """One step; the (active, changed) counts of the owned layers."""
        a, c = ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().vca_ca_slab_step(self.h, ctypes.byref(a), ctypes.byref(c)), "vca_ca_slab_step")
        return a.value, c.value

    def slab_stop(self, stop_reason: int) -> None:
        _check(lib().vca_ca_slab_stop(self.h, stop_reason), "vca_ca_slab_stop")

    def layers(self) -> tuple[list[int], int]:
        """Device addresses of layer 0 of the current type, flowId, temp, solidStep and arrivalStep planes,
        and the cells of one (pitched) layer."""
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        n = ctypes.c_uint64()
        _check(lib().vca_ca_layers(self.h, *[ctypes.byref(p) for p in ptrs], ctypes.byref(n)), "vca_ca_layers")
        return [p.value for p in ptrs], n.value

    def pack_layers(self, z0: int, types: int, full: int, buf_ptr: int) -> None:
        """Halo message into the buffer at address buf_ptr (vca_ca_pack_layers)."""
        _check(lib().vca_ca_pack_layers(self.h, z0, types, full, ctypes.c_void_p(buf_ptr)), "vca_ca_pack_layers")

    def unpack_layers(self, z0: int, types: int, full: int, buf_ptr: int) -> None:
        _check(lib().vca_ca_unpack_layers(self.h, z0, types, full, ctypes.c_void_p(buf_ptr)), "vca_ca_unpack_layers")

    def timing(self) -> tuple[float, float, int]:
        tot, ker, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_uint64()
        _check(lib().vca_ca_timing(self.h, ctypes.byref(tot), ctypes.byref(ker), ctypes.byref(n)), "vca_ca_timing")
        return tot.value, ker.value, n.value

    def kernel_times(self) -> dict:
        """Average device ms per step of each step kernel (handles created with VCA_PROFILE_KERNELS=1)."""
        d, r, c, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_uint64()
        _check(lib().vca_ca_kernel_times(self.h, ctypes.byref(d), ctypes.byref(r), ctypes.byref(c), ctypes.byref(n)),
               "vca_ca_kernel_times")
        return {"drop_ms": d.value, "rules_ms": r.value, "cand_ms": c.value, "steps": n.value}


class CaBatch:
    """Python face of vca_ca_batch_*: many LavaCA handles stepped by shared launches.  Members are
    added once their state is set up; advance() steps them and returns the ones whose stop rule held
    (they have left the batch and take every LavaCA call again)."""

    def __init__(self, device: int = 0, max_members: int = 256):
        h = ctypes.c_void_p()
        _check(lib().vca_ca_batch_create(device, max_members, ctypes.byref(h)), "vca_ca_batch_create")
        self.h = h
        self.members: dict[int, "LavaCA"] = {}

    def add(self, ca: "LavaCA") -> None:
        _check(lib().vca_ca_batch_add(self.h, ca.h), "vca_ca_batch_add")
        self.members[ca.h.value] = ca

    def advance(self, max_graphs: int = 1 << 30) -> tuple[list["LavaCA"], int]:
        """Steps until some member stops (or max_graphs graphs of 16 steps); returns the members that
        stopped and the number still running."""
        cap = max(1, len(self.members))
        out = (ctypes.c_void_p * cap)()
        n, running = ctypes.c_int(), ctypes.c_int()
        _check(lib().vca_ca_batch_advance(self.h, max_graphs, out, cap, ctypes.byref(n), ctypes.byref(running)),
               "vca_ca_batch_advance")
        done = [self.members.pop(out[i]) for i in range(n.value)]
        return done, running.value

    def run(self) -> list["LavaCA"]:
        """Steps until every member has stopped; returns them in the order they stopped."""
        order = []
        while self.members:
            done, _ = self.advance()
            order += done
        return order

    def remove(self, ca: "LavaCA") -> None:
        _check(lib().vca_ca_batch_remove(self.h, ca.h), "vca_ca_batch_remove")
        self.members.pop(ca.h.value, None)

    def info(self) -> dict:
        g, l, m = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int()
        _check(lib().vca_ca_batch_info(self.h, ctypes.byref(g), ctypes.byref(l), ctypes.byref(m)), "vca_ca_batch_info")
        return {"graphs": g.value, "launches": l.value, "members": m.value}

    def close(self) -> None:
        if self.h:
            lib().vca_ca_batch_destroy(self.h)
            self.h = ctypes.c_void_p()
            self.members.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class McParams:
    nx: int
    ny: int
    nz: int
    neighborhood: str = "moore"
    boundary: str = "absorbing"
    domain_full: bool = False
    seed: int = 42
    Q: int = 50
    J: float = 1.0
    kT: float = 0.0
    device: int = 0

    def desc(self) -> McDesc:
        return McDesc(self.nx, self.ny, self.nz, NB[self.neighborhood], BC[self.boundary], int(self.domain_full),
                      self.seed, self.Q, self.J, self.kT, self.device)


def mc_footprint(params: "McParams") -> int:
    """Device bytes an MC handle for these parameters can come to hold."""
    d = params.desc()
    b = ctypes.c_uint64()
    _check(lib().vca_mc_footprint(ctypes.byref(d), ctypes.byref(b)), "vca_mc_footprint")
    return b.value


class PottsMC:
    """Python face of the vca_mc_* handle (the reference's PottsMC with mc.update = checkerboard)."""

    def __init__(self, params: McParams):
        self.params = params
        self.n = params.nx * params.ny * params.nz
        h = ctypes.c_void_p()
        d = params.desc()
        _check(lib().vca_mc_create(ctypes.byref(d), ctypes.byref(h)), "vca_mc_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().vca_mc_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reconfigure(self, params: "McParams") -> None:
        """Another space / parameters on this handle (no more cells than at creation)."""
        d = params.desc()
        _check(lib().vca_mc_reconfigure(self.h, ctypes.byref(d)), "vca_mc_reconfigure")
        self.params = params
        self.n = params.nx * params.ny * params.nz

    def set_domain(self, domain: np.ndarray | None) -> None:
        d = None if domain is None else np.ascontiguousarray(domain, np.uint8)
        _check(lib().vca_mc_set_domain(self.h, _ptr(d)), "vca_mc_set_domain")

    def set_mobility(self, mobility: np.ndarray | None) -> None:
        m = None if mobility is None else np.ascontiguousarray(mobility, np.float32)
        _check(lib().vca_mc_set_mobility(self.h, _ptr(m)), "vca_mc_set_mobility")

    def set_domain_from_ca(self, ca: LavaCA) -> None:
        _check(lib().vca_mc_set_domain_from_ca(self.h, ca.h), "vca_mc_set_domain_from_ca")

    def set_mobility_from_ca(self, ca: LavaCA, mobility_min: float, use: bool = True) -> None:
        _check(lib().vca_mc_set_mobility_from_ca(self.h, ca.h, mobility_min, int(use)), "vca_mc_set_mobility_from_ca")

    def mobility(self) -> np.ndarray:
        out = np.empty(self.n, np.float32)
        _check(lib().vca_mc_mobility(self.h, _ptr(out)), "vca_mc_mobility")
        return out

    def initialize(self) -> None:
        _check(lib().vca_mc_initialize(self.h), "vca_mc_initialize")

    def sweep(self, count: int = 1) -> int:
        acc = ctypes.c_uint64()
        _check(lib().vca_mc_sweep(self.h, count, ctypes.byref(acc)), "vca_mc_sweep")
        return acc.value

    def info(self) -> McInfo:
        out = McInfo()
        _check(lib().vca_mc_get_info(self.h, ctypes.byref(out)), "vca_mc_get_info")
        return out

    def energy(self) -> float:
        e = ctypes.c_double()
        _check(lib().vca_mc_energy(self.h, ctypes.byref(e)), "vca_mc_energy")
        return e.value

    def grains(self, moore: bool = True, threshold: float = 0.5) -> GrainStats:
        out = GrainStats()
        _check(lib().vca_mc_grains(self.h, int(moore), threshold, ctypes.byref(out)), "vca_mc_grains")
        return out

    def crystals(self, out: np.ndarray | None = None) -> np.ndarray:
        """Orientations (N int32), into a new array or into ``out`` (e.g. a view of pinned memory)."""
        if out is None:
            out = np.empty(self.n, np.int32)
        _check(lib().vca_mc_crystals(self.h, _ptr(out)), "vca_mc_crystals")
        return out

    def set_spins(self, spins: np.ndarray) -> None:
        s = np.ascontiguousarray(spins, np.int32)
        _check(lib().vca_mc_set_spins(self.h, _ptr(s)), "vca_mc_set_spins")

    def set_slab(self, z_offset: int) -> None:
        _check(lib().vca_mc_set_slab(self.h, z_offset), "vca_mc_set_slab")

    def color_pass(self, color: int) -> None:
        _check(lib().vca_mc_color_pass(self.h, color), "vca_mc_color_pass")

    def pack_spins(self, z0: int, layers: int, buf_ptr: int) -> None:
        _check(lib().vca_mc_pack_spins(self.h, z0, layers, ctypes.c_void_p(buf_ptr)), "vca_mc_pack_spins")

    def unpack_spins(self, z0: int, layers: int, buf_ptr: int) -> None:
        _check(lib().vca_mc_unpack_spins(self.h, z0, layers, ctypes.c_void_p(buf_ptr)), "vca_mc_unpack_spins")

    def timing(self) -> tuple[float, float, int]:
        tot, ker, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_uint64()
        _check(lib().vca_mc_timing(self.h, ctypes.byref(tot), ctypes.byref(ker), ctypes.byref(n)), "vca_mc_timing")
        return tot.value, ker.value, n.value


def mc_energy_noalloc(spins_ptr: int, nx: int, ny: int, nz: int, energy_ptr: int, *, neighborhood: str = "moore",
                      boundary: str = "absorbing", domain_full: bool = False, seed: int = 42, mcs: int = 0,
                      J: float = 1.0, stream: int = 0) -> None:
    """vca_mc_energy_noalloc: queue the energy of a device spin grid (spins_ptr, nx*ny*nz int32) into
    the device double at energy_ptr on the CUDA stream handle ``stream`` (0: legacy default stream).
    Allocates nothing; grids above 2^28 cells raise VcaError."""
    _check(lib().vca_mc_energy_noalloc(ctypes.c_void_p(spins_ptr), nx, ny, nz, NB[neighborhood], BC[boundary],
                                       int(domain_full), seed, mcs, J, ctypes.c_void_p(energy_ptr),
                                       ctypes.c_void_p(stream) if stream else None), "vca_mc_energy_noalloc")
