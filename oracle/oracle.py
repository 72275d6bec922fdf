"""ctypes wrapper of the oracle (oracle/dem_oracle.c) and of the reference's own step
(oracle/_ref/libref_world.so).

TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
and reference legs may import this module, and only as the checker or as the timed
CPU baseline; nothing in world_b200/ imports it.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HIST_CAP = 24


class DemParams(ctypes.Structure):
    _fields_ = [
        ("lo", c_float * 3), ("hi", c_float * 3), ("grid", c_int32 * 3),
        ("particles_per_cell", c_int32), ("dgrid", c_int32 * 3),
        ("gravity", c_float), ("radius", c_float), ("max_force", c_float),
        ("wall_lo", c_float * 3), ("wall_hi", c_float * 3),
        ("restitution", c_float), ("friction", c_float),
        ("k_n", c_float), ("k_t", c_float), ("clamp_overlap", c_float),
        ("ln_e", c_float), ("damp_den", c_float), ("dt", c_float),
        ("history", c_int32), ("integrator", c_int32), ("picard_iterations", c_int32),
        ("picard_tolerance", c_float),
    ]


def _load_oracle() -> ctypes.CDLL:
    from . import build as oracle_build
    path = oracle_build.ORACLE_LIB
    if not os.path.exists(path):
        oracle_build.build_oracle()
    lib = ctypes.CDLL(path)
    P = POINTER(DemParams)
    vp = c_void_p
    lib.dem_params_derive.argtypes = [P, c_float, c_float, c_float]
    lib.dem_num_threads.restype = c_int
    lib.dem_set_num_threads.argtypes = [c_int]
    lib.dem_cell_keys.argtypes = [P, c_int64, vp, vp]
    lib.dem_candidates.argtypes = [P, c_int64, vp, vp, vp, vp, vp, c_int64, POINTER(c_int64)]
    lib.dem_candidates.restype = c_int64
    lib.dem_compute_rhs.argtypes = [P, c_int64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                    POINTER(c_int64), POINTER(c_int64)]
    lib.dem_step.argtypes = [P, c_int64, vp, vp, vp, vp, vp, vp, vp, POINTER(c_int32),
                             POINTER(c_float), POINTER(c_int64), POINTER(c_int64)]
    lib.dem_deposit.argtypes = [P, c_int64, vp, vp, vp]
    lib.dem_energy.argtypes = [P, c_int64, vp, vp, vp, vp, vp, vp, POINTER(c_int64)]
    lib.dem_energy.restype = c_double
    lib.dem_momentum.argtypes = [c_int64, vp, vp, vp]
    return lib


_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = _load_oracle()
    return _LIB


def _p(a):
    return None if a is None else c_void_p(a.ctypes.data)


def params_from_config(cfg) -> DemParams:
    """dem_params for a world_b200.SimConfig (same derivation as the library)."""
    p = DemParams()
    for a, ax in enumerate("xyz"):
        p.lo[a] = getattr(cfg.domain, f"{ax}_min")
        p.hi[a] = getattr(cfg.domain, f"{ax}_max")
        p.grid[a] = getattr(cfg, f"collision_grid_size_{ax}")
        p.dgrid[a] = getattr(cfg, f"density_grid_size_{ax}")
    ph = cfg.physics
    p.particles_per_cell = cfg.particles_per_cell
    p.gravity = ph.gravity
    p.max_force = ph.max_force
    p.wall_lo[0], p.wall_lo[1], p.wall_lo[2] = ph.wall_x_min, ph.wall_y_min, ph.floor_z
    p.wall_hi[0], p.wall_hi[1], p.wall_hi[2] = ph.wall_x_max, ph.wall_y_max, ph.ceiling_z
    p.restitution = ph.restitution
    p.friction = ph.friction
    p.dt = cfg.dt
    p.history = 1 if cfg.history else 0
    p.integrator = 0 if cfg.time_integrator == "semi_implicit_euler" else 1
    p.picard_iterations = cfg.picard_iterations
    p.picard_tolerance = cfg.picard_tolerance
    lib().dem_params_derive(ctypes.byref(p), ph.normal_stiffness, ph.tangential_stiffness,
                            ph.particle_radius)
    return p


class OracleSim:
    """The CPU restatement driven like ParticleDynamics: AoS state by grain id."""

    def __init__(self, params: DemParams, state, radius, mass):
        self.p = params
        self.state = np.ascontiguousarray(state, np.float32).reshape(-1).copy()
        self.n = self.state.size // 6
        self.radius = np.ascontiguousarray(radius, np.float32)
        self.mass = np.ascontiguousarray(mass, np.float32)
        self.hcnt = np.zeros(self.n, np.int32)
        self.hpart = np.zeros(self.n * HIST_CAP, np.int32)
        self.hxi = np.zeros(self.n * HIST_CAP * 3, np.float32)
        self.rhs = np.zeros(6 * self.n, np.float32)
        self.overflow = 0
        self.hist_overflow = 0
        self.picard_used = 0
        self.picard_residual = 0.0
        self.time = np.float32(0.0)

    def step(self, steps: int = 1) -> None:
        used = c_int32()
        res = c_float()
        ovf = c_int64()
        hovf = c_int64()
        for _ in range(steps):
            lib().dem_step(ctypes.byref(self.p), self.n, _p(self.state), _p(self.radius),
                           _p(self.mass), _p(self.hcnt), _p(self.hpart), _p(self.hxi),
                           _p(self.rhs), ctypes.byref(used), ctypes.byref(res),
                           ctypes.byref(ovf), ctypes.byref(hovf))
            self.overflow += ovf.value
            self.hist_overflow += hovf.value
            self.picard_used = used.value
            self.picard_residual = res.value
            self.time = np.float32(self.time + np.float32(self.p.dt))

    def cell_keys(self) -> np.ndarray:
        out = np.empty(self.n, np.int32)
        lib().dem_cell_keys(ctypes.byref(self.p), self.n, _p(self.state), _p(out))
        return out

    def candidates(self):
        offsets = np.zeros(self.n + 1, np.int64)
        ovf = c_int64()
        total = lib().dem_candidates(ctypes.byref(self.p), self.n, _p(self.state),
                                     _p(self.radius), _p(offsets), None, None, 0,
                                     ctypes.byref(ovf))
        cand = np.empty(max(total, 1), np.int32)
        contact = np.empty(max(total, 1), np.uint8)
        lib().dem_candidates(ctypes.byref(self.p), self.n, _p(self.state), _p(self.radius),
                             _p(offsets), _p(cand), _p(contact), total, ctypes.byref(ovf))
        return offsets, cand[:total], contact[:total], int(ovf.value)

    def compute_rhs(self) -> np.ndarray:
        out = np.empty(6 * self.n, np.float32)
        nc = np.zeros(self.n, np.int32)
        npart = np.zeros(self.n * HIST_CAP, np.int32)
        nxi = np.zeros(self.n * HIST_CAP * 3, np.float32)
        ovf = c_int64()
        hovf = c_int64()
        lib().dem_compute_rhs(ctypes.byref(self.p), self.n, _p(self.state), _p(self.radius),
                              _p(self.mass), _p(self.hcnt), _p(self.hpart), _p(self.hxi),
                              _p(nc), _p(npart), _p(nxi), _p(out), ctypes.byref(ovf),
                              ctypes.byref(hovf))
        return out

    def deposit(self) -> np.ndarray:
        nodes = self.p.dgrid[0] * self.p.dgrid[1] * self.p.dgrid[2]
        out = np.empty(4 * nodes, np.float64)
        lib().dem_deposit(ctypes.byref(self.p), self.n, _p(self.state), _p(self.mass), _p(out))
        return out

    def energy(self) -> float:
        ovf = c_int64()
        e = lib().dem_energy(ctypes.byref(self.p), self.n, _p(self.state), _p(self.radius),
                             _p(self.mass), _p(self.hcnt), _p(self.hpart), _p(self.hxi),
                             ctypes.byref(ovf))
        self.overflow += ovf.value
        return float(e)

    def momentum(self) -> np.ndarray:
        out = np.zeros(3, np.float64)
        lib().dem_momentum(self.n, _p(self.state), _p(self.mass), _p(out))
        return out


class ReferenceSim:
    """The reference's own ParticleDynamics (CUDA, sm_100a) via oracle/_ref."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        from . import build as oracle_build
        return os.path.exists(oracle_build.REF_LIB)

    @classmethod
    def library(cls) -> ctypes.CDLL:
        if cls._lib is None:
            from . import build as oracle_build
            L = ctypes.CDLL(oracle_build.REF_LIB)
            vp = c_void_p
            L.ref_create.argtypes = [ctypes.c_char_p]
            L.ref_create.restype = vp
            for name in ("ref_destroy",):
                getattr(L, name).argtypes = [vp]
            L.ref_n.argtypes = [vp]
            L.ref_n.restype = c_int
            L.ref_step.argtypes = [vp, c_int]
            L.ref_set_dt.argtypes = [vp, c_float]
            L.ref_time.argtypes = [vp]
            L.ref_time.restype = c_float
            for name in ("ref_get_state", "ref_set_state", "ref_get_rhs", "ref_get_neighbors",
                         "ref_density"):
                getattr(L, name).argtypes = [vp, vp]
            L.ref_neighbor_stride.argtypes = [vp]
            L.ref_neighbor_stride.restype = c_int
            L.ref_density_nodes.argtypes = [vp]
            L.ref_density_nodes.restype = ctypes.c_longlong
            L.ref_energy.argtypes = [vp]
            L.ref_energy.restype = c_float
            L.ref_overflow.argtypes = [vp]
            L.ref_overflow.restype = c_int
            L.ref_is_stable.argtypes = [vp]
            L.ref_is_stable.restype = c_int
            L.ref_max_accel.argtypes = [vp]
            L.ref_max_accel.restype = c_float
            cls._lib = L
        return cls._lib

    def __init__(self, yaml_path: str):
        self.L = self.library()
        self.h = self.L.ref_create(str(yaml_path).encode())
        self.n = self.L.ref_n(self.h)

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, k: int = 1):
        self.L.ref_step(self.h, k)

    def state(self) -> np.ndarray:
        out = np.empty(6 * self.n, np.float32)
        self.L.ref_get_state(self.h, _p(out))
        return out

    def set_state(self, st) -> None:
        st = np.ascontiguousarray(st, np.float32).reshape(-1)
        self.L.ref_set_state(self.h, _p(st))

    def rhs(self) -> np.ndarray:
        out = np.empty(6 * self.n, np.float32)
        self.L.ref_get_rhs(self.h, _p(out))
        return out

    def neighbor_sets(self) -> list[np.ndarray]:
        stride = self.L.ref_neighbor_stride(self.h)
        raw = np.empty(self.n * stride, np.int32)
        self.L.ref_get_neighbors(self.h, _p(raw))
        raw = raw.reshape(self.n, stride)
        out = []
        for row in raw:
            end = np.argmax(row < 0) if (row < 0).any() else stride
            out.append(np.sort(row[:end]))
        return out

    def density(self) -> np.ndarray:
        nodes = self.L.ref_density_nodes(self.h)
        out = np.empty(4 * nodes, np.float32)
        self.L.ref_density(self.h, _p(out))
        return out

    def energy(self) -> float:
        return float(self.L.ref_energy(self.h))

    def overflow(self) -> int:
        return int(self.L.ref_overflow(self.h))
