"""ParticleDynamics: the reference's step interface over libworld_b200.

Same members and methods as the reference's class (src/particle_dynamics.h:17-141):
`n`, `dt` (writable, re-applied every step), `time`, `positions`, `host_state`,
`host_mass` (per material), `host_material`, `host_density_grid`, grid sizes,
`take_step()`, `unpack_state()`, `compute_density_grid()`, `density_grid_nodes()`,
`compute_total_energy()`, `is_stable()`, `compute_max_acceleration()`,
`grid_overflow_count()` and the four `*_wct()` timers. `device_state.copy_from_host(
host_state)` pushes an edited host state, as the reference's tests do.

Additions: construction from arrays (per-grain radius and mass), `advance(k)`,
FP64 `compute_momentum()`, tangential history get/set, PyTorch zero-copy state
access, and the parity probes (cell keys, sorted order, candidate lists).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from ._lib import WD_HIST_CAP, check, lib, ptr
from .config import SimConfig


class _DeviceState:
    """`sim.device_state.copy_from_host(sim.host_state)` as in the reference tests."""

    def __init__(self, sim: "ParticleDynamics"):
        self._sim = sim

    def copy_from_host(self, host_state: np.ndarray) -> None:
        self._sim.set_state(host_state)


class ParticleDynamics:
    def __init__(self, config: Optional[SimConfig] = None, *, state: Optional[np.ndarray] = None,
                 material: Optional[np.ndarray] = None, radius: Optional[np.ndarray] = None,
                 mass: Optional[np.ndarray] = None):
        self.config = config if config is not None else SimConfig()
        h = ctypes.c_void_p()
        if state is None:
            check(lib.wd_create(self.config.handle, ctypes.byref(h)))
        else:
            st = np.ascontiguousarray(state, dtype=np.float32).reshape(-1)
            n = st.size // 6
            mat = None if material is None else np.ascontiguousarray(material, dtype=np.int32)
            rad = None if radius is None else np.ascontiguousarray(radius, dtype=np.float32)
            ms = None if mass is None else np.ascontiguousarray(mass, dtype=np.float32)
            for name, arr in (("material", mat), ("radius", rad), ("mass", ms)):
                if arr is not None and arr.size != n:
                    raise ValueError(f"{name} has {arr.size} entries for {n} grains")
            check(lib.wd_create_from_arrays(self.config.handle, n, ptr(st), ptr(mat), ptr(rad),
                                            ptr(ms), ctypes.byref(h)))
        self._attach(h)

    def _attach(self, h: ctypes.c_void_p) -> None:
        self._h = h
        n64 = ctypes.c_int64()
        check(lib.wd_get_n(h, ctypes.byref(n64)))
        self.n = int(n64.value)
        cfg = self.config
        self.collision_grid_size_x = cfg.collision_grid_size_x
        self.collision_grid_size_y = cfg.collision_grid_size_y
        self.collision_grid_size_z = cfg.collision_grid_size_z
        self.particles_per_cell = cfg.particles_per_cell
        self.density_grid_size_x = cfg.density_grid_size_x
        self.density_grid_size_y = cfg.density_grid_size_y
        self.density_grid_size_z = cfg.density_grid_size_z
        self._dt = float(cfg.dt)
        self.host_mass = np.asarray(cfg.masses, dtype=np.float32)
        self.grain_radius = np.empty(self.n, np.float32)
        self.grain_mass = np.empty(self.n, np.float32)
        self.host_material = np.empty(self.n, np.int32)
        check(lib.wd_get_grain_props(h, ptr(self.grain_radius), ptr(self.grain_mass),
                                     ptr(self.host_material)))
        self.host_state = np.zeros(6 * self.n, np.float32)
        self.positions = np.zeros(3 * self.n, np.float32)
        self.host_density_grid = np.zeros(4 * self.density_grid_nodes(), np.float32)
        self.device_state = _DeviceState(self)
        self.time_unpack_state = 0.0
        self.unpack_state()

    @classmethod
    def from_checkpoint(cls, config: SimConfig, path: str) -> "ParticleDynamics":
        """Resume from write_checkpoint(path): state, time, dt, radii, masses, materials
        and tangential springs; the run continues bit for bit."""
        obj = cls.__new__(cls)
        obj.config = config
        h = ctypes.c_void_p()
        check(lib.wd_create_from_checkpoint(config.handle, str(path).encode(), ctypes.byref(h)))
        obj._attach(h)
        dt = ctypes.c_float()
        check(lib.wd_get_dt(h, ctypes.byref(dt)))
        obj._dt = float(dt.value)
        return obj

    # -- lifetime --------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.wd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # -- time and dt -----------------------------------------------------------------
    @property
    def dt(self) -> float:
        return self._dt

    @dt.setter
    def dt(self, value: float) -> None:
        self._dt = float(np.float32(value))
        check(lib.wd_set_dt(self._h, ctypes.c_float(self._dt)))

    @property
    def time(self) -> float:
        t = ctypes.c_float()
        check(lib.wd_get_time(self._h, ctypes.byref(t)))
        return float(t.value)

    # -- stepping --------------------------------------------------------------------
    def take_step(self) -> None:
        check(lib.wd_step(self._h, 1))

    def advance(self, steps: int) -> None:
        check(lib.wd_step(self._h, int(steps)))

    def synchronize(self) -> None:
        check(lib.wd_synchronize(self._h))

    def picard_stats(self) -> tuple[int, float]:
        it = ctypes.c_int32()
        res = ctypes.c_float()
        check(lib.wd_get_picard_stats(self._h, ctypes.byref(it), ctypes.byref(res)))
        return int(it.value), float(res.value)

    # -- state -----------------------------------------------------------------------
    def unpack_state(self) -> None:
        check(lib.wd_get_state(self._h, ptr(self.host_state)))
        self.positions[:] = self.host_state.reshape(-1, 6)[:, :3].reshape(-1)

    def get_state(self) -> np.ndarray:
        out = np.empty(6 * self.n, np.float32)
        check(lib.wd_get_state(self._h, ptr(out)))
        return out

    def set_state(self, state: np.ndarray) -> None:
        st = np.ascontiguousarray(state, dtype=np.float32).reshape(-1)
        if st.size != 6 * self.n:
            raise ValueError(f"state has {st.size} floats, expected {6 * self.n}")
        check(lib.wd_set_state(self._h, ptr(st)))

    def get_positions(self) -> np.ndarray:
        out = np.empty(3 * self.n, np.float32)
        check(lib.wd_get_positions(self._h, ptr(out)))
        return out

    def get_rhs(self) -> np.ndarray:
        out = np.empty(6 * self.n, np.float32)
        check(lib.wd_get_rhs(self._h, ptr(out)))
        return out

    # PyTorch zero-copy (CUDA tensors, AoS by grain id); ordered on the sim's stream
    def state_tensor(self, out=None):
        import torch
        if out is None:
            out = torch.empty(6 * self.n, dtype=torch.float32, device="cuda")
        check(lib.wd_get_state_device(self._h, ptr(out)))
        check(lib.wd_synchronize(self._h))
        return out

    def set_state_tensor(self, t) -> None:
        import torch
        torch.cuda.current_stream().synchronize()
        check(lib.wd_set_state_device(self._h, ptr(t.contiguous())))

    # -- reverse pass (CUDA tensors, AoS3 by grain id) ---------------------------------
    def set_contact_params(self, mu: float, restitution: float, k_n: float) -> None:
        check(lib.wd_set_contact_params(self._h, ctypes.c_float(mu), ctypes.c_float(restitution),
                                        ctypes.c_float(k_n)))

    def adjoint_record(self, steps: int, checkpoint_every: int = 20) -> None:
        check(lib.wd_adjoint_record(self._h, int(steps), int(checkpoint_every)))

    def adjoint_backward(self, gx=None, gv=None):
        """(dL/dx0, dL/dv0 as (n, 3) CUDA tensors, dL/d(mu, e, k_n) as a float64 array)
        for dL/dx, dL/dv at the end of the recorded window."""
        import torch
        dev = torch.device("cuda")
        gx_ = None if gx is None else gx.detach().to(dev, torch.float32).contiguous()
        gv_ = None if gv is None else gv.detach().to(dev, torch.float32).contiguous()
        gx0 = torch.empty((self.n, 3), dtype=torch.float32, device=dev)
        gv0 = torch.empty((self.n, 3), dtype=torch.float32, device=dev)
        theta = np.zeros(3, np.float64)
        torch.cuda.current_stream().synchronize()
        check(lib.wd_adjoint_backward(self._h, ptr(gx_), ptr(gv_), ptr(gx0), ptr(gv0), ptr(theta)))
        return gx0, gv0, theta

    def deposit_vjp(self, ggrid):
        """(dL/dx, dL/dv) as (n, 3) CUDA tensors for dL/dgrid (4 * nodes) at the current state."""
        import torch
        dev = torch.device("cuda")
        g = ggrid.detach().to(dev, torch.float32).contiguous()
        gx = torch.empty((self.n, 3), dtype=torch.float32, device=dev)
        gv = torch.empty((self.n, 3), dtype=torch.float32, device=dev)
        torch.cuda.current_stream().synchronize()
        check(lib.wd_deposit_vjp(self._h, ptr(g), ptr(gx), ptr(gv)))
        return gx, gv

    # -- files and frames ------------------------------------------------------------
    def write_state_file(self, path: str) -> None:
        """The reference's state file (int32 n + 6n float32), for initialize_from_file."""
        check(lib.wd_write_state_file(self._h, str(path).encode()))

    def write_checkpoint(self, path: str) -> None:
        """State file at path plus path + ".sidecar" (time, dt, radii, masses,
        materials, tangential springs) for a bit-identical resume."""
        check(lib.wd_write_checkpoint(self._h, str(path).encode()))

    def pack_frame(self, meta5=None) -> np.ndarray:
        """The broadcast frame: 3n positions, time, then the five meta floats
        (real-time ratio and the four phase times in ms)."""
        out = np.empty(3 * self.n + 6, np.float32)
        m = None if meta5 is None else np.ascontiguousarray(meta5, np.float32)
        if m is not None and m.size != 5:
            raise ValueError("meta5 needs 5 floats")
        check(lib.wd_pack_frame(self._h, ptr(m), ptr(out)))
        return out

    # -- tangential history ----------------------------------------------------------
    def get_history(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        cnt = np.zeros(self.n, np.int32)
        part = np.zeros(self.n * WD_HIST_CAP, np.int32)
        xi = np.zeros(self.n * WD_HIST_CAP * 3, np.float32)
        check(lib.wd_get_history(self._h, ptr(cnt), ptr(part), ptr(xi)))
        return cnt, part, xi

    def set_history(self, count, partner, xi) -> None:
        check(lib.wd_set_history(self._h, ptr(np.ascontiguousarray(count, np.int32)),
                                 ptr(np.ascontiguousarray(partner, np.int32)),
                                 ptr(np.ascontiguousarray(xi, np.float32))))

    # -- fields ----------------------------------------------------------------------
    def density_grid_nodes(self) -> int:
        v = ctypes.c_int64()
        check(lib.wd_density_grid_nodes(self._h, ctypes.byref(v)))
        return int(v.value)

    def compute_density_grid(self) -> int:
        check(lib.wd_compute_density_grid(self._h, ptr(self.host_density_grid)))
        return int(self.host_density_grid.size)

    def compute_total_energy(self) -> float:
        e = ctypes.c_double()
        check(lib.wd_compute_total_energy(self._h, ctypes.byref(e)))
        return float(e.value)

    def grain_energies(self) -> np.ndarray:
        """Per-grain energy terms by grain id (float64): each pair's and each spring's
        energy is carried by the smaller-id grain of the pair, so any partition of the
        grains sums to compute_total_energy()."""
        out = np.empty(self.n, np.float64)
        check(lib.wd_grain_energies(self._h, ptr(out)))
        return out

    def compute_momentum(self) -> np.ndarray:
        out = (ctypes.c_double * 3)()
        check(lib.wd_compute_momentum(self._h, out))
        return np.array(list(out), dtype=np.float64)

    # -- diagnostics -----------------------------------------------------------------
    def is_stable(self) -> bool:
        v = ctypes.c_int32()
        check(lib.wd_is_stable(self._h, ctypes.byref(v)))
        return bool(v.value)

    def compute_max_acceleration(self) -> float:
        v = ctypes.c_float()
        check(lib.wd_compute_max_acceleration(self._h, ctypes.byref(v)))
        return float(v.value)

    def grid_overflow_count(self) -> int:
        v = ctypes.c_int64()
        check(lib.wd_grid_overflow_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def history_overflow_count(self) -> int:
        v = ctypes.c_int64()
        check(lib.wd_history_overflow_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def _timings(self) -> np.ndarray:
        out = (ctypes.c_float * 4)()
        check(lib.wd_timings(self._h, out))
        return np.array(list(out), dtype=np.float32)

    def find_neighbors_wct(self) -> float:
        return float(self._timings()[0])

    def compute_rhs_wct(self) -> float:
        return float(self._timings()[1])

    def take_step_wct(self) -> float:
        return float(self._timings()[2])

    def density_grid_wct(self) -> float:
        return float(self._timings()[3])

    def set_kernel_timing(self, enabled: bool) -> None:
        check(lib.wd_set_kernel_timing(self._h, 1 if enabled else 0))

    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        check(lib.wd_get_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def radix_search_count(self) -> tuple[int, int]:
        """(searches that ran the full radix sort, kernels each such search adds)."""
        c = ctypes.c_int64()
        k = ctypes.c_int32()
        check(lib.wd_radix_search_count(self._h, ctypes.byref(c), ctypes.byref(k)))
        return int(c.value), int(k.value)

    def set_neighbor_skin(self, skin: float) -> None:
        check(lib.wd_set_neighbor_skin(self._h, ctypes.c_float(skin)))

    def autotune(self, steps: int = 50, cache: Optional[str] = None) -> tuple[float, int]:
        """Pick the neighbor skin and contact-kernel block size by timing (the state is
        restored afterwards; results do not depend on the choice). Returns them."""
        sk = ctypes.c_float()
        bl = ctypes.c_int32()
        check(lib.wd_autotune(self._h, int(steps), None if cache is None else str(cache).encode(),
                              ctypes.byref(sk), ctypes.byref(bl)))
        return float(sk.value), int(bl.value)

    def tuning(self) -> dict:
        """The current schedule: neighbor skin (m), contact-kernel block size, and the
        list contact kernel's variant."""
        sk = ctypes.c_float()
        bl = ctypes.c_int32()
        rg = ctypes.c_int32()
        check(lib.wd_get_tuning(self._h, ctypes.byref(sk), ctypes.byref(bl), ctypes.byref(rg)))
        return {"neighbor_skin_m": float(sk.value), "contact_block": int(bl.value),
                "contact_variant": {0: "warp-cooperative",
                                    1: "bulk-staged persistent, 48 registers",
                                    2: "bulk-staged persistent, 64 registers",
                                    48: "per-lane, 48 registers",
                                    64: "per-lane, 64 registers"}.get(int(rg.value), str(rg.value))}

    def set_contact_kernel(self, block: int = 256, variant: int = 48) -> None:
        """Contact-kernel block size and list-kernel variant (48 / 64: per-lane with that
        many registers, 0: warp-cooperative, 1 / 2: bulk-staged persistent with 48 / 64
        registers, whose per-slot arrays arrive in shared memory by bulk copies); results
        do not depend on them."""
        check(lib.wd_set_contact_kernel(self._h, int(block), int(variant)))

    def set_build_kernel(self, tiled: bool) -> None:
        """Verlet-list build kernel: per-grain global loads (default) or each block's
        neighbour window staged in shared memory by bulk copies; the same lists."""
        check(lib.wd_set_build_kernel(self._h, 1 if tiled else 0))

    def picard_counts(self) -> tuple[int, int]:
        """(Picard iterations executed, list-mode steps redone with the per-iteration
        search) so far."""
        it, redo = ctypes.c_int64(), ctypes.c_int64()
        check(lib.wd_picard_counts(self._h, ctypes.byref(it), ctypes.byref(redo)))
        return int(it.value), int(redo.value)

    def list_exact_count(self) -> int:
        """Steps so far whose contact kernel measured the exact displacement since the
        last list build (the others decide on a bound and read no build positions)."""
        v = ctypes.c_int64()
        check(lib.wd_list_exact_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def list_resort_count(self) -> int:
        """(grain, step) pairs so far whose contacts a cell crossing had re-ordered, so
        that the list kernel evaluated them in sorted order."""
        v = ctypes.c_int64()
        check(lib.wd_list_resort_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def list_stats(self) -> tuple[int, int, float]:
        """(Verlet-list builds so far, kernels each build launches, mean list length)."""
        b = ctypes.c_int64()
        k = ctypes.c_int32()
        m = ctypes.c_double()
        check(lib.wd_list_stats(self._h, ctypes.byref(b), ctypes.byref(k), ctypes.byref(m)))
        return int(b.value), int(k.value), float(m.value)

    def kernels_per_step(self) -> int:
        v = ctypes.c_int64()
        check(lib.wd_kernels_per_step(self._h, ctypes.byref(v)))
        return int(v.value)

    # -- parity probes ---------------------------------------------------------------
    def debug_cell_keys(self) -> np.ndarray:
        out = np.empty(self.n, np.int32)
        check(lib.wd_debug_cell_keys(self._h, ptr(out)))
        return out

    def debug_sorted(self) -> tuple[np.ndarray, np.ndarray]:
        keys = np.empty(self.n, np.int32)
        ids = np.empty(self.n, np.int32)
        check(lib.wd_debug_sorted(self._h, ptr(keys), ptr(ids)))
        return keys, ids

    def debug_candidates(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        offsets = np.zeros(self.n + 1, np.int64)
        total = ctypes.c_int64()
        check(lib.wd_debug_candidates(self._h, ptr(offsets), None, None, 0, ctypes.byref(total)))
        cand = np.empty(max(int(total.value), 1), np.int32)
        contact = np.empty(max(int(total.value), 1), np.uint8)
        check(lib.wd_debug_candidates(self._h, ptr(offsets), ptr(cand), ptr(contact),
                                      int(total.value), ctypes.byref(total)))
        t = int(total.value)
        return offsets, cand[:t], contact[:t]
