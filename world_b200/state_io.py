"""Initial states and the reference's state file format.

State file (reader: src/particle_dynamics.cu:212-235; writer:
surrogate/decode_particles.py:355-361): little-endian int32 n, then n*6 float32 laid
out [x, y, z, vx, vy, vz] per grain. Grains get `initialization.particle_material`.

Checkpoint sidecar ("<state file>.sidecar", written by wd_write_checkpoint):
"WDCKPT01", uint32 version 2, uint32 flags (bit 0: springs), int64 n, float32 time,
float32 dt, uint64 state_hash (64-bit FNV-1a of the state file's bytes; absent in
version 1), float32 radius[n], float32 mass[n], int32 material[n], and with springs
int32 count[n], int32 partner[n*24], float32 xi[n*24*3]; little-endian, by grain id.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._lib import check, lib, ptr
from .config import SimConfig
from .scenes import grain_properties  # noqa: F401  (pure numpy; re-exported here)


def initial_state(cfg: SimConfig) -> tuple[np.ndarray, np.ndarray]:
    """(state[n, 6] float32, material[n] int32) for cfg's initialization section,
    built by the library's host code exactly as the reference's constructor does."""
    n = ctypes.c_int64()
    check(lib.wd_initial_state(cfg.handle, None, None, 0, ctypes.byref(n)))
    state = np.empty((n.value, 6), np.float32)
    material = np.empty(n.value, np.int32)
    check(lib.wd_initial_state(cfg.handle, ptr(state), ptr(material), n.value, ctypes.byref(n)))
    return state, material


def write_state_file(path: str | os.PathLike, state: np.ndarray) -> None:
    st = np.ascontiguousarray(state, dtype="<f4").reshape(-1, 6)
    with open(path, "wb") as f:
        f.write(np.int32(st.shape[0]).astype("<i4").tobytes())
        f.write(st.tobytes())


def read_state_file(path: str | os.PathLike) -> np.ndarray:
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < 4:
        raise ValueError(f"{path}: missing particle count")
    n = int(np.frombuffer(raw[:4], "<i4")[0])
    if n <= 0:
        raise ValueError(f"{path}: bad particle count {n}")
    body = np.frombuffer(raw[4:], "<f4")
    if body.size < 6 * n:
        raise ValueError(f"{path}: short of {6 * n} floats")
    return body[:6 * n].reshape(n, 6).copy()


CKPT_MAGIC = b"WDCKPT01"


def state_hash(data: bytes) -> int:
    """64-bit FNV-1a of a state file's bytes (the checkpoint sidecar's state_hash)."""
    h = 0xcbf29ce484222325
    for b in data:
        h = ((h ^ b) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    return h
HIST_CAP = 24


def read_checkpoint(path: str | os.PathLike, verify: bool = False) -> dict:
    """The state file at path and its sidecar as arrays (a reader for tooling). With
    `verify`, the sidecar's state_hash is checked against the state file (a pure-Python
    hash: seconds per MB; the library's loader always checks it)."""
    state = read_state_file(path)
    n = state.shape[0]
    with open(str(path) + ".sidecar", "rb") as f:
        raw = f.read()
    if raw[:8] != CKPT_MAGIC:
        raise ValueError(f"{path}.sidecar: bad magic {raw[:8]!r}")
    version, flags = (int(v) for v in np.frombuffer(raw[8:16], "<u4"))
    if version not in (1, 2):
        raise ValueError(f"{path}.sidecar: version {version}")
    sn = int(np.frombuffer(raw[16:24], "<i8")[0])
    if sn != n:
        raise ValueError(f"{path}.sidecar: {sn} grains, state file has {n}")
    time, dt = (float(v) for v in np.frombuffer(raw[24:32], "<f4"))
    o = 32
    out = {"state": state, "time": np.float32(time), "dt": np.float32(dt)}
    if version >= 2:
        out["state_hash"] = int(np.frombuffer(raw[32:40], "<u8")[0])
        if verify:
            with open(path, "rb") as f:
                if state_hash(f.read()) != out["state_hash"]:
                    raise ValueError(f"{path}.sidecar was written with another state file")
        o = 40
    for name, dtype, count in (("radius", "<f4", n), ("mass", "<f4", n), ("material", "<i4", n)):
        out[name] = np.frombuffer(raw[o:o + 4 * count], dtype).copy()
        o += 4 * count
    if flags & 1:
        for name, dtype, count in (("count", "<i4", n), ("partner", "<i4", n * HIST_CAP),
                                   ("xi", "<f4", n * HIST_CAP * 3)):
            out[name] = np.frombuffer(raw[o:o + 4 * count], dtype).copy()
            o += 4 * count
    if o != len(raw):
        raise ValueError(f"{path}.sidecar: {len(raw) - o} trailing bytes")
    return out
