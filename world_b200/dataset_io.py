"""Reader of the dataset the dataset driver writes (world_b200/bin/dataset).

The format is the reference's (written by src/dataset.cpp:163-232, read by
surrogate/dataset_io.py:8-17), so its surrogate tooling reads our output unchanged:

    grids.bin     char magic[8] = "RTPGRD01"
                  int32 rollouts, checkpoints, channels (4), nx, ny, nz, parameters
                  float32 checkpoint_times[checkpoints]
                  float32 grids[rollouts][checkpoints][channels][nx][ny][nz]
    manifest.csv  rollout, <parameters...>, status, final_time, overflow_cells,
                  deposited_mass   (status "ok" | "diverged"; diverged rows zero-filled)

Also the chaos driver's final_fields.bin: int32 members, int32 nodes, then each
member's terminal mass field (float32[nodes]), member 0 first.
"""
from __future__ import annotations

import csv
import os
from dataclasses import dataclass

import numpy as np

MAGIC = b"RTPGRD01"


@dataclass
class Dataset:
    grids: np.ndarray             # (rollouts, checkpoints, channels, nx, ny, nz) float32
    checkpoint_times: np.ndarray  # (checkpoints,) float32
    parameters: np.ndarray        # (rollouts, parameters) float64
    parameter_names: list[str]
    status: list[str]
    final_time: np.ndarray        # (rollouts,) float64
    overflow_cells: np.ndarray    # (rollouts,) int64
    deposited_mass: np.ndarray    # (rollouts,) float64

    @property
    def ok(self) -> np.ndarray:
        return np.array([s == "ok" for s in self.status])


def load(directory: str, mmap: bool = False) -> Dataset:
    grid_path = os.path.join(directory, "grids.bin")
    with open(grid_path, "rb") as f:
        magic = f.read(8)
        if magic != MAGIC:
            raise ValueError(f"{grid_path}: bad magic {magic!r}")
        head = np.frombuffer(f.read(28), dtype="<i4")
        R, K, C, nx, ny, nz, P = (int(v) for v in head)
        times = np.frombuffer(f.read(4 * K), dtype="<f4").copy()
        offset = f.tell()
    expected = R * K * C * nx * ny * nz
    actual = (os.path.getsize(grid_path) - offset) // 4
    if actual != expected:
        raise ValueError(f"{grid_path}: {actual} floats after the header, expected {expected}")
    shape = (R, K, C, nx, ny, nz)
    if mmap:
        grids = np.memmap(grid_path, dtype="<f4", mode="r", offset=offset, shape=shape)
    else:
        grids = np.fromfile(grid_path, dtype="<f4", offset=offset, count=expected).reshape(shape)
    with open(os.path.join(directory, "manifest.csv"), newline="") as f:
        rows = list(csv.reader(f))
    header, body = rows[0], rows[1:]
    if len(body) != R:
        raise ValueError(f"manifest has {len(body)} rows, grids has {R}")
    si = header.index("status")
    return Dataset(
        grids=grids, checkpoint_times=times,
        parameters=np.array([[float(v) for v in r[1:1 + P]] for r in body], np.float64).reshape(R, P),
        parameter_names=header[1:1 + P],
        status=[r[si] for r in body],
        final_time=np.array([float(r[si + 1]) for r in body]),
        overflow_cells=np.array([int(r[si + 2]) for r in body], np.int64),
        deposited_mass=np.array([float(r[si + 3]) for r in body]))


def load_final_fields(path: str) -> np.ndarray:
    """(members, nodes) float32 from the chaos driver's final_fields.bin."""
    with open(path, "rb") as f:
        members, nodes = (int(v) for v in np.frombuffer(f.read(8), dtype="<i4"))
        data = np.frombuffer(f.read(), dtype="<f4")
    if data.size != members * nodes:
        raise ValueError(f"{path}: {data.size} floats, expected {members * nodes}")
    return data.reshape(members, nodes)
