"""Test configuration: the `gpu` marker and shared helpers.

`pytest -m "not gpu"` runs on any machine: the oracle against the reference's golden
vectors and known answers, the config / state-file host logic, and the C ABI's
exports (no device calls). `pytest -m gpu` runs on a B200: the library's kernels
against the oracle (bit for bit) and against the reference's recorded outputs.
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_present() -> bool:
    return os.path.exists("/dev/nvidia0") or shutil.which("nvidia-smi") is not None


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle (and the library if its sources are newer) once per session."""
    from oracle import build as oracle_build
    oracle_build.build_oracle()
    lib = os.path.join(ROOT, "world_b200", "libworld_b200.so")
    if not os.path.exists(lib) and shutil.which("nvcc"):
        import importlib.util
        spec = importlib.util.spec_from_file_location("wd_build", os.path.join(ROOT, "world_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    yield


@pytest.fixture
def oracle_for():
    """OracleSim for a (config, state[n,6], radius, mass) tuple."""
    from oracle.oracle import OracleSim, params_from_config

    def make(cfg, state, radius=None, mass=None, material=None):
        from world_b200.state_io import grain_properties
        st = np.asarray(state, np.float32).reshape(-1, 6)
        mat = np.full(st.shape[0], cfg.particle_material, np.int32) if material is None else material
        r, m = grain_properties(cfg, mat, radius)
        if mass is not None:
            m = np.asarray(mass, np.float32)
        return OracleSim(params_from_config(cfg), st, r, m)

    return make


def load_golden(name: str) -> dict:
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        pytest.fail(f"golden fixture {path} missing (tests/golden/make_golden.py records it)")
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def golden_config(rec: dict, tmp_path):
    """SimConfig and initial state of a golden case, through the library's loader."""
    from world_b200 import SimConfig, load_config
    from cases import write_state
    text = str(rec["yaml"])
    if not text:
        return SimConfig(), rec["state0"].reshape(-1, 6)
    state_path = tmp_path / "state.bin"
    write_state(str(state_path), rec["state0"])
    lines = []
    for line in text.splitlines():
        if line.strip().startswith("state_path:"):
            line = f"  state_path: {state_path}"
        lines.append(line)
    yaml_path = tmp_path / "case.yaml"
    yaml_path.write_text("\n".join(lines) + "\n")
    return load_config(str(yaml_path)), rec["state0"].reshape(-1, 6)


def scaled_error(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| over the largest magnitude of b: relative error at the array's scale."""
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b))) / scale if scale > 0 else float(np.max(np.abs(a - b), initial=0.0))
