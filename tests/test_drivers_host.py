"""The dataset and chaos drivers' argument and input checks, which run before any
device call, and the dataset reader on a hand-made file."""
from __future__ import annotations

import os

import numpy as np
import pytest

from driver_cases import DESIGN_CSV, run_driver, write_blob
from world_b200 import dataset_io


@pytest.fixture(scope="module", autouse=True)
def _drivers(_built):
    import importlib.util
    from conftest import ROOT
    spec = importlib.util.spec_from_file_location("wb_build", os.path.join(ROOT, "world_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build_drivers()


def test_dataset_missing_design(tmp_path):
    cfg = write_blob(tmp_path / "blob.yaml")
    r = run_driver("dataset", [cfg, tmp_path / "none.csv", tmp_path / "out"], tmp_path)
    assert r.returncode == 1
    assert "could not open design" in r.stderr


def test_dataset_unknown_column_writes_nothing(tmp_path):
    cfg = write_blob(tmp_path / "blob.yaml")
    (tmp_path / "d.csv").write_text("throw_vx,spin\n1.0,2.0\n")
    r = run_driver("dataset", [cfg, tmp_path / "d.csv", tmp_path / "out"], tmp_path)
    assert r.returncode == 1
    assert "design column 'spin' is not a known parameter" in r.stderr
    assert not (tmp_path / "out").exists()


def test_dataset_ragged_row(tmp_path):
    cfg = write_blob(tmp_path / "blob.yaml")
    (tmp_path / "d.csv").write_text("throw_vx,friction\n1.0\n")
    r = run_driver("dataset", [cfg, tmp_path / "d.csv", tmp_path / "out"], tmp_path)
    assert r.returncode == 1
    assert "design row has 1 values, expected 2" in r.stderr


def test_dataset_nothing_to_do(tmp_path):
    cfg = write_blob(tmp_path / "blob.yaml", checkpoints=0)
    (tmp_path / "d.csv").write_text(DESIGN_CSV)
    r = run_driver("dataset", [cfg, tmp_path / "d.csv", tmp_path / "out"], tmp_path)
    assert r.returncode == 1
    assert "nothing to do (5 rollouts, 0 checkpoints)" in r.stderr
    (tmp_path / "e.csv").write_text("friction\n")
    cfg = write_blob(tmp_path / "blob2.yaml")
    r = run_driver("dataset", [cfg, tmp_path / "e.csv", tmp_path / "out"], tmp_path)
    assert r.returncode == 1
    assert "nothing to do (0 rollouts" in r.stderr


def test_chaos_needs_a_perturbation(tmp_path):
    cfg = write_blob(tmp_path / "blob.yaml")
    r = run_driver("chaos", [cfg, 4], tmp_path)
    assert r.returncode == 1
    assert "perturbation is 0" in r.stderr


def test_dataset_reader_round_trip(tmp_path):
    R, K, C, nx, ny, nz, P = 3, 2, 4, 2, 3, 2, 2
    rng = np.random.default_rng(0)
    grids = rng.random((R, K, C, nx, ny, nz)).astype(np.float32)
    times = np.array([0.5, 1.0], np.float32)
    with open(tmp_path / "grids.bin", "wb") as f:
        f.write(b"RTPGRD01")
        f.write(np.array([R, K, C, nx, ny, nz, P], "<i4").tobytes())
        f.write(times.tobytes())
        f.write(grids.tobytes())
    (tmp_path / "manifest.csv").write_text(
        "rollout,a,b,status,final_time,overflow_cells,deposited_mass\n"
        "0,1,2,ok,1,0,3.5\n1,3,4,diverged,0.5,7,0\n2,5,6,ok,1,0,2.25\n")
    d = dataset_io.load(str(tmp_path))
    np.testing.assert_array_equal(d.grids, grids)
    np.testing.assert_array_equal(d.checkpoint_times, times)
    assert d.parameter_names == ["a", "b"]
    np.testing.assert_array_equal(d.parameters, [[1, 2], [3, 4], [5, 6]])
    assert list(d.ok) == [True, False, True]
    assert d.overflow_cells.tolist() == [0, 7, 0]
    with open(tmp_path / "grids.bin", "ab") as f:
        f.write(b"\0\0\0\0")
    with pytest.raises(ValueError):
        dataset_io.load(str(tmp_path))
