"""The C++ drop-in header (include/world_b200/particle_dynamics.hpp): compiled with
g++ against libworld_b200.so, it runs the reference's own test cases written the way
the reference writes them (tests/cpp/reference_cases.cpp)."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

from conftest import ROOT

LIBDIR = os.path.join(ROOT, "world_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "reference_cases.cpp")


def build(tmp_path) -> str:
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.fail("no C++ compiler to build the drop-in test")
    exe = str(tmp_path / "reference_cases")
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", f"-I{os.path.join(ROOT, 'include')}",
           SRC, "-o", exe, f"-L{LIBDIR}", "-lworld_b200", f"-Wl,-rpath,{LIBDIR}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    assert "warning" not in res.stderr, res.stderr
    return exe


def test_header_compiles_and_config_cases_pass(tmp_path):
    exe = build(tmp_path)
    res = subprocess.run([exe, "config"], capture_output=True, text=True, cwd=tmp_path, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr


@pytest.mark.gpu
def test_reference_cases_through_the_cpp_dropin(tmp_path):
    exe = build(tmp_path)
    res = subprocess.run([exe, "all"], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "12 cases, 0 failed" in res.stdout
