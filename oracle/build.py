"""Build recipe for the oracle (test infrastructure, never the product).

Outputs:
  oracle/_build/libdem_oracle.so   the CPU restatement (dem_oracle.c), gcc with
                                   -ffp-contract=off and OpenMP.
  oracle/_ref/libref_world.so      the reference's own step: its unmodified sources
                                   compiled where they lie (REFERENCE_SRC below, read
                                   only) for sm_100a, plus ref_harness.cu (C entry
                                   points over its ParticleDynamics). Built only
                                   when the reference tree is present; the compiled
                                   library travels with the repository snapshot.

The reference's own Makefile is not used (it fetches GLFW, GoogleTest and
uWebSockets from the network). Its step needs only the eight src/*.cu files and
src/sim_config.cpp, with the same flags it builds with (-std=c++17 -O3; the arch is
pinned to sm_100a instead of -arch=native).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_LIB = os.path.join(BUILD, "libdem_oracle.so")
REF_LIB = os.path.join(REF_OUT, "libref_world.so")
REFERENCE_SRC = os.environ.get("WORLD_REFERENCE_SRC", "/root/reference/src")

REF_CU = ["kernel", "density_grid_kernel", "compute_rhs_kernel", "particle_dynamics",
          "find_neighbors_kernel", "semi_implicit_euler_kernel",
          "backward_euler_picard_kernel", "energy_kernel"]


def _newer(out: str, deps: list[str]) -> bool:
    return os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps)


def build_oracle() -> str:
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "dem_oracle.c")
    hdr = os.path.join(HERE, "dem_oracle.h")
    if _newer(ORACLE_LIB, [src, hdr]):
        return ORACLE_LIB
    cc = shutil.which("gcc") or "cc"
    cmd = [cc, "-std=c99", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
           "-shared", src, "-o", ORACLE_LIB, "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed: {' '.join(cmd)}\n{res.stderr}")
    return ORACLE_LIB


def build_reference() -> str | None:
    """Compile the reference step for sm_100a. Returns None when the tree is absent."""
    if not os.path.isdir(REFERENCE_SRC):
        return REF_LIB if os.path.exists(REF_LIB) else None
    os.makedirs(os.path.join(REF_OUT, "obj"), exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    flags = ["-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O3",
             "-Xcompiler", "-fPIC", f"-I{REFERENCE_SRC}"]
    jobs = [(os.path.join(REFERENCE_SRC, f + ".cu"), os.path.join(REF_OUT, "obj", f + ".o"))
            for f in REF_CU]
    jobs.append((os.path.join(REFERENCE_SRC, "sim_config.cpp"),
                 os.path.join(REF_OUT, "obj", "sim_config.o")))
    jobs.append((os.path.join(HERE, "ref_harness.cu"), os.path.join(REF_OUT, "obj", "ref_harness.o")))
    headers = [os.path.join(REFERENCE_SRC, h) for h in os.listdir(REFERENCE_SRC) if h.endswith(".h")]

    def one(job):
        src, obj = job
        if _newer(obj, [src] + headers):
            return obj
        cmd = [nvcc] + flags + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", src, "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"reference build failed: {' '.join(cmd)}\n{res.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=8) as ex:
        objs = list(ex.map(one, jobs))
    if not _newer(REF_LIB, objs):
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", REF_LIB] + objs
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"reference link failed: {' '.join(cmd)}\n{res.stderr}")
    return REF_LIB


def build() -> None:
    build_oracle()
    build_reference()


if __name__ == "__main__":
    build()
    print(ORACLE_LIB)
    print(REF_LIB if os.path.exists(REF_LIB) else "(reference not built)")
    sys.exit(0)
