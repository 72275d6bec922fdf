"""Build libworld_b200.so in-tree for sm_100a.

Every CUDA translation unit is compiled with nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) and -fmad=false: the kernels spell out
their fused multiply-adds, so the CPU oracle can reproduce them bit for bit. The
host translation units go through the same nvcc driver (g++ underneath, no -march
flags, so host float arithmetic matches the reference's own host code).

    python -m world_b200.build        # or world_b200.build.build()
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libworld_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-fmad=false",
                     "-Xcompiler", "-fPIC,-O2,-fno-fast-math", "-Xptxas", "-O3",
                     f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}"]
RDC_SOURCES = {"wd_launch.cu"}
BIN = os.path.join(HERE, "bin")
DRIVERS = ["dataset", "chaos"]
SOURCES = ["wd_search.cu", "wd_contact.cu", "wd_lists.cu", "wd_fields.cu", "wd_ensemble.cu",
           "wd_adjoint.cu", "wd_launch.cu",
           "wd_sim.cu",
           "wd_config.cpp", "wd_io.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the sm_100a library cannot be built")


def _compile(src: str, extra: list[str]) -> str:
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "world_b200.h"))
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    # relocatable device code only where the device runtime is called (the list build's
    # device-side graph launches); elsewhere it would put the call ABI on every kernel
    rdc = ["-rdc=true"] if src in RDC_SOURCES else []
    cmd = [nvcc()] + CUDA_FLAGS + rdc + extra + ["-x", "cu" if src.endswith(".cu") else "c++",
                                                 "-c", path, "-o", out]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return out


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    extra = extra or []
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), SOURCES))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(o) for o in objs):
        return LIB
    # -rdc=true at the link runs the device link of wd_launch.cu against the device runtime
    cmd = [nvcc()] + ARCH + ["-rdc=true", "-shared", "-o", LIB] + objs + [
        "-lcudadevrt", "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


def build_drivers(verbose: bool = False) -> list[str]:
    """The dataset and chaos drivers (world_b200/drivers/*.cpp), linked against the
    library with an rpath to it, into world_b200/bin/."""
    lib = build(verbose=verbose)
    os.makedirs(BIN, exist_ok=True)
    outs = []
    for name in DRIVERS:
        src = os.path.join(HERE, "drivers", name + ".cpp")
        out = os.path.join(BIN, name)
        deps = [src, lib] + [os.path.join(ROOT, "include", "world_b200", h)
                             for h in os.listdir(os.path.join(ROOT, "include", "world_b200"))]
        if not (os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps)):
            cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-Wall",
                   f"-I{os.path.join(ROOT, 'include')}", src, "-o", out,
                   f"-L{HERE}", "-lworld_b200", "-Wl,-rpath,$ORIGIN/.."]
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                raise RuntimeError(f"driver build failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
            if verbose:
                print(f"built {out}")
        outs.append(out)
    return outs


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
    build_drivers(verbose=True)
