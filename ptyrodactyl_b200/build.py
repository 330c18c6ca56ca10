"""Compile the sm_100a engine into ``ptyrodactyl_b200/libptyro_b200.so``.

Run ``python -m ptyrodactyl_b200.build`` (or call :func:`build`). nvcc
cross-compiles without a GPU, so this also works on build hosts.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libptyro_b200.so")
SOURCES = ["ms_engine.cu", "diag.cu", "ms_static.cu", "ms_sched.cu", "atoms.cu", "ms_jvp.cu", "ms_resident.cu", "elements.cu", "ms_generic.cu"] + [f"pass_{n}.cu" for n in (16, 32, 64, 128, 256, 512, 1024)]
HEADERS = ["fft_core.cuh", "unit_consts.cuh", "ms_pass.cuh", "ms_pair.cuh", "ms_half.cuh", "ms_bwd.cuh", "ms_bwd_lam.cuh",
           "ms_jvp.cuh", "ms_pipe.cuh", "ms_wait.cuh", "ms_resident.cuh", "pass_launch.cuh", "engine.cuh"]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]
LINK_FLAGS = ["-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a"]
OBJ_DIR = os.path.join(PKG, "_build")


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the sm_100a engine cannot be built")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "ptyro_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """Build the shared library if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = nvcc_path()
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc, *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                            text=True)))
    failed = []
    for src, pr in procs:
        out, _ = pr.communicate()
        if verbose and out:
            print(out)
        if pr.returncode != 0:
            failed.append((src, out))
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(f"{s}:\n{o}" for s, o in failed))
    cmd = [nvcc, *LINK_FLAGS, *objs, "-o", LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(force=True, verbose=True, extra=extra))
