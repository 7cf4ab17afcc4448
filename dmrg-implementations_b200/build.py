"""Build the CUDA engine for sm_100a (in-tree).

Produces:
  dmrg2/libdmrg2_b200.so   the engine behind the C ABI of include/dmrg2_b200.h
  bin/dmrg2_gpu             CLI, argv/stdout-compatible with the reference's
                            gpu-rocm/dmrg2-gpu test driver

    python dmrg-implementations_b200/build.py [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "dmrg2" / "libdmrg2_b200.so"
CLI = PKG / "bin" / "dmrg2_gpu"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(REPO / "include")]
LIB_SOURCES = ["gemm.cu", "lanczos.cu", "svd.cu", "eig.cu", "contract.cu", "engine.cu", "capi.cu", "noalloc.cu", "umma.cu", "cholqr.cu", "rsvd.cu"]
CLI_SOURCES = ["cli.cpp", "mpo_builders.cpp"]


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _headers():
    return [p for p in CSRC.iterdir() if p.suffix in (".cuh", ".h")] + [REPO / "include" / "dmrg2_b200.h"]


def _compile(src: str, force: bool) -> Path:
    s = CSRC / src
    o = OBJ / (src + ".o")
    if force or _newer(o, [s] + _headers()):
        cmd = [NVCC] + ARCH + FLAGS + ["-c", str(s), "-o", str(o)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return o


def build(force: bool = False, verbose: bool = True) -> Path:
    OBJ.mkdir(exist_ok=True)
    (PKG / "bin").mkdir(exist_ok=True)
    srcs = LIB_SOURCES + CLI_SOURCES
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = dict(zip(srcs, ex.map(lambda s: _compile(s, force), srcs)))
    lib_objs = [objs[s] for s in LIB_SOURCES]
    if force or _newer(LIB, lib_objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in lib_objs] + ["-lcudart"]
        subprocess.run(cmd, check=True)
    cli_objs = [objs[s] for s in CLI_SOURCES]
    if force or _newer(CLI, cli_objs + [LIB]):
        cmd = [NVCC] + ARCH + ["-o", str(CLI)] + [str(o) for o in cli_objs] + [
            "-L", str(LIB.parent), "-ldmrg2_b200", "-Xlinker", "-rpath=$ORIGIN/../dmrg2", "-lcudart"]
        subprocess.run(cmd, check=True)
    if verbose:
        print(f"built {LIB.relative_to(REPO)} and {CLI.relative_to(REPO)}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
