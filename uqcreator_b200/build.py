"""Build recipe of the CUDA extension libuqc_b200.so (sm_100a), in-tree.

    python -m uqcreator_b200.build          # or __graft_entry__.build()

Host C++ files are compiled with -ffp-contract=off so tables and mesh
geometry are bit-identical to the reference's; device code uses FMA.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libuqc_b200.so"
BUILD = PKG / "_build"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_SRCS = ["config.cpp", "tables.cpp", "mesh.cpp"]
CUDA_SRCS = ["solver.cu", "kernels_bb.cu", "kernels_euler2d.cu", "kernels_sw.cu", "kernels_linear.cu", "kernels_euler1d.cu", "kernels_logsin.cu"]


def _sources():
    return [CSRC / s for s in HOST_SRCS + CUDA_SRCS] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + \
        [ROOT / "include" / "uqc.h"]


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _sources())


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    common = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-I" + str(ROOT / "include"), "-I" + str(CSRC)]
    jobs = []
    for s in HOST_SRCS:
        o = BUILD / (Path(s).stem + ".o")
        jobs.append((["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-I" + str(ROOT / "include"), "-I" + str(CSRC),
                      "-c", str(CSRC / s), "-o", str(o)], o))
    for s in CUDA_SRCS:
        o = BUILD / (Path(s).stem + ".o")
        jobs.append(([NVCC, *ARCH, "-lineinfo", *common, "-Xptxas", "-v" if verbose else "-O3", "-c", str(CSRC / s), "-o", str(o)], o))
    # the translation units compile in parallel (the kernel units dominate)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
        for f in [ex.submit(_run, cmd, verbose) for cmd, _ in jobs]:
            f.result()
    objs = [o for _, o in jobs]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    _run(cmd, verbose)
    os.replace(tmp, LIB)
    return LIB


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd[:3])} ...")


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(LIB)
