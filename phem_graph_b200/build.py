"""Builds libphem.so in-tree: the sm_100a CUDA kernels, the C ABI and the
synthetic-input generators; and libphem_gen.so, the generators alone.

    python -m phem_graph_b200.build            # incremental
    python -m phem_graph_b200.build --force    # rebuild everything

nvcc cross-compiles sm_100a without a GPU, so this runs on any machine with
CUDA 12.9.  Objects go to phem_graph_b200/_build/, the library to
phem_graph_b200/libphem.so (both git-ignored; the .so travels with the tree).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libphem.so"
GEN_LIB = PKG / "libphem_gen.so"  # the host generators alone (no CUDA)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
    "--expt-relaxed-constexpr", "-I", str(ROOT / "include"),
]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-pthread", "-I", str(ROOT / "include")]

CU_SOURCES = ["api.cu", "cc.cu", "msf.cu", "csr.cu", "noalloc.cu", "batch.cu", "batch_api.cu", "server.cu",
              "gen_dev.cu"]
CXX_SOURCES = ["gen.cpp", "io.cpp"]
HEADERS = ["common.cuh", "internal.h", "batch.h", "uf.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: CUDA 12.9 toolkit required to build libphem.so")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:4])} ...")


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [ROOT / "include" / "phem.h"]
    objs = []
    jobs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([nvcc(), *NVCC_FLAGS, "-c", str(s), "-o", str(o)])
    for src in CXX_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(["g++", *CXX_FLAGS, "-c", str(s), "-o", str(o)])
    procs = [(cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
             for cmd in jobs]
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose and out:
            sys.stderr.write(out)
        if p.returncode != 0:
            sys.stderr.write(out)
            failed = True
    if failed:
        raise RuntimeError("libphem.so: compilation failed")
    if force or jobs or _stale(LIB, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xcompiler", "-pthread"])
    gen_obj = BUILD / "gen.cpp.o"
    if force or _stale(GEN_LIB, [gen_obj]):
        _run(["g++", "-shared", "-pthread", "-o", str(GEN_LIB), str(gen_obj)])
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
