"""Builds libflame3d_b200.so in-tree with nvcc for sm_100a (B200).

Every translation unit under csrc/ is compiled separately (so per-file flags are possible) and
linked into one shared library next to this file.  The library has a plain C ABI
(include/flame3d_b200.h); nothing in it depends on torch or Python.

    python flame3d.jl_b200/build.py [--force] [--verbose-ptxas]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
BUILD = HERE / "_build"
LIB = HERE / "libflame3d_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "--expt-relaxed-constexpr", "-I", str(INCLUDE)]
# The 1:1 kernels keep every multiply and add separately rounded, so they match a strict IEEE
# evaluation of the reference arithmetic bit for bit.  The fused kernels let ptxas contract.
PER_FILE = {
    "kernels_ref.cu": ["-fmad=false"],
    "chemistry.cu": ["-fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA 12.9 toolkit is required to build")


def host_compiler() -> list[str]:
    # The image exports CXX as a wrapper; nvcc wants a plain g++ for its host passes.
    gxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else shutil.which("g++")
    return ["-ccbin", gxx] if gxx else []


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources() + headers() + [Path(__file__)])


def compile_one(src: Path, verbose_ptxas: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    cmd = [nvcc(), *host_compiler(), *ARCH, *COMMON, *PER_FILE.get(src.name, []), "-c",
           str(src), "-o", str(obj)]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas and r.stderr:
        print(r.stderr, file=sys.stderr)
    return obj


PROBE_SRC = CSRC / "probe" / "fp64_peak.cu"
PROBE_LIB = HERE / "libflame3d_probe.so"


def build_probe(force: bool = False) -> Path:
    """libflame3d_probe.so: the FP64 FMA throughput probe bench.py measures the compute roof
    with (kept out of the reference-facing library)."""
    if not force and PROBE_LIB.exists() and PROBE_LIB.stat().st_mtime > PROBE_SRC.stat().st_mtime:
        return PROBE_LIB
    cmd = [nvcc(), *host_compiler(), *ARCH, *COMMON, "-shared", str(PROBE_SRC), "-o",
           str(PROBE_LIB)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {PROBE_SRC.name}:\n{r.stdout}\n{r.stderr}")
    return PROBE_LIB


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    build_probe(force)
    if not force and not needs_build():
        return LIB
    BUILD.mkdir(exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, verbose_ptxas), sources()))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *host_compiler(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas))
