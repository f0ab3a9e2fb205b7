"""Builds libgrains_b200.so (sm_100a) and the Basilisk coupling library
libgrains_b200_basilisk.so over it, in the package directory.

Each CUDA translation unit is compiled separately so that the FP64 units can
be built with -fmad=false (no contraction of a*b+c into FMA, which keeps the
FP64 arithmetic in the reference's rounding order) while the FP32-split unit
keeps FMA contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libgrains_b200.so"
# the Basilisk coupling C ABI (host code over libgrains_b200.so)
OUT_BASILISK = PKG / "libgrains_b200_basilisk.so"
BUILD = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(CSRC),
          "-I", str(PKG.parent / "include")]

# (source, extra flags)
UNITS = [
    ("gdem_integrate.cu", ["-fmad=false"]),
    ("gdem_contact64.cu", ["-fmad=false"]),
    ("gdem_contact32.cu", ["-fmad=false"]),
    ("gdem_host.cu", ["-fmad=false"]),
    ("gdem_noalloc.cu", ["-fmad=false"]),
    ("gdem_adjoint.cu", ["-fmad=false"]),
    ("xml_reader.cpp", []),
    ("gdem_rawdata.cpp", []),
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + \
        list((PKG.parent / "include").glob("*.h"))
    objs = []
    for src, flags in UNITS:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if not _stale(o, [s, *headers]) and not ptxas_info:
            continue
        cmd = [_nvcc(), *ARCH, *COMMON, *flags, "-c", str(s), "-o", str(o)]
        if ptxas_info and s.suffix == ".cu":
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if _stale(OUT, objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    src = CSRC / "gdem_basilisk.cpp"
    if _stale(OUT_BASILISK, [src, OUT, *headers]):
        # the system g++ (shared libstdc++, the one the host process loads)
        cmd = [os.environ.get("GRAINS_B200_CXX", "g++"), "-std=c++17", "-O2", "-fPIC", "-shared",
               "-I", str(PKG.parent / "include"), str(src), "-o", str(OUT_BASILISK),
               "-L", str(PKG), "-l:libgrains_b200.so", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
