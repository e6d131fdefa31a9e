"""Builds libtgb200.so, the CUDA backend, in-tree for sm_100a with nvcc.

    python -m terraingen_b200.build            # build if any source is newer than the library
    python -m terraingen_b200.build --force    # rebuild everything

noise.cu is compiled with -fmad=false so its float and double arithmetic rounds exactly as the
reference's -ffp-contract=off build does (bit-exact noise); the other units may contract.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
LIBDIR = PACKAGE / "lib"
LIBRARY = LIBDIR / "libtgb200.so"
INCLUDE = PACKAGE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", "-I", str(CSRC), "-I", str(INCLUDE)]

# Per-unit extra flags.
UNITS = {
    "noise.cu": ["-fmad=false", "-Xcompiler", "-ffp-contract=off"],
    "craters.cu": [],
    "boulders.cu": [],
    "diamond_square.cu": ["-fmad=false"],
    "seams.cu": ["-fmad=false"],
    "datums.cu": ["-fmad=false"],
    "batch.cu": ["-fmad=false"],
    "batch_api.cu": [],
    "serve.cu": [],
    "probe.cu": [],
    "static_scratch.cu": [],
    "api.cu": [],
    "geotiff.cu": [],
    "population.cpp": [],
    "population_gpu.cu": ["-fmad=false"],
    "crater_records.cu": ["-fmad=false"],
}

# Host units are compiled by the host compiler with the reference's floating-point flags, so
# their draws and records round as the reference's do.
HOST_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", str(CSRC), "-I",
              str(INCLUDE)]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libtgb200")
    return path


def sources() -> list[Path]:
    return [CSRC / name for name in UNITS if (CSRC / name).exists()]


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    return any(p.stat().st_mtime > built for p in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return LIBRARY
    LIBDIR.mkdir(exist_ok=True)
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    compiler = nvcc()
    objects = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        if src.suffix == ".cpp":
            cxx = shutil.which("g++") or "g++"
            subprocess.run([cxx, *HOST_FLAGS, *UNITS[src.name], "-c", str(src), "-o", str(obj)],
                           check=True)
            objects.append(str(obj))
            continue
        cmd = [compiler, *ARCH, *COMMON, *UNITS[src.name], "-c", str(src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objects.append(str(obj))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [compiler, *ARCH, "-shared", "-o", str(tmp), *objects, "-lcudart_static", "-lrt",
           "-ldl", "-lpthread", "-lz"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


def main(argv: list[str] | None = None) -> int:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--verbose", action="store_true", help="print ptxas register usage")
    args = parser.parse_args(argv)
    path = build(force=args.force, verbose=args.verbose)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
