"""Build libdgswem_cuda.so (sm_100a) in-tree, and the oracle used by the tests.

    python -m dgswem_b200.build            # library + oracle
    python -m dgswem_b200.build --lib-only

The library is compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a``
only; there is no other architecture and no CPU fallback.
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
LIBDIR = PKG / "lib"
LIBNAME = "libdgswem_cuda.so"
# (source, extra nvcc flags): the strict kernel variant is compiled without
# fused multiply-add contraction; the mixed one is the fast one with FP32
# edge and volume arithmetic, whose FP32 divisions and square roots are the
# approximate ones (the flags do not change FP64 operations)
SOURCES = [("hydro.cu", []), ("kernels_fast.cu", ["-fmad=true"]), ("kernels_strict.cu", ["-fmad=false"]),
           ("kernels_mixed.cu", ["-fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"]),
           ("adjoint.cu", ["-fmad=true"]), ("kernels_p2_fast.cu", ["-fmad=true"]),
           ("kernels_p2_strict.cu", ["-fmad=false"]),
           ("kernels_p2_mixed.cu", ["-fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"]),
           ("deck.cpp", []), ("partition.cpp", [])]
HEADERS = ["cr_math.cuh", "hydro_device.cuh", "hydro_kernels.cuh", "hydro_p2.cuh", "kernel_launch.inc", "abi_util.h", "partition.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# host code is compiled with OpenMP (the deck reader's tables, the edge search,
# the device numbering and geometry table use all host threads)
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O2,-fopenmp", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libdgswem_cuda")
    return path


def host_cxx() -> str:
    # the image's default $CXX wrapper lacks libgomp; plain g++ is used for host code
    return shutil.which("g++") or "g++"


def _stale(target: Path, inputs) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in inputs)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    LIBDIR.mkdir(exist_ok=True)
    out = LIBDIR / LIBNAME
    inputs = [CSRC / s for s, _ in SOURCES] + [CSRC / h for h in HEADERS] + [ROOT / "include" / "dgswem_cuda.h",
                                                                            Path(__file__)]
    if not force and not _stale(out, inputs):
        return out
    objs, cmds = [], []
    build = PKG / "_build"
    build.mkdir(exist_ok=True)
    for src, extra in SOURCES:
        obj = build / (Path(src).stem + ".o")
        cmd = [nvcc(), "-ccbin", host_cxx(), *NVCC_FLAGS, *extra, *ARCH, "-I", str(ROOT / "include"), "-I", str(CSRC),
               "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(str(obj))
    # the translation units compile independently: one nvcc per unit at once
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for r in list(pool.map(lambda c: subprocess.run(c, check=False), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    link = [nvcc(), "-ccbin", host_cxx(), "-shared", "-Xcompiler", "-fopenmp", *ARCH, "-o", str(out), *objs]
    subprocess.run(link, check=True)
    return out


def build_oracle() -> Path:
    """Compile the test-only oracle (oracle/Makefile) into oracle/_build/."""
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    return ROOT / "oracle" / "_build" / "liboracle.so"


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--lib-only", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register/spill report")
    args = ap.parse_args(argv)
    print(build_library(force=args.force, verbose=args.verbose))
    if not args.lib_only:
        print(build_oracle())
    return 0


if __name__ == "__main__":
    sys.exit(main())
