"""Build recipe: nvcc for sm_100a, in-tree outputs under gisspa_b200/lib/.

    python -m gisspa_b200.build            # library + drop-in driver
    python -m gisspa_b200.build --force

Outputs
  gisspa_b200/lib/libgisspa_b200.so   C ABI of include/gisspa.h (CUDA kernels)
  gisspa_b200/lib/gisspa_main         drop-in CLI for the reference's ./main
  gisspa_b200/lib/gisspa_merge        drop-in for its duplicate-merging script
  gisspa_b200/lib/libgisspa_peak.so   FP32 FMA microbenchmark (bench.py's roofline peak)
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(LIBDIR, "libgisspa_b200.so")
DRIVER = os.path.join(LIBDIR, "gisspa_main")
MERGE = os.path.join(LIBDIR, "gisspa_merge")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def _run(cmd, cwd=None) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=cwd)


def build_library(force: bool = False) -> str:
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + glob.glob(os.path.join(CSRC, "*.cpp"))
                  + [os.path.join(INCLUDE, "gisspa.h")])
    if not force and _newer(LIB, srcs):
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    _run([NVCC] + NVCC_FLAGS + ARCH + ["-shared", "-I" + INCLUDE, "-o", LIB,
                                       os.path.join(CSRC, "gisspa.cu"),
                                       os.path.join(CSRC, "noalloc.cu"),
                                       os.path.join(CSRC, "merge.cu"),
                                       os.path.join(CSRC, "hdf5io.cpp"), "-lz"])
    return LIB


PEAK = os.path.join(LIBDIR, "libgisspa_peak.so")


def build_peak(force: bool = False) -> str:
    """FP32 FMA microbenchmark used by bench.py for the roofline peak (not
    part of the search's C ABI)."""
    src = os.path.join(CSRC, "peak", "fma_peak.cu")
    if not force and _newer(PEAK, [src]):
        return PEAK
    os.makedirs(LIBDIR, exist_ok=True)
    _run([NVCC] + NVCC_FLAGS + ARCH + ["-shared", "-o", PEAK, src])
    return PEAK


CPU_BASELINE = os.path.join(ROOT, "oracle", "_cpu", "libgisspa_cpu.so")


def build_cpu_baseline(force: bool = False) -> str:
    """C++/OpenMP restatement of the correlation and scoring (oracle/cpu),
    timed by bench.py as the CPU baseline; x86-64-v3 (AVX2 + FMA) so that it
    runs on any current host."""
    src = os.path.join(ROOT, "oracle", "cpu", "gisspa_cpu.cpp")
    if not force and _newer(CPU_BASELINE, [src]):
        return CPU_BASELINE
    os.makedirs(os.path.dirname(CPU_BASELINE), exist_ok=True)
    _run(["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-std=c++17", "-shared", "-fPIC", "-Wall",
          "-o", CPU_BASELINE, src])
    return CPU_BASELINE


def build_driver(force: bool = False) -> str:
    dsrc = sorted(glob.glob(os.path.join(CSRC, "driver", "*.cpp")))
    deps = dsrc + glob.glob(os.path.join(CSRC, "driver", "*.hpp")) + [LIB, os.path.join(INCLUDE, "gisspa.h")]
    if not force and _newer(DRIVER, deps):
        return DRIVER
    _run(["g++", "-O2", "-std=c++17", "-Wall", "-I" + INCLUDE] + dsrc +
         ["-L" + LIBDIR, "-lgisspa_b200", "-Wl,-rpath,$ORIGIN", "-o", DRIVER])
    return DRIVER


def build_merge_cli(force: bool = False) -> str:
    src = os.path.join(CSRC, "driver", "merge", "merge_main.cpp")
    deps = [src, LIB, os.path.join(INCLUDE, "gisspa.h")]
    if not force and _newer(MERGE, deps):
        return MERGE
    _run(["g++", "-O2", "-std=c++17", "-Wall", "-I" + INCLUDE, src,
          "-L" + LIBDIR, "-lgisspa_b200", "-Wl,-rpath,$ORIGIN", "-o", MERGE])
    return MERGE


def build_reference_checker(ref: Optional[str] = None) -> bool:
    """Compile the reference's own sources (directory `ref`, or the
    GISSPA_REFERENCE environment variable) into oracle/_ref (test
    infrastructure) when they are present on this machine."""
    ref = ref or os.environ.get("GISSPA_REFERENCE")
    if not ref or not os.path.isdir(ref):
        return False
    _run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "ref-default", "REF=" + ref])
    return True


def build_all(force: bool = False, reference: Optional[str] = None) -> None:
    """Library, drop-in driver and merge CLI; the reference checker too when
    `reference` (or GISSPA_REFERENCE) names the reference's source tree."""
    build_library(force)
    build_driver(force)
    build_merge_cli(force)
    build_peak(force)
    build_cpu_baseline(force)
    build_reference_checker(reference)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--reference", default=None,
                    help="reference source tree to build the parity checker from (default: $GISSPA_REFERENCE)")
    a = ap.parse_args()
    build_all(a.force, a.reference)
    return 0


if __name__ == "__main__":
    sys.exit(main())
