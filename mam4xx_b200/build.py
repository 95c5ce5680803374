"""Build the native libraries in-tree.

  mam4xx_b200/libmam4b.so    sm_100a kernels + C ABI
                             (nvcc -gencode arch=compute_100a,code=sm_100a)
  mam4xx_b200/libmam4b_peaks.so  measurement helper: FP64/FP32 vector peak
                             (csrc/fp_peaks.cu), the FP64 roofline's denominator

Usage: python -m mam4xx_b200.build [--force]
(The CPU checkers have their own recipe, oracle/build_oracle.py.)
"""

import argparse
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mam4xx_b200")
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libmam4b.so")
PEAKS_LIB = os.path.join(PKG, "libmam4b_peaks.so")
PEAKS_SRC = os.path.join(CSRC, "fp_peaks.cu")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    # no FMA contraction: the FP64 step rounds every product and sum as the
    # reference CPU build does, so only libm differs (parity, see tests)
    "--fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_product(force=False):
    srcs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith((".cu", ".cuh", ".inc")) and not f.startswith("_")
            and os.path.join(CSRC, f) != PEAKS_SRC]
    srcs.append(os.path.join(ROOT, "include", "mam4b.h"))
    nvcc = os.environ.get("NVCC", "nvcc")
    if force or not _newer(PEAKS_LIB, [PEAKS_SRC]):
        _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", PEAKS_SRC, "-o", PEAKS_LIB])
    if not force and _newer(LIB, srcs):
        return LIB
    _run([nvcc] + NVCC_FLAGS + [os.path.join(CSRC, "mam4b_step.cu"), "-o", LIB])
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    build_product(force=a.force)


if __name__ == "__main__":
    main()
