"""Build recipe of the CPU checkers (test infrastructure only).

  oracle/libmam4oracle.so    gcc, plain C restatement (oracle/mam4_oracle.c)
  oracle/libmam4oracle_ulp.so the same with every libm result moved by a few
                             ulps (seeded): the algorithm's own sensitivity
  oracle/libmam4oracle_gpu.so the same source compiled for the GPU with nvcc
                             (CUDA libm, no FMA contraction): the libm-matched
                             diagnostic oracle
  oracle/libmam4oracle_count.so the restatement compiled as C++ with an
                             operation-counting real type (oracle/opcount.cpp):
                             the algorithmic flop count of the step
  oracle/_ref/libmam4ref.so  g++, the mam4xx reference headers included
                             read-only from <ref>/src and compiled unchanged
                             against the host shim in oracle/shim; built only
                             when the reference tree exists (no cmake, no
                             Kokkos/EKAT: the shim stands in for the small
                             surface the headers use)
  oracle/_ref/libmam4ref_gpu.so  nvcc, the same reference headers compiled
                             unchanged for the GPU (sm_100a) against the
                             same shim in its device mode, CUDA libm, no FMA
                             contraction (oracle/ref/ref_step_gpu.cu): the
                             libm-matched layer of the reference itself
  oracle/_ref/libmam4ref_tuned.so  the same reference build tuned for speed
                             (-O3 -march=x86-64-v3: AVX2 and FMA, FP
                             contraction allowed): the timed CPU baseline;
                             loaded only on hosts with AVX2 and FMA

The parity builds use -O3 -ffp-contract=off so that every expression rounds
in source order, and OpenMP for the multi-core CPU baseline. No
-march=native: the libraries travel to other hosts.

The mam4xx tree is taken from build(ref=...), else from the environment
variable MAM4XX_REFERENCE, else from the default checkout location below.
"""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PORT_SO = os.path.join(HERE, "libmam4oracle.so")
ULP_SO = os.path.join(HERE, "libmam4oracle_ulp.so")
REF_SO = os.path.join(HERE, "_ref", "libmam4ref.so")
REF_TUNED_SO = os.path.join(HERE, "_ref", "libmam4ref_tuned.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libmam4ref_gpu.so")
GPU_SO = os.path.join(HERE, "libmam4oracle_gpu.so")
COUNT_SO = os.path.join(HERE, "libmam4oracle_count.so")
DEFAULT_REF = "/root/reference"  # default checkout of the mam4xx tree
TUNED = ["-O3", "-march=x86-64-v3", "-ffp-contract=fast", "-fPIC", "-shared", "-fopenmp"]

COMMON = ["-O3", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off"]


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(ref=None, force=False):
    deps = [os.path.join(HERE, "mam4_oracle.c"), os.path.join(HERE, "oracle_api.h"),
            os.path.join(ROOT, "include", "mam4b.h"),
            os.path.join(ROOT, "mam4xx_b200", "csrc", "coag_tables.inc")]
    if force or _stale(PORT_SO, deps):
        _run(["gcc", "-std=c99"] + COMMON + [os.path.join(HERE, "mam4_oracle.c"), "-o", PORT_SO, "-lm"])
    if force or _stale(ULP_SO, deps):
        # same restatement with each libm result moved by one ulp (seeded):
        # measures the algorithm's own sensitivity to last-bit differences
        _run(["gcc", "-std=gnu99", "-DORACLE_ULP_NOISE"] + COMMON +
             [os.path.join(HERE, "mam4_oracle.c"), "-o", ULP_SO, "-lm"])
    if force or _stale(GPU_SO, deps + [os.path.join(HERE, "mam4_oracle_gpu.cu")]):
        # the same restatement as device code (CUDA libm, no FMA contraction)
        _run([os.environ.get("NVCC", "nvcc"), "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a",
              "-O3", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC", "-shared",
              os.path.join(HERE, "mam4_oracle_gpu.cu"), "-o", GPU_SO])
    if force or _stale(COUNT_SO, deps + [os.path.join(HERE, "opcount.cpp")]):
        # single-threaded: the tally is one global
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
              os.path.join(HERE, "opcount.cpp"), "-o", COUNT_SO, "-lm"])
    ref = ref or os.environ.get("MAM4XX_REFERENCE") or DEFAULT_REF
    src = os.path.join(ref, "src")
    if os.path.isdir(os.path.join(src, "mam4xx")):
        shim = os.path.join(HERE, "shim")
        rdeps = [os.path.join(HERE, "ref", "ref_step.cpp"), os.path.join(shim, "kokkos_ekat_shim.hpp")]
        if force or _stale(REF_SO, rdeps):
            os.makedirs(os.path.dirname(REF_SO), exist_ok=True)
            _run(["g++", "-std=c++17"] + COMMON + ["-I", shim, "-I", src,
                  os.path.join(HERE, "ref", "ref_step.cpp"), "-o", REF_SO])
        if force or _stale(REF_TUNED_SO, rdeps):
            _run(["g++", "-std=c++17"] + TUNED + ["-I", shim, "-I", src,
                  os.path.join(HERE, "ref", "ref_step.cpp"), "-o", REF_TUNED_SO])
        gdeps = [os.path.join(HERE, "ref", "ref_step_gpu.cu"),
                 os.path.join(shim, "kokkos_ekat_shim.hpp"), os.path.join(HERE, "oracle_api.h")]
        if force or _stale(REF_GPU_SO, gdeps):
            _run([os.environ.get("NVCC", "nvcc"), "-x", "cu",
                  "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                  "--fmad=false", "--expt-relaxed-constexpr", "-diag-suppress", "20012,20014",
                  "-Xcompiler", "-fPIC", "-shared", "-I", shim, "-I", src,
                  os.path.join(HERE, "ref", "ref_step_gpu.cu"), "-o", REF_GPU_SO])
    return PORT_SO


if __name__ == "__main__":
    build(force=True)
