"""Build recipe of the C++ process test harness (test infrastructure only).

  tests/cpp/_build/libmam4b_process_check.so
      g++, tests/cpp/microphysics_process_check.cpp: the product header
      include/mam4b_microphysics.hpp over the mam4xx reference containers
      (headers included read-only from <ref>/src and <ref>/src/validation,
      compiled against the host shim in oracle/shim), linked with
      mam4xx_b200/libmam4b.so and the CUDA runtime. Built only where the
      mam4xx tree exists; the tree is taken from build(ref=...), else from
      MAM4XX_REFERENCE, else from the default checkout location.

Usage: python tests/cpp/build_process_check.py
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "libmam4b_process_check.so")
SRC = os.path.join(HERE, "microphysics_process_check.cpp")
DEFAULT_REF = "/root/reference"  # default checkout of the mam4xx tree
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(ref=None, force=False):
    ref = ref or os.environ.get("MAM4XX_REFERENCE") or DEFAULT_REF
    src = os.path.join(ref, "src")
    if not os.path.isdir(os.path.join(src, "mam4xx")):
        return None
    deps = [SRC, os.path.join(ROOT, "include", "mam4b_microphysics.hpp"),
            os.path.join(ROOT, "include", "mam4b.h"),
            os.path.join(ROOT, "oracle", "shim", "kokkos_ekat_shim.hpp")]
    if not force and os.path.exists(OUT) and all(
            os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    pkg = os.path.join(ROOT, "mam4xx_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "oracle", "shim"), "-I", src,
           "-I", os.path.join(src, "validation"), "-I", os.path.join(CUDA, "include"),
           SRC, "-o", OUT, "-L", pkg, "-l:libmam4b.so",
           "-Wl,-rpath,$ORIGIN/../../../mam4xx_b200",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    sys.exit(0 if build(force=True) else 1)
