"""Build the engine library ``libdtb_b200.so`` in-tree with nvcc for sm_100a.

Usage: ``python digital_twin_brain-open_b200/build.py [--force]``.  Rebuilds only
when a source is newer than the library.  ``--fmad=false`` keeps every float
operation separately rounded, which the bit-exact parity with the CPU oracle
relies on (the kernels also use explicitly rounded intrinsics).
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libdtb_b200.so")
SOURCES = ["dtb_engine.cu", "dtb_kernels.cu", "dtb_generate.cu", "dtb_host.cu", "dtb_compact.cu", "dtb_compact_noalloc.cu", "dtb_batch.cu", "dtb_serve.cu", "dtb_bold.cu", "dtb_da.cu"]
HEADERS = ["dtb_device.cuh", "dtb_kernels.h", "dtb_engine.h", "dtb_host.h", "dtb_compact.h", "dtb_batch.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "dtb_b200.h")]
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    srcs = [os.path.join(CSRC, f) for f in SOURCES if os.path.exists(os.path.join(CSRC, f))]
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "--fmad=false", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC,-O3", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           "-o", LIB + ".tmp", *srcs, "-lz"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
