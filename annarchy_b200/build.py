"""In-tree build of the native parts.

* ``_lib/libannarchy_b200.so``: the C ABI runtime (csrc/runtime.cu), built by
  nvcc for sm_100a; it links the CUDA runtime statically and NVRTC
  dynamically, and fetches the few driver-API entry points it needs at run
  time, so it loads on machines without a GPU driver.
* ``_lib/device_check.o``: the device header compiled with nvcc for sm_100a
  through a sample instantiation of every template (a build-time check and
  the source of the ``-Xptxas -v`` register report).

The per-network kernels are generated and compiled by NVRTC at
``Network.compile()``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_lib")
CSRC = os.path.join(HERE, "csrc")
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _sources(*rel):
    return [os.path.join(CSRC, r) for r in rel]


def build_runtime(force=False, verbose=False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    out = os.path.join(LIB_DIR, "libannarchy_b200.so")
    srcs = _sources("runtime.cu", "selector.cu", "bsr_tc.cu", "connect.cuh",
                    "device/anb_device.cuh") + [
        os.path.join(os.path.dirname(HERE), "include", "annarchy_b200.h")]
    srcs = [s for s in srcs if os.path.exists(s)]
    if force or _newer(out, srcs):
        cu = [s for s in srcs if s.endswith(".cu")]
        log = _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xptxas", "-v", "-shared",
                    "-Xcompiler", "-fPIC", "-I", CSRC, "-o", out, *cu, "-lnvrtc"], verbose)
        with open(os.path.join(LIB_DIR, "runtime.ptxas.txt"), "w") as f:
            f.write(log)
    return out


def build_device_check(force=False, verbose=False) -> str:
    out = os.path.join(LIB_DIR, "device_check.o")
    srcs = _sources("device/anb_device.cuh", "device/device_check.cu")
    if force or _newer(out, srcs):
        log = _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xptxas", "-v", "-c", "-o", out,
                    os.path.join(CSRC, "device", "device_check.cu")], verbose)
        with open(os.path.join(LIB_DIR, "device_check.ptxas.txt"), "w") as f:
            f.write(log)
    return out


def build_all(force=False, verbose=False):
    build_runtime(force, verbose)
    build_device_check(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
