"""Builds the in-tree CUDA library (libpdc.so, sm_100a) with nvcc.

The library is built in place under primal_dual_contacts_miror_b200/_lib so it
travels with the source tree; nothing is installed into site-packages.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libpdc.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]
SOURCES = ["pdc_api.cu"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    files = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h", ".hpp")):
                files.append(os.path.join(d, f))
    return files


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _deps())


def build(force=False, verbose=False, extra_flags=()):
    """Compile libpdc.so for sm_100a.  Returns the library path."""
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *NVCC_FLAGS, *extra_flags, "-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


HOST_SRC = os.path.join(PKG, "host", "force_solver_host.cpp")
HOST_BIN = os.path.join(LIBDIR, "force_solver_host")


def build_host(force=False):
    """Compile the C++ host program (the reference-side adapter over the C ABI),
    linked against the in-tree libpdc.so.  Returns the executable's path."""
    lib = build()
    if (not force and os.path.exists(HOST_BIN) and os.path.getmtime(HOST_BIN) > os.path.getmtime(HOST_SRC)
            and os.path.getmtime(HOST_BIN) > os.path.getmtime(lib)):
        return HOST_BIN
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), HOST_SRC, "-o", HOST_BIN + ".tmp",
           "-L", LIBDIR, "-lpdc", "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("g++ failed:\n" + res.stdout + res.stderr)
    os.replace(HOST_BIN + ".tmp", HOST_BIN)
    return HOST_BIN


def build_oracle():
    """Compile the CPU oracle used by the tests and the CPU baseline."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return os.path.join(ROOT, "oracle", "_build", "libpdc_oracle.so")


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
