"""Build recipe for the in-tree sm_100a library (libprism_b200.so) and CLI.

nvcc cross-compiles for sm_100a without a GPU, so this runs anywhere the
CUDA 12.9 toolkit is installed.  Outputs land next to this file and travel
with the repository snapshot.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libprism_b200.so")
CLI = os.path.join(HERE, "bin", "prism")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]

LIB_SOURCES = [os.path.join(HERE, "csrc", "prism_b200.cu")]
LIB_DEPS = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))] + [
    os.path.join(ROOT, "include", "prism_b200.h")]
# the C++ interface (prism::Compressor, Buffer, prism_context, initialize)
HOST_SOURCES = [os.path.join(HERE, "host", f) for f in ("parameters.cpp", "io.cpp", "compressor.cpp", "prism.cpp")]
CLI_SOURCES = [os.path.join(HERE, "host", "prism_cli.cpp")] + HOST_SOURCES
# the reference's own driver compiled unchanged against the C++ interface
REF_EXAMPLE = os.path.join(HERE, "bin", "prism_ref_example")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build_lib(force=False, verbose=False):
    if not force and not _stale(LIB, LIB_DEPS):
        return LIB
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-shared"] + LIB_SOURCES + ["-o", LIB]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


def build_cli(force=False, verbose=False):
    srcs = [s for s in CLI_SOURCES if os.path.exists(s)]
    if len(srcs) != len(CLI_SOURCES):
        return None
    build_lib(force=force, verbose=verbose)
    hdrs = [os.path.join(HERE, "host", f) for f in os.listdir(os.path.join(HERE, "host"))]
    if not force and not _stale(CLI, srcs + hdrs + [LIB]):
        return CLI
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    cmd = _host_cmd(srcs, CLI)
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return CLI


def _host_cmd(srcs, out):
    return ["g++", "-O2", "-std=c++17", "-I" + os.path.join(HERE, "host"), "-I" + os.path.join(ROOT, "include"),
            "-I/usr/local/cuda/include"] + srcs + ["-L" + HERE, "-lprism_b200", "-Wl,-rpath,$ORIGIN/..",
                                                   "-L/usr/local/cuda/lib64", "-lcudart", "-o", out]


def build_ref_example(ref_dir, force=False, verbose=False):
    """Compile the reference's examples/prism.cpp, unmodified, against this
    library's C++ headers (prism.hpp, compressor.hpp) and link it with the
    library: the check that a reference caller recompiles unchanged.  Needs
    the reference source tree; the binary lands in bin/ and travels with the
    built library."""
    src = os.path.join(ref_dir, "examples", "prism.cpp")
    if not os.path.exists(src):
        return None
    build_lib(force=force, verbose=verbose)
    hdrs = [os.path.join(HERE, "host", f) for f in os.listdir(os.path.join(HERE, "host"))]
    if not force and not _stale(REF_EXAMPLE, [src] + HOST_SOURCES + hdrs + [LIB]):
        return REF_EXAMPLE
    os.makedirs(os.path.dirname(REF_EXAMPLE), exist_ok=True)
    cmd = _host_cmd([src] + HOST_SOURCES, REF_EXAMPLE)
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return REF_EXAMPLE


if __name__ == "__main__":
    build_lib(force=True, verbose=True)
    build_cli(force=True, verbose=True)
