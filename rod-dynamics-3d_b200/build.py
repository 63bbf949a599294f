"""Builds librodgpu.so (the CUDA hot path + C ABI) in-tree for sm_100a.

Usage: python rod-dynamics-3d_b200/build.py [--force]
The library is written next to this file so it travels with the repository.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librodgpu.so")
HOSTLIB = os.path.join(HERE, "librodhost.so")
HOST_SRCS = [os.path.join(HERE, "host", "scene_gen.cpp"), os.path.join(HERE, "host", "config_default.cpp")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# -fmad=false: no contraction of a*b+c into FMA, so every FP64 expression
# rounds as written (bit-exact contact predicate against the FP64 oracle).
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-fmad=false", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-shared",
         "-Xcompiler", "-fvisibility=default"]


# host C++ compiled into librodgpu.so beside the CUDA sources (the config
# defaults, shared with the reference-baseline harness)
LIB_HOST_SRCS = [os.path.join(HERE, "host", "config_default.cpp")]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu")) + LIB_HOST_SRCS


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "rodgpu.h"))
    return hs


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in sources() + headers() + [__file__])


def build_host(force=False, verbose=False):
    """Host C++ helpers (scene generator, mass properties)."""
    if (not force and os.path.exists(HOSTLIB)
            and all(os.path.getmtime(p) <= os.path.getmtime(HOSTLIB) for p in HOST_SRCS)):
        return HOSTLIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", HOSTLIB] + HOST_SRCS
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("g++ failed building librodhost.so")
    return HOSTLIB


def module_path():
    import sysconfig
    return os.path.join(HERE, "rod_dynamics_py" + sysconfig.get_config_var("EXT_SUFFIX"))


MODULE_SRCS = [os.path.join(HERE, "host", f) for f in ("rod_dynamics_py.cpp", "simulator.cpp", "scene_gen.cpp")]
MODULE_HDRS = [os.path.join(HERE, "host", f) for f in ("simulator.hpp", "json_min.hpp")]


def build_module(force=False, verbose=False):
    """The Python module rod_dynamics_py (pybind11; C++ host code over the C
    ABI of librodgpu.so).  Skipped when pybind11 is not importable."""
    import sysconfig
    try:
        import pybind11
    except ImportError:
        return None
    out = module_path()
    deps = MODULE_SRCS + MODULE_HDRS + [LIB, os.path.join(HERE, "..", "include", "rodgpu.h")]
    if not force and os.path.exists(out) and all(os.path.getmtime(p) <= os.path.getmtime(out) for p in deps):
        return out
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden",
           "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
           "-o", out] + MODULE_SRCS + ["-L", HERE, "-lrodgpu", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("g++ failed building rod_dynamics_py")
    return out


def build(force=False, verbose=False):
    build_host(force, verbose)
    if not force and up_to_date():
        build_module(False, verbose)
        return LIB
    cmd = [NVCC] + FLAGS + ["-o", LIB] + sources() + ["-lcudart"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building librodgpu.so")
    build_module(True, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
