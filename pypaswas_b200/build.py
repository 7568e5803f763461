"""Builds libpaswas_b200.so in-tree with nvcc for sm_100a (B200), and the
CPython extension _hitbuild with gcc.

Usage: python -m pypaswas_b200.build [--force]
"""
import os
import subprocess
import sys

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PACKAGE_DIR)
CSRC = os.path.join(PACKAGE_DIR, "csrc")
SOURCES = [os.path.join(CSRC, "engine.cu"), os.path.join(CSRC, "noalloc.cu"), os.path.join(CSRC, "server.cpp"),
           os.path.join(CSRC, "format.cpp"), os.path.join(CSRC, "reader.cpp")]
DEPENDS = SOURCES + [os.path.join(CSRC, f) for f in ("pw_device.cuh", "pw_kernels.cuh", "pw_score16.cuh", "pw_band.cuh", "pw_band16.cuh", "pw_tiles.cuh", "pw_plan.h", "pw_finish.cuh", "pw_host.h", "server.cpp")] + [
    os.path.join(REPO_DIR, "include", "paswas_b200.h")]
LIBRARY = os.path.join(PACKAGE_DIR, "libpaswas_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared", "-lpthread", "-Xptxas", "-O3"]


HITBUILD_SRC = os.path.join(CSRC, "hitbuild.c")


def hitbuild_path():
    import sysconfig
    return os.path.join(PACKAGE_DIR, "_hitbuild" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_hitbuild(force=False):
    """Compiles the CPython extension that builds the driver's Hit objects
    (csrc/hitbuild.c) against this interpreter's headers."""
    import sysconfig
    out = hitbuild_path()
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(HITBUILD_SRC):
        return out
    cc = os.environ.get("CC", "gcc")
    tmp = out + ".tmp"
    subprocess.run([cc, "-O2", "-shared", "-fPIC", "-std=c11", "-Wall", "-I", sysconfig.get_paths()["include"],
                    "-o", tmp, HITBUILD_SRC], check=True)
    os.replace(tmp, out)
    return out


def up_to_date():
    if not os.path.exists(LIBRARY):
        return False
    t = os.path.getmtime(LIBRARY)
    return all(os.path.getmtime(p) <= t for p in DEPENDS if os.path.exists(p))


def build(force=False, verbose=False):
    """Compiles the engine and the Hit-building extension if any source
    changed; returns the engine library path."""
    build_hitbuild(force)
    if not force and up_to_date():
        return LIBRARY
    tmp = LIBRARY + ".tmp"
    cmd = [NVCC] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", tmp] + SOURCES
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
