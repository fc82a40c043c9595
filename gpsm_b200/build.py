"""Build libgpsm.so (the engine and its C ABI) and the gpsm_run CLI in-tree.

Every CUDA source is compiled for sm_100a only:
    nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3
The shared library is written next to this file so that it travels with the
source tree; nothing is installed into site-packages or a JIT cache.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgpsm.so")
CLI = os.path.join(HERE, "gpsm_run")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I" + INCLUDE, "-I" + CSRC, "-Xcompiler", "-fPIC,-Wall"]
CUFLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr"]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp") and f != "gpsm_run.cpp")
    host = os.path.join(CSRC, "host")
    if os.path.isdir(host):
        cpp += sorted(os.path.join("host", f) for f in os.listdir(host) if f.endswith(".cpp"))
    return cu, cpp


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose=False, force=False):
    """Compile every .cu/.cpp under csrc/ into libgpsm.so (and gpsm_run)."""
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = _sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    for d, _, fs in os.walk(INCLUDE):
        headers += [os.path.join(d, f) for f in fs]
    objs = []
    for f in cu + cpp:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f.replace(os.sep, "_") + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            flags = COMMON + (CUFLAGS if f.endswith(".cu") else ["-x", "c++"])
            _run([NVCC] + flags + ["-c", src, "-o", obj], verbose)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda", "-lpthread"], verbose)
    cli_src = os.path.join(CSRC, "gpsm_run.cpp")
    if os.path.exists(cli_src) and (force or _newer(CLI, [cli_src, LIB] + headers)):
        _run([NVCC] + COMMON + ["-x", "c++", cli_src, "-o", CLI, "-L" + HERE, "-lgpsm",
              "-Xlinker", "-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
