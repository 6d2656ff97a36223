"""Builds the sm_100a shared library libfluide_b200.so in-tree.

Every .cu file under csrc/ is compiled with nvcc for sm_100a (`-gencode arch=compute_100a,code=sm_100a
-lineinfo -O3`) into csrc/../_build/, then linked into fluide_engine_b200/libfluide_b200.so together with
the static CUDA runtime.  The library is self-contained: the only runtime dependency is the driver.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libfluide_b200.so")
ROOT = os.path.dirname(PKG)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"  # the system compiler; never a wrapper that links libstdc++ statically
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX, "--expt-relaxed-constexpr"]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs + [os.path.join(ROOT, "include", "fluide_b200.h")]


def _stale(target, deps):
    return not os.path.exists(target) or os.path.getmtime(target) < max(os.path.getmtime(d) for d in deps)


def build(force=False, verbose=False):
    """Compiles and links the library when any source is newer than it; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    headers = _headers()
    objs = []

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        if force or _stale(obj, [src] + headers):
            cmd = [NVCC] + ARCH + FLAGS + ["-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stderr[-6000:]))
            if verbose:
                sys.stderr.write(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, srcs))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s" % r.stderr[-6000:])
    build_python_module(force=force)
    return LIB


def build_python_module(force=False):
    """Builds the PyFluidEngine pybind11 module (fluide_engine_b200/PyFluidEngine*.so) against the library."""
    import sysconfig

    try:
        import pybind11
    except ImportError:  # pybind11 is a build-time dependency of the Python module only
        return None
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = os.path.join(PKG, "PyFluidEngine" + suffix)
    src = os.path.join(CSRC, "python", "pyfluidengine.cpp")
    deps = [src, LIB, os.path.join(ROOT, "include", "fluide_engine.hpp"), os.path.join(ROOT, "include", "fluide_b200.h")]
    if not force and not _stale(out, deps):
        return out
    cmd = [HOST_CXX, "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"], "-I", os.path.join(ROOT, "include"),
           src, "-o", out, "-L", PKG, "-l:libfluide_b200.so", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("PyFluidEngine build failed:\n%s" % r.stderr[-6000:])
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
