"""Build recipe for oracle/_ref/ -- TEST INFRASTRUCTURE ONLY.

Compiles the reference's own CPU simulator (AleksanderSiwek/Fluide_Engine, src/) from the sources
where they lie (the reference checkout's src/ named by FE_REFERENCE_SRC, else /root/reference/src when that
exists), together with oracle/ref_harness.cpp, into two shared
libraries under oracle/_ref/ (git-ignored):

* libfe_ref_serial.so   -- parallel_utils loops run on the calling thread (use_threads=false).  The
                           threaded P2G of the reference is a data race (pic_simulator.cpp:384-412),
                           so this deterministic build is the one that pins the C restatement.
* libfe_ref_threaded.so -- the loops as written (one std::thread per hardware thread); this is the
                           timed CPU baseline.

The reference does not compile with g++ as written (it targets MSVC).  Five mechanical adjustments
are applied without touching the reference tree:
  1. two headers (common/parallel_utils.hpp, common/array3.hpp) bind rvalue lambdas to non-const
     references; sed-patched copies that take forwarding references are generated into
     oracle/_ref/gen/ and force-included (-include) ahead of everything, so their include guards turn
     the originals into no-ops;
  2./3. extra member qualifications (grid_systems/face_centered_grid3d.hpp:30,
     emmiter/volume_emmiter.hpp:22) are accepted with -fpermissive;
  4. <concurrent_vector.h> (MSVC PPL) resolves to oracle/shim/concurrent_vector.h;
  5. TriangleMesh::IsInside (3d/triangle_mesh.cpp:151) calls an unqualified abs on a double, which MSVC
     resolves to abs(double) but g++ to the C library's int abs(int) (truncating the winding sum, so no
     point would ever be inside); a force-included header brings std::abs into the global namespace, giving
     the MSVC meaning.  It is the reference's only unqualified abs.
The generated headers are build intermediates and are deleted after the build.
"""
import os
import re
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
def _reference_src():
    """Reference source tree: $FE_REFERENCE_SRC, else the read-only checkout at /root/reference/src (None if neither)."""
    env = os.environ.get("FE_REFERENCE_SRC")
    if env:
        return env
    default = "/root/reference/src"
    return default if os.path.isdir(default) else None


REF = _reference_src()
OUT = os.path.join(HERE, "_ref")
CXX = os.environ.get("FE_REF_CXX", "g++")  # the system g++; a $CXX that links libstdc++ statically breaks loading next to numpy
FLAGS = ["-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-fpermissive", "-w", "-pthread"]


def _sources():
    srcs = []
    for root, _dirs, files in os.walk(REF):
        if "python_wrapper" in root:
            continue
        for f in files:
            if f.endswith(".cpp") and f != "main.cpp":
                srcs.append(os.path.join(root, f))
    return sorted(srcs)


def _gen_headers(gen_dir, threaded):
    os.makedirs(gen_dir, exist_ok=True)
    common = os.path.join(REF, "common")
    with open(os.path.join(common, "parallel_utils.hpp")) as f:
        pu = f.read()
    pu = pu.replace("static void ForEach(size_t size, Callback& functor)", "static void ForEach(size_t size, Callback&& functor)")
    pu = pu.replace("static void ForEach3(size_t sizeX, size_t sizeY, size_t sizeZ, Callback& functor)",
                    "static void ForEach3(size_t sizeX, size_t sizeY, size_t sizeZ, Callback&& functor)")
    if not threaded:
        pu = re.sub(r"bool use_threads = true", "bool use_threads = false", pu)
    with open(os.path.join(gen_dir, "parallel_utils.hpp"), "w") as f:
        f.write(pu)
    with open(os.path.join(common, "array3.hpp")) as f:
        a3 = f.read()
    a3 = a3.replace("void ForEachIndex(Callback& functor)", "void ForEachIndex(Callback&& functor)")
    a3 = a3.replace("void ParallelForEachIndex(Callback& functor)", "void ParallelForEachIndex(Callback&& functor)")
    a3 = a3.replace('#include "vector3.hpp"', '#include "%s"' % os.path.join(common, "vector3.hpp"))
    a3 = a3.replace('#include "parallel_utils.hpp"', '#include "%s"' % os.path.join(gen_dir, "parallel_utils.hpp"))
    with open(os.path.join(gen_dir, "array3.hpp"), "w") as f:
        f.write(a3)
    with open(os.path.join(gen_dir, "msvc_abs.hpp"), "w") as f:
        f.write("#include <cmath>\n#include <cstdlib>\nusing std::abs;\n")


def _build_variant(name, threaded):
    gen = os.path.join(OUT, "gen_" + name)
    objdir = os.path.join(OUT, "obj_" + name)
    os.makedirs(objdir, exist_ok=True)
    _gen_headers(gen, threaded)
    inc = ["-I", os.path.join(HERE, "shim"), "-I", REF, "-I", "/usr/local/cuda/include",
           "-include", os.path.join(gen, "parallel_utils.hpp"), "-include", os.path.join(gen, "array3.hpp"),
           "-include", os.path.join(gen, "msvc_abs.hpp")]
    srcs = _sources() + [os.path.join(HERE, "ref_harness.cpp")]

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(os.path.dirname(src)) + "_" + os.path.basename(src) + ".o")
        cmd = [CXX] + FLAGS + inc + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed: %s\n%s" % (src, r.stderr[-4000:]))
        return obj

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(compile_one, srcs))
    lib = os.path.join(OUT, "libfe_ref_%s.so" % name)
    r = subprocess.run([CXX, "-shared", "-pthread", "-o", lib] + objs, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed: %s" % r.stderr[-4000:])
    for d in (gen, objdir):
        for f in os.listdir(d):
            os.remove(os.path.join(d, f))
        os.rmdir(d)
    return lib


def build(force=False):
    """Builds both variants when the reference sources are present; returns the list of built libraries."""
    if not REF or not os.path.isdir(REF):
        return []
    os.makedirs(OUT, exist_ok=True)
    built = []
    for name, threaded in (("serial", False), ("threaded", True)):
        lib = os.path.join(OUT, "libfe_ref_%s.so" % name)
        deps = _sources() + [os.path.join(HERE, "ref_harness.cpp"), __file__]
        if not force and os.path.exists(lib) and os.path.getmtime(lib) >= max(os.path.getmtime(d) for d in deps):
            built.append(lib)
            continue
        built.append(_build_variant(name, threaded))
    return built


if __name__ == "__main__":
    print("\n".join(build(force="--force" in sys.argv)))
