"""Build recipe for the reference's own CUDA library, used as a checker and as the
reference arm of bench.py. Test infrastructure: nothing in the product links it.

The reference (LASP-D3) ships only CUDA sources; its CMake build needs Fortran and a
network fetch of googletest, so this recipe drives nvcc directly on the three
translation units, with the flags of the reference's CMakeLists.txt:35-41
(-O2 -lineinfo --maxrregcount=64, separable compilation), for sm_100a.

The reference's parameter headers are missing from its tree; the stand-in headers in
ref_build/{original,extended}/ declare the tables and ref_tables.cpp fills them from
the same seeded generator the engine uses.

Outputs (git-ignored, travel to the GPU box with the snapshot):
    oracle/_ref/libd3_ref.so       5-reference table (95 elements)
    oracle/_ref/libd3_ref_ext.so   7-reference table (103 elements, USE_EXTENDED_PARAMETERS)
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference tree: $LASP_D3_REFERENCE (default: the path the build container mounts)
REF_SRC = os.path.join(os.environ.get("LASP_D3_REFERENCE", "/root/reference"), "src")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
REF_FLAGS = ["-std=c++17", "-O2", "-lineinfo", "--maxrregcount=64", "-rdc=true", "-Xcompiler", "-fPIC"]
UNITS = ["d3.cu", "d3_buffer.cu", "d3_kernel.cu"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_variant(extended: bool, verbose=False):
    name = "libd3_ref_ext.so" if extended else "libd3_ref.so"
    target = os.path.join(OUT, name)
    tag = "ext" if extended else "orig"
    inc = os.path.join(HERE, "ref_build", "extended" if extended else "original")
    defs = ["-DUSE_EXTENDED_PARAMETERS"] if extended else []
    srcs = [os.path.join(REF_SRC, u) for u in UNITS]
    deps = srcs + [os.path.join(HERE, "ref_build", "ref_tables.cpp"), os.path.join(inc, os.listdir(inc)[0]),
                   os.path.join(HERE, "..", "lasp-d3_b200", "csrc", "d3_synth_params.h")]
    if not _stale(target, deps):
        return target
    objdir = os.path.join(OUT, "obj_" + tag)
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        _run([NVCC] + REF_FLAGS + ARCH + defs + ["-I", inc, "-I", REF_SRC, "-c", s, "-o", o])
        objs.append(o)
    o = os.path.join(objdir, "ref_tables.o")
    _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off"] + defs +
         ["-c", os.path.join(HERE, "ref_build", "ref_tables.cpp"), "-o", o])
    objs.append(o)
    _run([NVCC, "-shared", "-rdc=true"] + ARCH + objs + ["-o", target, "-lcudart"])
    if verbose:
        print("built", target)
    return target


def build(verbose=False):
    """Build both reference variants when the reference sources are present."""
    if not os.path.isdir(REF_SRC):
        return []
    os.makedirs(OUT, exist_ok=True)
    return [build_variant(False, verbose), build_variant(True, verbose)]


if __name__ == "__main__":
    print(build(verbose=True))
    sys.exit(0)
