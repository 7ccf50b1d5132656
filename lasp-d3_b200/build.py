"""In-tree build of libd3.so (the drop-in C-ABI library) for sm_100a.

    python lasp-d3_b200/build.py [--verbose] [--ptxas]

Output: lasp-d3_b200/lib/libd3.so (git-ignored; it travels with the source tree).
The library is self-contained: CUDA runtime linked dynamically, no torch.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(OUT_DIR, "libd3.so")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["d3_engine.cu", "d3_noalloc.cu", "d3_mlp.cu"]
CXX_SOURCES = ["d3_geometry.cpp", "d3_api.cpp"]
HEADERS = ["d3_engine.h", "d3_pairs.cuh", "d3_geometry.h", "d3_synth_params.h", "d3_mlp.h", "d3_atm.cuh", "d3_atm32.cuh", "d3_atm32b.cuh",
           "d3_surrogate.cuh"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in CU_SOURCES + CXX_SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "d3.h"))
    deps.append(os.path.join(HERE, "cli", "d3_cli.cpp"))
    if not os.path.exists(os.path.join(OUT_DIR, "d3_cli")):
        return True
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, ptxas=False, force=False):
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    objs = []
    log = ""
    for s in CU_SOURCES:
        o = os.path.join(obj_dir, s + ".o")
        cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr"] + ARCH
        if ptxas:
            cmd += ["-Xptxas", "-v"]
        cmd += ["-c", os.path.join(CSRC, s), "-o", o]
        log += _run(cmd, verbose)
        objs.append(o)
    for s in CXX_SOURCES:
        o = os.path.join(obj_dir, s + ".o")
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-I/usr/local/cuda/include", "-c",
               os.path.join(CSRC, s), "-o", o]
        _run(cmd, verbose)
        objs.append(o)
    tmp = LIB + ".tmp"
    _run([NVCC, "-shared"] + ARCH + objs + ["-o", tmp, "-lcudart"], verbose)
    os.replace(tmp, LIB)
    # command-line front end on the library (drop-in for the reference's d3_cpp)
    cli = os.path.join(OUT_DIR, "d3_cli")
    _run(["g++", "-std=c++17", "-O2", "-I", os.path.join(HERE, "..", "include"), os.path.join(HERE, "cli", "d3_cli.cpp"),
          "-L", OUT_DIR, "-ld3", "-Wl,-rpath,$ORIGIN", "-o", cli + ".tmp"], verbose)
    os.replace(cli + ".tmp", cli)
    if ptxas:
        print(log)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, ptxas="--ptxas" in sys.argv, force=True))
