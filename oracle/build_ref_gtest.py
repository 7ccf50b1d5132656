"""Build recipe: the reference's own googletest suite (test/d3_test.cpp of LASP-D3),
compiled unmodified where it lies (it includes the reference's own src/d3.h) against this
repository's libd3.so, with the gtest-compatible header of tests/gtest_shim.

TEST INFRASTRUCTURE: the output oracle/_ref/d3_test_ref is run by
tests/test_reference_gtest_gpu.py as evidence that the library is a drop-in for the
reference's C API. Needs the reference tree (this machine only); the binary travels with
the repository snapshot (oracle/_ref is git-ignored, not snapshot-ignored).

    python oracle/build_ref_gtest.py
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# the reference tree: $LASP_D3_REFERENCE (default: the path the build container mounts)
REF = os.environ.get("LASP_D3_REFERENCE", "/root/reference")
OUT = os.path.join(HERE, "_ref", "d3_test_ref")


def build(verbose=False):
    src = os.path.join(REF, "test", "d3_test.cpp")
    if not os.path.exists(src):
        return None
    lib = os.path.join(ROOT, "lasp-d3_b200", "lib")
    if not os.path.exists(os.path.join(lib, "libd3.so")):
        raise RuntimeError("build libd3.so first (python lasp-d3_b200/build.py)")
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    shim = os.path.join(ROOT, "tests", "gtest_shim")
    cmd = ["g++", "-std=c++17", "-O1", "-w", "-I", shim, src, os.path.join(shim, "gtest_main.cc"), "-L", lib, "-ld3",
           "-Wl,-rpath,$ORIGIN/../../lasp-d3_b200/lib", "-o", OUT]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
