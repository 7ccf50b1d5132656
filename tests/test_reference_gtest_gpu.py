"""The reference's own googletest suite (LASP-D3 test/d3_test.cpp: handle operations,
negative energy, run-to-run stability, force sum, stress symmetry, numerical forces,
supercell consistency, on its six test systems), compiled unmodified against its own
src/d3.h and linked against this repository's libd3.so (oracle/build_ref_gtest.py, with the
gtest-compatible header of tests/gtest_shim). Skipped where the binary was not built
(the reference sources are needed to build it)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle", "_ref", "d3_test_ref")


@pytest.mark.skipif(not os.path.exists(BIN), reason="reference test suite not built (needs the reference sources)")
def test_reference_suite_passes_against_libd3():
    out = subprocess.run([BIN], capture_output=True, text=True, timeout=900)
    tail = "\n".join(out.stdout.splitlines()[-5:])
    assert out.returncode == 0, tail + "\n" + out.stderr[-3000:]
    assert "Running 42 tests." in out.stdout
    assert "failed 0." in out.stdout
