"""Structure files and the command-line front end, host side: .arc / extxyz readers
against generated files, the cell-from-parameters convention, and d3_cli's --help and
--parse-only (no GPU)."""
import os
import subprocess

import numpy as np

import d3_io
import d3_systems as S

HERE = os.path.dirname(os.path.abspath(__file__))
CLI = os.path.join(HERE, "..", "lasp-d3_b200", "lib", "d3_cli")


def test_cell_from_parameters_round_trip():
    h = np.array([[10.0, 0, 0], [2.0, 9.0, 0], [1.5, -0.7, 8.0]])
    a, b, c = (np.linalg.norm(h[i]) for i in range(3))
    ang = lambda u, v: np.degrees(np.arccos(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v)))
    g = d3_io.cell_from_parameters(a, b, c, ang(h[1], h[2]), ang(h[0], h[2]), ang(h[0], h[1]))
    np.testing.assert_allclose(g, h, atol=1e-12)


def test_arc_round_trip(tmp_path):
    s1 = S.triclinic_box(120, seed=2)
    s2 = S.water_box(0)
    p = os.path.join(tmp_path, "x.arc")
    d3_io.write_arc(p, [s1, s2])
    r = d3_io.read_arc(p)
    assert len(r) == 2
    for a, b in zip(r, (s1, s2)):
        np.testing.assert_array_equal(a["Z"], b["Z"])
        np.testing.assert_allclose(a["cell"], b["cell"], atol=2e-8)
        np.testing.assert_allclose(a["pos"], b["pos"], atol=2e-8)


def test_extxyz_reader(tmp_path):
    s = S.triclinic_box(50, seed=4)
    p = os.path.join(tmp_path, "x.extxyz")
    with open(p, "w") as f:
        for k in range(2):
            f.write("%d\n" % len(s["Z"]))
            f.write('Lattice="%s" Properties=species:S:1:pos:R:3 energy=%d pbc="T T T"\n'
                    % (" ".join("%.9f" % v for v in np.asarray(s["cell"]).ravel()), k))
            for z, r in zip(s["Z"], s["pos"]):
                f.write("%s %.9f %.9f %.9f\n" % (d3_io.SYMBOLS[z - 1], *r))
    r = d3_io.read_structures(p)
    assert len(r) == 2 and r[1]["energy"] == 1.0
    np.testing.assert_array_equal(r[0]["Z"], s["Z"])
    np.testing.assert_allclose(r[0]["pos"], s["pos"], atol=1e-8)
    np.testing.assert_allclose(r[0]["cell"], s["cell"], atol=1e-8)


def test_cli_help_and_parse_only(tmp_path):
    assert subprocess.run([CLI, "--help"], capture_output=True).returncode == 0
    assert subprocess.run([CLI], capture_output=True).returncode != 0
    s = S.triclinic_box(77, seed=5)
    p = os.path.join(tmp_path, "y.arc")
    d3_io.write_arc(p, [s, s])
    out = subprocess.run([CLI, "--parse-only", p], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.count("Atoms: 77") == 2
    vals = [float(l.split(": ")[1]) for l in out.stdout.splitlines() if l.startswith("Cell[")][:9]
    np.testing.assert_allclose(np.reshape(vals, (3, 3)), s["cell"], atol=1e-7)
    bad = subprocess.run([CLI, "--damping", "nope", p], capture_output=True)
    assert bad.returncode != 0
