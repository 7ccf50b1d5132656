"""Consumers of the path on the GPU: the command-line front end against the library, the
graph-replayed MD harness (random walk: last step against a direct evaluation; velocity
Verlet: total energy conserved, which needs forces = -dE/dx) and the ASE-style
calculator."""
import os
import subprocess

import numpy as np
import pytest

import d3_io
import d3_md
import d3_systems as S
from d3_b200 import D3, OPT_ATM_FORCE_SCALED, OPT_PRECISION

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
CLI = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "lasp-d3_b200", "lib", "d3_cli")


def direct(s, precision=0, rc=95.0, rc_atm=40.0, damping=1, scaled=False):
    d = D3(s["Z"], len(s["Z"]), rc=rc, rc_cn=40.0, rc_atm=rc_atm, damping=damping)
    d.set_option(OPT_PRECISION, precision)
    if scaled:
        d.set_option(OPT_ATM_FORCE_SCALED, 1)
    d.set_cell(s["cell"])
    d.set_atoms(s["pos"], s["Z"])
    out = d.compute()
    d.close()
    return out


def test_cli_matches_library(tmp_path):
    s = S.triclinic_box(300, seed=8)
    p = os.path.join(tmp_path, "s.arc")
    d3_io.write_arc(p, [s])
    s = d3_io.read_arc(p)[0]  # positions as written (9 decimals)
    out = subprocess.run([CLI, "--fp64", "--use-atm", "--damping", "bj", "--rc", "95", "--quiet", p],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    e_cli = float(out.stdout.split()[-1])
    e_lib = direct(s)[0]
    assert abs(e_cli - e_lib) <= 1e-10 * abs(e_lib)
    # the reference CLI's defaults: float ABI, zero damping, rc 60 bohr, no ATM
    out = subprocess.run([CLI, p], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    e_f = float([l for l in out.stdout.splitlines() if l.startswith("Energy:")][0].split()[1])
    e_ref = direct(s, rc=60.0, rc_atm=None, damping=0)[0]
    assert abs(e_f - e_ref) <= 1e-5 * abs(e_ref)


def test_graph_random_walk_last_step():
    s = S.triclinic_box(200, seed=3)
    md = d3_md.GraphMD(s, mode="random-walk", step=0.01, precision=True, max_steps=40)
    e, _, _ = md.run(25)
    assert np.all(np.isfinite(e)) and len(e) == 25
    fin = dict(s, pos=md.pos.cpu().numpy())
    e_direct = direct(fin, precision=1, scaled=True)[0]
    assert abs(e[-1] - e_direct) <= 1e-7 * abs(e_direct)
    assert abs(e[0] - e[-1]) > 0  # the structure moved
    md.close()


def test_graph_velocity_verlet_conserves_energy():
    s = S.triclinic_box(300, seed=12)
    md = d3_md.GraphMD(s, mode="nve", dt=0.5, precision=False, max_steps=400)
    rng = np.random.default_rng(0)
    m = np.array([d3_md.MASS[int(z)] for z in s["Z"]])
    kT = 8.617333e-5 * 300.0  # eV
    v = rng.normal(size=(len(m), 3)) * np.sqrt(kT / m / d3_md.KE_UNIT)[:, None]  # A/fs
    md.set_velocities(v)
    e, k, _ = md.run(300)
    tot = e + k
    span = np.ptp(e)
    assert span > 1e-4  # the potential energy did change along the trajectory
    assert np.abs(tot - tot[0]).max() <= 0.02 * span, (np.abs(tot - tot[0]).max(), span)
    md.close()


class FakeAtoms:
    def __init__(self, s):
        self.s = s

    def get_atomic_numbers(self):
        return np.asarray(self.s["Z"])

    def get_positions(self):
        return np.asarray(self.s["pos"])

    def get_cell(self):
        return np.asarray(self.s["cell"])


def test_ase_style_calculator():
    s = S.triclinic_box(150, seed=6)
    calc = d3_md.D3ASECalculator()
    calc.calculate(FakeAtoms(s))
    e, f, st = direct(s)
    assert abs(calc.results["energy"] - e) <= 1e-12 * abs(e)
    np.testing.assert_allclose(calc.results["forces"], f, rtol=0, atol=1e-12)
    np.testing.assert_allclose(calc.results["stress"], [st[0, 0], st[1, 1], st[2, 2], st[1, 2], st[0, 2], st[0, 1]],
                               rtol=0, atol=1e-14)
