"""Engine (FP64 path, through the C ABI) against the FP64 oracle.

Tolerances (the accuracy bar of the FP64 plain form): energy 1e-9 relative, forces
1e-7 eV/A, stress 1e-7 eV/A^3, on the same seeded inputs. Cases follow the reference's
own test systems (test/d3_test.cpp:343-417), the 96-atom water box and small
triclinic boxes of the benchmark generator, both damping types, both table layouts,
ATM on and off, and the option paths.
"""
import numpy as np
import pytest

import d3_systems as S
import oracle
from d3_b200 import D3, OPT_ATM_FORCE_SCALED, OPT_SMOOTH_CN, TABLE_7REF

pytestmark = pytest.mark.gpu

E_REL, F_ABS, S_ABS = 1e-9, 1e-7, 1e-7


def perturbed(sys_, amp=0.1, seed=0):
    rng = np.random.default_rng(seed)
    out = dict(sys_)
    out["pos"] = sys_["pos"] + rng.uniform(-amp, amp, sys_["pos"].shape)
    return out


def run_engine(sys_, rc, rc_cn, rc_atm, damping, functional, table=0, options=(), init_elements=None):
    d = D3(init_elements if init_elements is not None else sys_["Z"], len(sys_["Z"]), rc=rc, rc_cn=rc_cn,
           rc_atm=rc_atm, damping=damping, functional=functional, table=table)
    for opt, val in options:
        d.set_option(opt, val)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    e, f, s = d.compute()
    cn, g, ea = d.atom_arrays()
    d.close()
    return e, f, s, cn, g, ea


def check(sys_, rc=40.0, rc_cn=40.0, rc_atm=None, damping=1, functional=1, table=0, options=(), **okw):
    e, f, s, cn, g, ea = run_engine(sys_, rc, rc_cn, rc_atm, damping, functional, table, options)
    r = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], rc=rc, rc_cn=rc_cn, rc_atm=rc_atm, damping=damping,
                       functional=functional, extended=(table == TABLE_7REF), **okw)
    assert abs(e - r["energy"]) <= E_REL * abs(r["energy"]), (e, r["energy"])
    np.testing.assert_allclose(cn, r["cn"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(f, r["forces"], rtol=0, atol=F_ABS)
    np.testing.assert_allclose(s, r["stress"], rtol=0, atol=S_ABS)
    np.testing.assert_allclose(g, r["dedcn"], rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(ea, r["energy_atoms_hartree"], rtol=1e-9, atol=1e-15)
    return e, r


@pytest.mark.parametrize("damping", [0, 1])
@pytest.mark.parametrize("atm", [None, 40.0])
def test_small_system(damping, atm):
    check(S.gtest_small_system(), damping=damping, rc_atm=atm)


@pytest.mark.parametrize("damping", [0, 1])
@pytest.mark.parametrize("surface", [False, True])
def test_bcc_fe(damping, surface):
    # perturbed so that forces are not zero by symmetry; small cell: repeated-index ATM triplets
    check(perturbed(S.gtest_bcc_fe(surface)), rc=30.0, rc_cn=30.0, rc_atm=30.0, damping=damping)


def test_water_box_config0():
    # 96-atom water, PBE-D3(BJ), rc 95 / rc_CN 40 / rc_ATM 40 bohr, 13^3 image box
    check(S.water_box(0), rc=95.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)


@pytest.mark.parametrize("table", [0, 1])
def test_triclinic_box(table):
    sys_ = S.triclinic_box(n=300, seed=5)
    check(sys_, rc=60.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0, table=table)


def test_atm_force_scaled_option():
    sys_ = perturbed(S.gtest_bcc_fe(), seed=3)
    check(sys_, rc=30.0, rc_cn=30.0, rc_atm=30.0, options=((OPT_ATM_FORCE_SCALED, 1),), atm_force_scaled=True)


def test_smooth_cn_option():
    check(S.gtest_small_system(), rc_atm=40.0, options=((OPT_SMOOTH_CN, 1),), smooth_cn=True)


def test_unwrapped_input_box_semantics():
    # atoms outside the home cell: the reference enumerates images of the UNWRAPPED
    # positions inside its image box (src/d3_kernel.cu:632-667); the engine wraps for
    # its cell list but keeps the same (i, j, shift) set
    sys_ = S.triclinic_box(n=120, seed=9)
    rng = np.random.default_rng(1)
    shift = rng.integers(-2, 3, size=(120, 3))
    sys_["pos"] = sys_["pos"] + shift @ sys_["cell"]
    check(sys_, rc=40.0, rc_cn=40.0, rc_atm=40.0)


def test_atm_half_list_matches_reference_enumeration():
    # the set of (apex, j, lattice shift) entries equals the reference's enumeration:
    # j <= apex, every image in the box, 1e-12 <= r^2 <= rc_ATM^2
    sys_ = S.water_box(1)
    rc_atm = 40.0
    d = D3(sys_["Z"], len(sys_["Z"]), rc=95.0, rc_cn=40.0, rc_atm=rc_atm)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    d.compute()
    rows = d.atm_pairs()
    d.close()
    got = set(map(tuple, rows.tolist()))
    _, mcb, _ = oracle.cell_box(sys_["cell"], 95.0, 40.0)
    pos = sys_["pos"] * oracle.ANG2BOHR
    cell = sys_["cell"] * oracle.ANG2BOHR
    half = mcb // 2
    T = np.array([(x, y, z) for z in range(-half[2], half[2] + 1) for y in range(-half[1], half[1] + 1)
                  for x in range(-half[0], half[0] + 1)])
    shifts = T @ cell
    want = set()
    r2max = float(np.float32(rc_atm)) ** 2
    for a in range(len(pos)):
        for b in range(a + 1):
            d2 = ((pos[a] - (pos[b] + shifts)) ** 2).sum(1)
            ok = np.nonzero((d2 >= 1e-12) & (d2 <= r2max))[0]
            for k in ok:
                want.add((a, b, *T[k].tolist()))
    assert got == want


def test_custom_functional_params():
    sys_ = S.gtest_small_system()
    d = D3(sys_["Z"], len(sys_["Z"]), rc=40.0, rc_cn=40.0, damping=1, functional=99)
    d.set_functional_params(1.0, 0.7875, 0.4289, 4.4407)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    e, f, s = d.compute()
    d.close()
    r = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], rc=40.0, rc_cn=40.0, damping=1, functional=0)
    assert abs(e - r["energy"]) <= 1e-6 * abs(r["energy"])  # params given in double vs float-rounded table


def test_element_superset_at_init():
    # handle created with more elements than the frame uses (reference :389-422 would
    # re-map types; the engine keeps the init mapping)
    sys_ = S.gtest_small_system()
    init = [1, 6, 7, 8, 29]
    e, f, s, *_ = run_engine(sys_, 40.0, 40.0, 40.0, 1, 1, init_elements=init)
    r = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], rc=40.0, rc_cn=40.0, rc_atm=40.0, damping=1,
                       functional=1, init_elements=init)
    assert abs(e - r["energy"]) <= E_REL * abs(r["energy"])
    np.testing.assert_allclose(f, r["forces"], atol=F_ABS)
