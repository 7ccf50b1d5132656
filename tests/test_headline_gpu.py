"""Parity at the benchmark's own configuration: the config-1 generator (H40/C30/N10/O15/Cu5,
triclinic cell a=(58,0,0) b=(5,58,0) c=(3,4,58) A at 20,000 atoms) with the benchmark
cutoffs rc 95 / rc_CN 40 / rc_ATM 40 bohr, PBE-D3(BJ), through the C ABI.

* 2,000 atoms (same density, so the same per-apex list length): the whole evaluation
  against the FP64 oracle, 5- and 7-reference tables. FP64 form at its bar (energy 1e-9
  relative, forces 1e-7 eV/A, stress 1e-7 eV/A^3, CN 1e-12, dE/dCN 1e-9); precision form at
  its bar (energy 1e-6 relative, forces 1e-4 eV/A, stress 1e-6 eV/A^3).
* 20,000 atoms (the benchmark box itself): CN of every atom (1e-12) and, for a random
  sample of atoms, every pass's per-atom terms (two-body, ATM apex share, chain rule)
  against the oracle's per-atom export; FP64 within 1e-9 of each column's largest value,
  precision form within 1e-6 (two-body energy), 1e-5 (ATM apex energy) and 1e-4 (the
  derivative columns, which sum FP32 terms of both signs) of it; CN to 1e-4.
* Work counts (integers): the engine's counters of in-range CN pairs, two-body pairs and
  ATM triplets equal the oracle's exact counts of the reference enumeration (FP64 form;
  the FP32 range tests of the precision form may differ by pairs within rounding of a
  cutoff, at most 1e-6 of the count).
* The reference's cell-list regime (boxes thicker than 3 x 95 bohr): the engine against the
  FP64 oracle and against the reference build's own output (golden vectors, FP32 level).
"""
import os

import numpy as np
import pytest

import d3_systems as S
import oracle
from d3_b200 import D3, OPT_PRECISION, TABLE_5REF, TABLE_7REF

pytestmark = pytest.mark.gpu

RC, RCN, RATM = 95.0, 40.0, 40.0
HF = oracle.HARTREE_EV * oracle.ANG2BOHR  # hartree/bohr -> eV/A
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_outputs.npz")


def engine(sys_, precision, table=TABLE_5REF, rc=RC, rc_cn=RCN, rc_atm=RATM):
    d = D3(sys_["Z"], len(sys_["Z"]), rc=rc, rc_cn=rc_cn, rc_atm=rc_atm, damping=1, functional=0, table=table)
    d.set_option(OPT_PRECISION, precision)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    e, f, s = d.compute()
    cn, g, ea = d.atom_arrays()
    terms = d.pass_terms()
    _, cnt = d.pass_times()
    d.close()
    return dict(energy=e, forces=f, stress=s, cn=cn, dedcn=g, terms=terms, counters=[int(x) for x in cnt])


_CACHE = {}


def oracle_full(key, sys_, table):
    if key not in _CACHE:
        _CACHE[key] = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], rc=RC, rc_cn=RCN, rc_atm=RATM, damping=1,
                                     functional=0, extended=(table == TABLE_7REF), c6_mode=1)
    return _CACHE[key]


def oracle_counts(key, sys_):
    k = ("counts",) + key
    if k not in _CACHE:
        _CACHE[k] = oracle.counts(sys_["pos"], sys_["cell"], rc=RC, rc_cn=RCN, rc_atm=RATM)
    return _CACHE[k]


@pytest.fixture(scope="module")
def box2000():
    return S.triclinic_box(2000, seed=3)


@pytest.fixture(scope="module")
def box20000():
    return S.triclinic_box(20000, seed=1)  # the benchmark's box


@pytest.mark.parametrize("table", [TABLE_5REF, TABLE_7REF])
@pytest.mark.parametrize("precision", [0, 1])
def test_config1_density_2000_atoms_against_oracle(box2000, table, precision):
    r = oracle_full(("b2000", table), box2000, table)
    g = engine(box2000, precision, table)
    if precision == 0:
        assert abs(g["energy"] - r["energy"]) <= 1e-9 * abs(r["energy"]), (g["energy"], r["energy"])
        np.testing.assert_allclose(g["forces"], r["forces"], rtol=0, atol=1e-7)
        np.testing.assert_allclose(g["stress"], r["stress"], rtol=0, atol=1e-7)
        np.testing.assert_allclose(g["cn"], r["cn"], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(g["dedcn"], r["dedcn"], rtol=1e-9, atol=1e-15)
    else:
        assert abs(g["energy"] - r["energy"]) <= 1e-6 * abs(r["energy"]), (g["energy"], r["energy"])
        assert np.abs(g["forces"] - r["forces"]).max() <= 1e-4
        assert np.abs(g["stress"] - r["stress"]).max() <= 1e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_work_counters_equal_oracle_counts_2000(box2000, precision):
    want = oracle_counts(("b2000",), box2000)
    got = engine(box2000, precision)["counters"]
    have = (got[2], got[1], got[0] // 2)  # CN pairs, two-body pairs, ATM triplets
    if precision == 0:
        assert have == want, (have, want)
    else:
        for h, w in zip(have, want):
            assert abs(h - w) <= 1e-6 * w, (have, want)


# per-term bars relative to each column group's largest oracle value over the sample
GROUPS = [("two-body energy", slice(0, 1), 1e-9, 1e-6), ("two-body dE/dCN", slice(1, 2), 1e-9, 1e-4),
          ("two-body force", slice(2, 5), 1e-9, 1e-4), ("two-body virial", slice(5, 11), 1e-9, 1e-4),
          ("ATM apex energy", slice(11, 12), 1e-9, 1e-5), ("ATM apex dE/dCN", slice(12, 13), 1e-9, 1e-4),
          ("ATM apex force", slice(13, 16), 1e-9, 1e-4), ("ATM apex virial", slice(16, 22), 1e-9, 1e-4),
          ("chain-rule force", slice(22, 25), 1e-9, 1e-4), ("chain-rule virial", slice(25, 31), 1e-9, 1e-4)]


@pytest.fixture(scope="module")
def headline(box20000):
    # engine (both forms) and the oracle's per-atom terms of a random sample of atoms,
    # the chain-rule columns driven by the FP64 engine's complete dE/dCN (itself checked
    # at the sampled atoms through the two-body and ATM apex columns)
    fp64 = engine(box20000, 0)
    prec = engine(box20000, 1)
    sub = np.sort(np.random.default_rng(5).choice(len(box20000["Z"]), size=24, replace=False))
    t, cn = oracle.terms(box20000["pos"], box20000["Z"], box20000["cell"], sub, rc=RC, rc_cn=RCN, rc_atm=RATM,
                         dedcn=fp64["dedcn"])
    return fp64, prec, sub, t, cn


def test_config1_20000_cn_of_every_atom(headline):
    fp64, prec, _, _, cn = headline
    np.testing.assert_allclose(fp64["cn"], cn, rtol=1e-12, atol=1e-12)
    # FP32 CN terms (fast exponential) carry about 5e-5 relative error per atom
    np.testing.assert_allclose(prec["cn"], cn, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("precision", [0, 1])
def test_config1_20000_sampled_pass_terms(headline, precision):
    fp64, prec, sub, t, _ = headline
    got = (prec if precision else fp64)["terms"][sub]
    bad = []
    for name, cols, tol64, tol32 in GROUPS:
        scale = np.abs(t[:, cols]).max()
        err = np.abs(got[:, cols] - t[:, cols]).max()
        if not err <= (tol32 if precision else tol64) * scale + 1e-300:
            bad.append("%s: max error %.3e of scale %.3e" % (name, err, scale))
    assert not bad, bad


@pytest.mark.parametrize("precision", [0, 1])
def test_work_counters_equal_oracle_counts_20000(box20000, headline, precision):
    fp64, prec, *_ = headline
    want = oracle_counts(("b20000",), box20000)
    got = (prec if precision else fp64)["counters"]
    have = (got[2], got[1], got[0] // 2)
    if precision == 0:
        assert have == want, (have, want)
    else:
        for h, w in zip(have, want):
            assert abs(h - w) <= 1e-6 * w, (have, want)


def _golden(name):
    g = np.load(GOLDEN)
    if name + "/energy" not in g.files:
        pytest.fail("golden fixture %s missing: run tests/golden/make_golden.py on a GPU box" % name)
    return (float(g[name + "/energy"]), g[name + "/forces"], g[name + "/stress"], g[name + "/pos"].astype(np.float64),
            g[name + "/Z"], g[name + "/cell"].astype(np.float64))


@pytest.mark.parametrize("name", ["celllist_cubic", "celllist_sheared"])
def test_cell_list_regime(name):
    # the reference takes its cell-list path here (grid counts > 2 in every direction); the
    # engine returns every pair within the cutoffs, which the FP64 oracle's image box also
    # enumerates; the reference's 27-cell stencil misses 4 far two-body pairs of the
    # sheared box (tests/test_oracle_terms_cpu.py), too weak to show at FP32 level
    e_ref, f_ref, s_ref, pos, Z, cell = _golden(name)
    sys_ = {"pos": pos, "Z": Z, "cell": cell}
    assert oracle.cell_box(cell, RC, RCN)[0] == 1
    r = oracle.compute(pos, Z, cell, rc=RC, rc_cn=RCN, rc_atm=RATM, damping=1, functional=0)
    g = engine(sys_, 0)
    assert abs(g["energy"] - r["energy"]) <= 1e-9 * abs(r["energy"])
    np.testing.assert_allclose(g["forces"], r["forces"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(g["stress"], r["stress"], rtol=0, atol=1e-7)
    assert g["counters"][2] == oracle.counts(pos, cell, rc=RC, rc_cn=RCN, rc_atm=RATM)[0]
    # against the reference build itself (float, float atomics): FP32-level bars
    assert abs(g["energy"] - e_ref) <= 2e-5 * abs(e_ref), (g["energy"], e_ref)
    assert np.abs(g["forces"] - f_ref).max() <= 1e-4 * np.abs(g["forces"]).max() + 1e-7
    assert np.abs(g["stress"] - s_ref).max() <= 1e-4 * np.abs(g["stress"]).max() + 1e-9
