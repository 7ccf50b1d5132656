"""The oracle's per-atom term export and exact work counts (used by the large-box parity
tests), and the restatement of the reference's cell-list pair enumeration, checked on the
CPU against the oracle's full evaluation and against direct enumerations."""
import numpy as np
import pytest

import d3_systems as S
import oracle

RC, RCN, RATM = 30.0, 20.0, 20.0


@pytest.fixture(scope="module")
def box():
    return S.triclinic_box(150, seed=13)


def test_terms_sum_to_the_full_evaluation(box):
    full = oracle.compute(box["pos"], box["Z"], box["cell"], rc=RC, rc_cn=RCN, rc_atm=RATM, c6_mode=1, raw=True)
    n = len(box["Z"])
    t, cn = oracle.terms(box["pos"], box["Z"], box["cell"], np.arange(n), rc=RC, rc_cn=RCN, rc_atm=RATM,
                         dedcn=full["dedcn"])
    np.testing.assert_allclose(cn, full["cn"], rtol=0, atol=0)
    e = t[:, 0].sum() + 3.0 * t[:, 11].sum()
    assert abs(e - full["energy_hartree"]) <= 1e-12 * abs(full["energy_hartree"])
    v6 = (t[:, 5:11] + t[:, 16:22] + t[:, 25:31]).sum(0)
    V = full["virial_raw"].reshape(3, 3)
    want = np.array([V[0, 0], V[1, 1], V[2, 2], V[0, 1], V[0, 2], V[1, 2]])
    np.testing.assert_allclose(v6, want, rtol=1e-10, atol=1e-14)
    # a subset gives the same rows as the whole set
    sub = np.array([3, 77, 149])
    ts, _ = oracle.terms(box["pos"], box["Z"], box["cell"], sub, rc=RC, rc_cn=RCN, rc_atm=RATM, dedcn=full["dedcn"])
    np.testing.assert_array_equal(ts, t[sub])


def test_counts_match_direct_enumeration(box):
    _, mcb, _ = oracle.cell_box(box["cell"], RC, RCN)
    reach = mcb // 2
    rc2, rcn2, ra2 = (float(np.float32(x)) ** 2 for x in (RC, RCN, RATM))
    ncn, n2, n3 = oracle.counts(box["pos"], box["cell"], rc=RC, rc_cn=RCN, rc_atm=RATM)
    assert ncn == len(oracle.all_pairs(box["cell"], box["pos"], rcn2, True, reach, float_input=False))
    assert n2 == len(oracle.all_pairs(box["cell"], box["pos"], rc2, False, reach, float_input=False))
    # ATM: per apex a, unordered pairs of distinct half-list entries (b <= a, in range of a)
    # within rc_ATM of each other
    cell = np.asarray(box["cell"], np.float64) * oracle.ANG2BOHR
    pos = np.asarray(box["pos"], np.float64) * oracle.ANG2BOHR
    T = np.array([(x, y, z) for z in range(-reach[2], reach[2] + 1) for y in range(-reach[1], reach[1] + 1)
                  for x in range(-reach[0], reach[0] + 1)])
    img = (pos[None, :, :] + (T @ cell)[:, None, :])  # [T][j][3]
    want = 0
    for a in range(len(pos)):
        v = img[:, : a + 1].reshape(-1, 3)
        d2 = ((pos[a] - v) ** 2).sum(1)
        L = v[(d2 >= 1e-12) & (d2 <= ra2)]
        dd = ((L[:, None, :] - L[None, :, :]) ** 2).sum(-1)
        ok = (dd >= 1e-12) & (dd <= ra2)
        want += int(np.triu(ok, 1).sum())
    assert n3 == want


def test_cell_list_pairs_complete_for_a_cubic_box_and_not_for_a_sheared_one():
    # cubic: the reference's 27-cell stencil finds every pair; sheared: its grid counts
    # come from the rows of the cell inverse (not the reciprocal vectors), so along x its
    # grid cells are thinner than the cutoff and a few pairs are missed
    rc2 = float(np.float32(95.0)) ** 2
    cubic = S.cell_list_box(400, seed=31, edge=160.0)
    assert oracle.cell_list_pairs(cubic["cell"], cubic["pos"], 95.0, 40.0, rc2, False) == \
        oracle.all_pairs(cubic["cell"], cubic["pos"], rc2, False, 1)
    sheared = S.cell_list_box(500, seed=31, edge=250.0, shear=1.0)
    ref = oracle.cell_list_pairs(sheared["cell"], sheared["pos"], 95.0, 40.0, rc2, False)
    full = oracle.all_pairs(sheared["cell"], sheared["pos"], rc2, False, 1)
    assert ref < full and len(full - ref) == 4
