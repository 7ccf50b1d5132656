"""Precision form (FP32 pair/triplet arithmetic, FP64 weights, dE/dCN and reductions)
against the FP64 oracle. Targets of the form: energy within 1e-6 relative, forces within
1e-4 eV/A, stress within 1e-6 eV/A^3 (the accuracy bar of the mixed-precision form)."""
import numpy as np
import pytest

import d3_systems as S
import oracle
from d3_b200 import D3, OPT_ATM_FORCE_SCALED, OPT_PRECISION

pytestmark = pytest.mark.gpu


def run(sys_, rc, rc_cn, rc_atm, damping, functional, table=0, options=()):
    d = D3(sys_["Z"], len(sys_["Z"]), rc=rc, rc_cn=rc_cn, rc_atm=rc_atm, damping=damping, functional=functional,
           table=table)
    d.set_option(OPT_PRECISION, 1)
    for o, v in options:
        d.set_option(o, v)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    e, f, s = d.compute()
    d.close()
    return e, f, s


@pytest.mark.parametrize("damping", [0, 1])
@pytest.mark.parametrize("case", ["small", "fe", "water", "tric"])
def test_precision_form_error_bounds(case, damping):
    if case == "small":
        sys_, kw = S.gtest_small_system(), dict(rc=40.0, rc_cn=40.0, rc_atm=40.0, functional=1)
    elif case == "fe":
        sys_ = S.gtest_bcc_fe(True)
        sys_["pos"] = sys_["pos"] + np.random.default_rng(0).uniform(-0.1, 0.1, sys_["pos"].shape)
        kw = dict(rc=30.0, rc_cn=30.0, rc_atm=30.0, functional=1)
    elif case == "water":
        sys_, kw = S.water_box(0), dict(rc=95.0, rc_cn=40.0, rc_atm=40.0, functional=0)
    else:
        sys_, kw = S.triclinic_box(400, seed=21), dict(rc=95.0, rc_cn=40.0, rc_atm=40.0, functional=0)
    e, f, s = run(sys_, damping=damping, **kw)
    r = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], damping=damping, **kw)
    assert abs(e - r["energy"]) <= 1e-6 * abs(r["energy"]), (e, r["energy"])
    assert np.abs(f - r["forces"]).max() <= 1e-4
    assert np.abs(s - r["stress"]).max() <= 1e-6


def test_precision_form_scaled_atm_forces():
    sys_ = S.gtest_bcc_fe()
    sys_["pos"] = sys_["pos"] + np.random.default_rng(4).uniform(-0.1, 0.1, sys_["pos"].shape)
    kw = dict(rc=30.0, rc_cn=30.0, rc_atm=30.0, functional=1, damping=1)
    e, f, s = run(sys_, options=((OPT_ATM_FORCE_SCALED, 1),), **kw)
    r = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], atm_force_scaled=True, **kw)
    assert abs(e - r["energy"]) <= 1e-6 * abs(r["energy"])
    assert np.abs(f - r["forces"]).max() <= 1e-4


def _half_list_lengths(sys_, rc_bohr, stride=25):
    """Half-list lengths (entries j <= a within rc, all images) of every stride-th apex,
    for cells whose heights exceed rc (images -1..1 suffice)."""
    pos, cell = sys_["pos"], sys_["cell"]
    rc = rc_bohr * 0.52917726
    imgs = np.array([[i, j, k] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)], float) @ cell
    out = []
    for a in range(0, len(pos), stride):
        v = (pos[: a + 1][None] + imgs[:, None]) - pos[a]
        d2 = (v * v).sum(-1)
        out.append(int(((d2 <= rc * rc) & (d2 >= 1e-12)).sum()))
    return np.array(out)


@pytest.mark.parametrize("case", ["tric", "split", "fe", "water"])
def test_atm_schedules_agree(case):
    """Block-pair schedule (each triplet once; lists longer than its capacity go to the
    mirror kernel) against the mirror-symmetric schedule (each triplet twice): the same
    in-range triplets (visit counters equal) and the same energy, forces and stress to FP32
    level. "split": rc_ATM 50 bohr in a 3,000-atom box, so that about a sixth of the half
    lists are longer than the block-pair capacity for five element types (6,656 entries)
    and one evaluation runs both kernels; its cells are lower than 2 rc_ATM, so atoms
    repeat within a list (pair weights below 1)."""
    from d3_b200 import OPT_ATM_SCHEDULE

    if case == "tric":
        sys_, kw = S.triclinic_box(3000, seed=5), dict(rc=95.0, rc_cn=40.0, rc_atm=40.0)
    elif case == "split":
        sys_, kw = S.triclinic_box(3000, seed=5), dict(rc=95.0, rc_cn=40.0, rc_atm=50.0)
        lens = _half_list_lengths(sys_, 50.0)
        assert lens.max() > 6656 and lens.min() < 4096
    elif case == "fe":
        sys_ = S.gtest_bcc_fe(True)
        sys_["pos"] = sys_["pos"] + np.random.default_rng(1).uniform(-0.1, 0.1, sys_["pos"].shape)
        kw = dict(rc=30.0, rc_cn=30.0, rc_atm=30.0)
    else:
        sys_, kw = S.water_box(0), dict(rc=95.0, rc_cn=40.0, rc_atm=40.0)
    out = []
    for sched in (0, 1):
        d = D3(sys_["Z"], len(sys_["Z"]), damping=1, functional=0, **kw)
        d.set_option(OPT_PRECISION, 1)
        d.set_option(OPT_ATM_SCHEDULE, sched)
        d.set_cell(sys_["cell"])
        d.set_atoms(sys_["pos"], sys_["Z"])
        e, f, s = d.compute()
        _, cnt = d.pass_times()
        atm = d.atom_arrays()
        out.append((e, f, s, int(cnt[0]), atm[2]))
        d.close()
    (e0, f0, s0, c0, a0), (e1, f1, s1, c1, a1) = out
    assert c0 == c1 and c0 > 0
    assert abs(e0 - e1) <= 1e-7 * abs(e1)
    assert np.abs(f0 - f1).max() <= 1e-5 * np.abs(f1).max() + 1e-9
    assert np.abs(s0 - s1).max() <= 1e-6 * np.abs(s1).max() + 1e-12
    # per-atom energy shares (E/3 of every triplet through the atom) agree as well
    assert np.abs(a0 - a1).max() <= 1e-6 * np.abs(a1).max()


@pytest.mark.parametrize("shape", [(8, 0, 0, 0, 0), (4, 2, 0, 0, 0), (6, 0, 4096, 0, 0), (12, 0, 4096, 0, 0),
                                   (0, 0, 0, 3, 0), (8, 0, 0, 5, 0), (0, 0, 0, 0, 1), (8, 0, 0, 0, 1)])
@pytest.mark.parametrize("case", ["tric", "fe"])
def test_block_pair_shapes_agree(case, shape):
    """Launch shapes of the block-pair ATM kernel (warps per CTA, CTAs per SM, list
    capacity, CTAs sharing an apex; above 8 warps each stages one y block at a time, 8
    and fewer two) against the default shape (12 warps where they fit): the same in-range triplets and the same results to FP32 level. A
    4,096-entry capacity sends the longest lists of the 3,000-atom box (up to about 4,100
    entries at rc_ATM 40) to the mirror kernel; a split of 3 or 5 makes several CTAs add
    their shares of each apex; the last two skip out-of-range visits per two steps."""
    from d3_b200 import OPT_ATM_CTAS_PER_SM, OPT_ATMB_FINE_SKIP, OPT_ATMB_LIST_CAPACITY, OPT_ATMB_SPLIT, OPT_ATMB_WARPS

    if case == "tric":
        sys_, kw = S.triclinic_box(3000, seed=5), dict(rc=95.0, rc_cn=40.0, rc_atm=40.0)
    else:
        sys_ = S.gtest_bcc_fe(True)
        sys_["pos"] = sys_["pos"] + np.random.default_rng(1).uniform(-0.1, 0.1, sys_["pos"].shape)
        kw = dict(rc=30.0, rc_cn=30.0, rc_atm=30.0)
    out = []
    for opts in ((), ((OPT_ATMB_WARPS, shape[0]), (OPT_ATM_CTAS_PER_SM, shape[1]), (OPT_ATMB_LIST_CAPACITY, shape[2]),
                      (OPT_ATMB_SPLIT, shape[3]), (OPT_ATMB_FINE_SKIP, shape[4]))):
        d = D3(sys_["Z"], len(sys_["Z"]), damping=1, functional=0, **kw)
        d.set_option(OPT_PRECISION, 1)
        for o, v in opts:
            d.set_option(o, v)
        d.set_cell(sys_["cell"])
        d.set_atoms(sys_["pos"], sys_["Z"])
        e, f, s = d.compute()
        _, cnt = d.pass_times()
        out.append((e, f, s, int(cnt[0])))
        d.close()
    (e0, f0, s0, c0), (e1, f1, s1, c1) = out
    assert c0 == c1 and c0 > 0
    assert abs(e0 - e1) <= 1e-7 * abs(e0)
    assert np.abs(f0 - f1).max() <= 1e-5 * np.abs(f0).max() + 1e-9
    assert np.abs(s0 - s1).max() <= 1e-6 * np.abs(s0).max() + 1e-12
