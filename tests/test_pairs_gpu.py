"""The two-body pass on compact atom groups (default) against the one-warp-per-atom kernel
(D3_OPT_PAIR_KERNEL = 1), both forms, on geometries that exercise the group cut and the
merged block stencil: the benchmark generator (2 x 2 row blocks), atoms given outside the
cell (exact per-pair image box), a small cell whose stencil wraps many periods, the water
box (13^3 image box), zero damping, and a batch of uneven structures. FP64: per-atom
energies, dE/dCN and forces equal to 1e-12 relative (summation order only); FP32: to 1e-5
of the largest value; the in-range pair counts equal."""
import numpy as np
import pytest

import d3_systems as S
from d3_b200 import D3, D3Batch, OPT_PAIR_KERNEL, OPT_PRECISION

pytestmark = pytest.mark.gpu


def run(sys_, kernel, precision, rc=95.0, rc_cn=40.0, rc_atm=None, damping=1):
    d = D3(sys_["Z"], len(sys_["Z"]), rc=rc, rc_cn=rc_cn, rc_atm=rc_atm, damping=damping, functional=0)
    d.set_option(OPT_PRECISION, precision)
    d.set_option(OPT_PAIR_KERNEL, kernel)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    e, f, s = d.compute()
    t = d.pass_terms()
    _, cnt = d.pass_times()
    d.close()
    return e, f, s, t, int(cnt[1])


def unwrapped(n=300, seed=9):
    s = S.triclinic_box(n, seed=seed)
    rng = np.random.default_rng(2)
    s["pos"] = s["pos"] + rng.integers(-2, 3, size=(n, 3)) @ s["cell"]
    return s


CASES = {
    "config1_2000": lambda: S.triclinic_box(2000, seed=3),
    "unwrapped": unwrapped,
    "small_cell": lambda: S.gtest_bcc_fe(True),
    "water": lambda: S.water_box(0),
}


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("damping", [0, 1])
def test_grouped_two_body_matches_per_atom_kernel(case, precision, damping):
    sys_ = CASES[case]()
    a = run(sys_, 0, precision, damping=damping)
    b = run(sys_, 1, precision, damping=damping)
    assert a[4] == b[4] or (precision and abs(a[4] - b[4]) <= 1e-6 * b[4]), (a[4], b[4])
    tol = 1e-12 if precision == 0 else 1e-5
    for cols in (slice(0, 1), slice(1, 2), slice(2, 5), slice(5, 11)):
        scale = np.abs(b[3][:, cols]).max()
        assert np.abs(a[3][:, cols] - b[3][:, cols]).max() <= tol * scale, cols
    assert abs(a[0] - b[0]) <= tol * abs(b[0])


def test_grouped_two_body_batch():
    structs = S.batch_structs(24, seed=5, nmin=8, nmax=600)
    el = sorted(set(int(z) for s in structs for z in s["Z"]))
    n = sum(len(s["Z"]) for s in structs)
    out = []
    for kernel in (0, 1):
        b = D3Batch(el, len(structs), n, rc=95.0, rc_cn=40.0, rc_atm=None)
        b.set_option(OPT_PAIR_KERNEL, kernel)
        b.set_structures(structs)
        out.append(b.compute())
        b.close()
    np.testing.assert_allclose(out[0][0], out[1][0], rtol=1e-12)
    for fa, fb in zip(out[0][1], out[1][1]):
        np.testing.assert_allclose(fa, fb, rtol=0, atol=1e-12 * max(1.0, np.abs(fb).max()))
