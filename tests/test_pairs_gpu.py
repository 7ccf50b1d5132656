"""The pair passes on compact atom groups (default: CN, two-body, chain rule) against the
one-warp-per-atom kernels (D3_OPT_PAIR_KERNEL = 1), both forms, on geometries that exercise
the group cut and the merged block stencils: the benchmark generator (2 x 2 row blocks),
atoms given outside the cell (exact per-pair image box), a small cell whose stencils wrap
many periods, the water box (13^3 image box), zero damping, and a batch of uneven
structures. FP64: CN, per-atom two-body and chain-rule terms equal to 1e-12 relative
(summation order only); FP32: energies and CN to 1e-5, the derivative columns (sums of
terms of both signs) to 1e-4 of the largest value; the in-range pair counts equal.
The smooth CN cutoff in the precision form is checked against the FP64 oracle."""
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
    cn = d.atom_arrays()[0]
    _, cnt = d.pass_times()
    d.close()
    return e, f, s, t, int(cnt[1]), cn, int(cnt[2])


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
    for k in (4, 6):  # two-body and CN in-range pair counts
        assert a[k] == b[k] or (precision and abs(a[k] - b[k]) <= 1e-6 * b[k]), (k, a[k], b[k])
    tol = 1e-12 if precision == 0 else 1e-5
    np.testing.assert_allclose(a[5], b[5], rtol=tol, atol=tol)
    for cols in (slice(0, 1), slice(1, 2), slice(2, 5), slice(5, 11), slice(22, 25), slice(25, 31)):
        # FP32: the derivative columns sum terms of both signs in a different order
        ctol = tol if (precision == 0 or cols.start == 0) else 1e-4
        scale = np.abs(b[3][:, cols]).max()
        assert np.abs(a[3][:, cols] - b[3][:, cols]).max() <= ctol * scale, cols
    assert abs(a[0] - b[0]) <= tol * abs(b[0])
    assert np.abs(a[1] - b[1]).max() <= tol * np.abs(b[1]).max()


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


@pytest.mark.parametrize("kernel", [0, 1])
def test_smooth_cn_precision_form_against_oracle(kernel):
    # the tanh^3 CN cutoff (the reference's SMOOTH_CUTOFF_CN) in the FP32 pair arithmetic
    # of the precision form, both pair-kernel layouts, at the precision form's bars
    import oracle
    from d3_b200 import OPT_SMOOTH_CN

    sys_ = S.triclinic_box(300, seed=7)
    d = D3(sys_["Z"], len(sys_["Z"]), rc=60.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)
    d.set_option(OPT_PRECISION, 1)
    d.set_option(OPT_SMOOTH_CN, 1)
    d.set_option(OPT_PAIR_KERNEL, kernel)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    e, f, s = d.compute()
    cn = d.atom_arrays()[0]
    d.close()
    r = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], rc=60.0, rc_cn=40.0, rc_atm=40.0, damping=1,
                       functional=0, smooth_cn=True)
    np.testing.assert_allclose(cn, r["cn"], rtol=1e-5, atol=1e-5)
    assert abs(e - r["energy"]) <= 1e-6 * abs(r["energy"])
    assert np.abs(f - r["forces"]).max() <= 1e-4
    assert np.abs(s - r["stress"]).max() <= 1e-6
