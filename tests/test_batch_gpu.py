"""Batching form: many independent periodic structures of uneven size in one handle and
one launch per pass; each structure's results equal those of its own single handle and
of the FP64 oracle."""
import numpy as np
import pytest

import d3_systems as S
import oracle
from d3_b200 import D3, D3Batch, OPT_PRECISION

pytestmark = pytest.mark.gpu

KW = dict(rc=95.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)


def structures(count=12, seed=5):
    return S.batch_structs(count=count, seed=seed, nmin=8, nmax=300)


def single(s, precision=0):
    d = D3(s["Z"], len(s["Z"]), **KW)
    d.set_option(OPT_PRECISION, precision)
    d.set_cell(s["cell"])
    d.set_atoms(s["pos"], s["Z"])
    out = d.compute()
    d.close()
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_single_handles(precision):
    sts = structures()
    elements = sorted(set(int(z) for s in sts for z in s["Z"]))
    b = D3Batch(elements, len(sts), sum(len(s["Z"]) for s in sts), **KW)
    b.set_option(OPT_PRECISION, precision)
    b.set_structures(sts)
    e, f, st = b.compute()
    b.close()
    # FP64: equal to rounding; FP32 arithmetic: lane assignment of the ATM entries varies
    # between launches, so FP32 partial sums differ in their last bits
    etol, ftol, stol = (1e-12, 1e-11, 1e-12) if precision == 0 else (1e-8, 1e-7, 1e-9)
    for k, s in enumerate(sts):
        e1, f1, s1 = single(s, precision)
        assert abs(e[k] - e1) <= etol * abs(e1) + 1e-14
        assert np.abs(f[k] - f1).max() <= ftol
        assert np.abs(st[k] - s1).max() <= stol


def test_batch_matches_oracle():
    sts = structures(count=6, seed=9)
    elements = sorted(set(int(z) for s in sts for z in s["Z"]))
    b = D3Batch(elements, len(sts), sum(len(s["Z"]) for s in sts), **KW)
    b.set_structures(sts)
    e, f, st = b.compute()
    b.close()
    for k, s in enumerate(sts):
        r = oracle.compute(s["pos"], s["Z"], s["cell"], init_elements=elements, **KW)
        assert abs(e[k] - r["energy"]) <= 1e-9 * abs(r["energy"])
        assert np.abs(f[k] - r["forces"]).max() <= 1e-7
        assert np.abs(st[k] - r["stress"]).max() <= 1e-7


def test_batch_refuses_single_structure_calls():
    sts = structures(count=3, seed=2)
    elements = sorted(set(int(z) for s in sts for z in s["Z"]))
    b = D3Batch(elements, 3, sum(len(s["Z"]) for s in sts), **KW)
    b.set_structures(sts)
    import ctypes

    e = np.zeros(1)
    st = b.lib.d3_compute_f64(b.h, e.ctypes.data, None, None)
    assert st != 0 and b"batch" in b.lib.d3_last_error()
    b.close()
