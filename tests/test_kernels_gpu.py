"""Device-side helpers and engine bookkeeping (GPU)."""
import numpy as np
import pytest

import d3_systems as S
from d3_b200 import D3, peak_probe, selftest_math

pytestmark = pytest.mark.gpu


def test_refined_math_helpers_match_cuda_double():
    # rsqrt / reciprocal / inverse cube root used in the ATM kernel: float seed + Newton
    # steps, against CUDA's double 1/sqrt, 1/x and cbrt over [1e-12, 1e14]. One step
    # squares the seed's relative error (~1e-7 -> ~1e-13); two reach double rounding.
    err = selftest_math()
    assert err[0] < 2e-13 and err[1] < 2e-13 and err[2] < 2e-12, err
    assert err[3] < 4e-16 and err[4] < 4e-16 and err[5] < 6e-16, err


def test_pass_times_and_counters():
    s = S.water_box(0)
    d = D3(s["Z"], len(s["Z"]), rc=95.0, rc_cn=40.0, rc_atm=40.0)
    d.set_cell(s["cell"])
    d.set_atoms(s["pos"], s["Z"])
    d.compute()
    pt, cnt = d.pass_times()
    d.close()
    assert set(pt) == {"bin", "cn", "twobody", "atm_list", "atm", "chain", "finalize"}
    assert all(v >= 0 for v in pt.values())
    assert cnt[0] > 0 and cnt[0] % 2 == 0  # every triplet is visited from both entries
    assert cnt[1] > 0 and cnt[2] > 0


def test_peak_probe_is_plausible():
    fp64 = peak_probe(True)
    fp32 = peak_probe(False)
    assert 5.0 < fp64 < 200.0 and fp32 > fp64
