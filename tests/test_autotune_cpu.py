"""The autotuner on the host: a stand-in handle whose pass times depend on the options set
(a known optimum per knob) shows that the tuner times every candidate, keeps the fastest
pair kernel / bin width and the fastest block-pair ATM shape (precision form) or mirror
tile and CTAs (FP64 form), applies them, and caches them by workload key."""
import pytest

import d3_autotune
from d3_b200 import (OPT_ATM_CTAS_PER_SM, OPT_ATM_TILE, OPT_ATMB_LIST_CAPACITY, OPT_ATMB_WARPS, OPT_BIN_DIVISOR,
                     OPT_PAIR_KERNEL)


class FakeHandle:
    def __init__(self):
        self.opt = {}

    def set_option(self, k, v):
        self.opt[k] = v

    def compute(self):
        pass

    def pass_times(self):
        o = self.opt.get
        pair = 10.0 + abs(o(OPT_BIN_DIVISOR, 6) - 4) + (3.0 if o(OPT_PAIR_KERNEL, 0) == 1 else 0.0)
        # precision optimum: 10 warps; FP64 optimum: tile 128, 2 CTAs per SM
        atm = 100.0 - (20.0 if o(OPT_ATMB_WARPS, 0) == 10 else 0.0) + (5.0 if o(OPT_ATMB_LIST_CAPACITY, 0) else 0.0)
        atm += abs(o(OPT_ATM_TILE, 0) - 128) / 64.0 + (0.0 if o(OPT_ATM_CTAS_PER_SM, 0) == 2 else 1.0)
        return {"bin": 0.0, "cn": 0.0, "twobody": pair, "atm_list": 0.0, "atm": atm, "chain": 0.0, "finalize": 0.0}, None


@pytest.mark.parametrize("precision", [0, 1])
def test_tuner_keeps_the_fastest_candidates(tmp_path, monkeypatch, precision):
    monkeypatch.setenv("D3_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    h = FakeHandle()
    key = "test|p%d" % precision
    res = d3_autotune.tune(h, key, repeats=1)
    assert res["bin_divisor"] == 4 and res["pair_kernel"] == 0
    if precision:
        assert res["atmb_warps"] == 10 and res["atmb_mcap"] == 0
        assert len([t for t in res["trials"] if "atmb_warps" in t]) == len(d3_autotune.ATMB_SHAPES)
        assert res["atmb_fine_skip"] == 0
    else:
        assert res["atm_tile"] == 128 and res["atm_ctas_per_sm"] == 2
    # applied to the handle, and reused from the cache without timing
    assert h.opt[OPT_BIN_DIVISOR] == 4 and h.opt[OPT_ATMB_WARPS] == res["atmb_warps"]
    h2 = FakeHandle()
    again = d3_autotune.tune(h2, key)
    assert again["cached"] and h2.opt[OPT_ATM_TILE] == res["atm_tile"]
