"""Sharded evaluation on the GPU: the ranks of a world of 2 or 3 are run one after the
other on one GPU (each its own handle), their dE/dCN parts summed, then their result
parts summed; the sum must equal the unsharded evaluation of the same structure (FP64:
summation order only; precision form: FP32 level). The two-stage API is the one a real
multi-GPU run drives with NCCL all-reduces (d3_shard.py)."""
import numpy as np
import pytest

import d3_systems as S
from d3_b200 import D3, OPT_ATM_SCHEDULE, OPT_PRECISION

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def make(sys_, precision, schedule=0, rc_atm=40.0):
    d = D3(sys_["Z"], len(sys_["Z"]), rc=95.0, rc_cn=40.0, rc_atm=rc_atm)
    d.set_option(OPT_PRECISION, precision)
    d.set_option(OPT_ATM_SCHEDULE, schedule)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    return d


def sharded(sys_, world, precision, schedule=0, rc_atm=40.0):
    n = len(sys_["Z"])
    hs = [make(sys_, precision, schedule, rc_atm) for _ in range(world)]
    Gs = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(world)]
    outs = [torch.zeros(10 + 3 * n, dtype=torch.float64, device="cuda") for _ in range(world)]
    for r, h in enumerate(hs):
        h.shard_begin(r, world, Gs[r].data_ptr())
    G = sum(Gs)
    for r, h in enumerate(hs):
        h.shard_end(G.data_ptr(), outs[r].data_ptr())
    torch.cuda.synchronize()
    o = sum(outs).cpu().numpy()
    return float(o[0]), o[1:1 + 3 * n].reshape(n, 3), o[1 + 3 * n:10 + 3 * n].reshape(3, 3)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("precision,schedule", [(0, 0), (1, 0), (1, 1)])
def test_sharded_sum_equals_single(world, precision, schedule):
    sys_ = S.triclinic_box(600, seed=9)
    e0, f0, s0 = make(sys_, precision, schedule).compute()
    e1, f1, s1 = sharded(sys_, world, precision, schedule)
    tol = 1e-12 if precision == 0 else 1e-7
    assert abs(e1 - e0) <= tol * abs(e0)
    assert np.abs(f1 - f0).max() <= tol * 100 * np.abs(f0).max()
    assert np.abs(s1 - s0).max() <= tol * 100 * np.abs(s0).max()


def test_sharded_without_atm_and_small_cell():
    # two-body + CN only, and a small cell (repeated-index ATM triplets) with ATM
    sys_ = S.triclinic_box(300, seed=4)
    e0, f0, s0 = make(sys_, 0, rc_atm=None).compute()
    e1, f1, s1 = sharded(sys_, 2, 0, rc_atm=None)
    assert abs(e1 - e0) <= 1e-12 * abs(e0)
    assert np.abs(f1 - f0).max() <= 1e-10 * np.abs(f0).max()
    fe = S.gtest_bcc_fe(True)
    fe["pos"] = fe["pos"] + np.random.default_rng(0).uniform(-0.1, 0.1, fe["pos"].shape)
    d = D3(fe["Z"], len(fe["Z"]), rc=30.0, rc_cn=30.0, rc_atm=30.0)
    d.set_cell(fe["cell"])
    d.set_atoms(fe["pos"], fe["Z"])
    e0, f0, s0 = d.compute()
    n = len(fe["Z"])
    hs = []
    for _ in range(2):
        h = D3(fe["Z"], n, rc=30.0, rc_cn=30.0, rc_atm=30.0)
        h.set_cell(fe["cell"])
        h.set_atoms(fe["pos"], fe["Z"])
        hs.append(h)
    Gs = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    outs = [torch.zeros(10 + 3 * n, dtype=torch.float64, device="cuda") for _ in range(2)]
    for r, h in enumerate(hs):
        h.shard_begin(r, 2, Gs[r].data_ptr())
    G = Gs[0] + Gs[1]
    for r, h in enumerate(hs):
        h.shard_end(G.data_ptr(), outs[r].data_ptr())
    torch.cuda.synchronize()
    o = (outs[0] + outs[1]).cpu().numpy()
    assert abs(o[0] - e0) <= 1e-12 * abs(e0)
    assert np.abs(o[1:1 + 3 * n].reshape(n, 3) - f0).max() <= 1e-10 * np.abs(f0).max()


def test_sharded_batch_handle():
    # a batch handle of three structures: results are 10 S + 3 n values, S taken from the handle
    from d3_b200 import D3Batch

    structs = [S.triclinic_box(200, seed=11), S.triclinic_box(150, seed=12), S.water_box(0)]
    elements = sorted(set(int(z) for s in structs for z in s["Z"]))
    n = sum(len(s["Z"]) for s in structs)

    def batch():
        b = D3Batch(elements, len(structs), n, rc=95.0, rc_cn=40.0, rc_atm=40.0)
        b.set_structures(structs)
        return b

    e0, f0, s0 = batch().compute()
    world = 2
    hs = [batch() for _ in range(world)]
    assert hs[0].shard_structures() == len(structs) and hs[0].shard_length() == n
    Gs = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(world)]
    outs = [torch.zeros(10 * len(structs) + 3 * n, dtype=torch.float64, device="cuda") for _ in range(world)]
    for r, h in enumerate(hs):
        h.shard_begin(r, world, Gs[r].data_ptr())
    G = sum(Gs)
    for r, h in enumerate(hs):
        h.shard_end(G.data_ptr(), outs[r].data_ptr())
    torch.cuda.synchronize()
    o = sum(outs).cpu().numpy()
    nS = len(structs)
    np.testing.assert_allclose(o[:nS], e0, rtol=1e-12)
    f1 = o[nS:nS + 3 * n].reshape(n, 3)
    np.testing.assert_allclose(f1, np.concatenate(f0), rtol=0, atol=1e-10 * np.abs(np.concatenate(f0)).max())
    np.testing.assert_allclose(o[nS + 3 * n:].reshape(nS, 3, 3), s0, rtol=0, atol=1e-10 * np.abs(s0).max())
