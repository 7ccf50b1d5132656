"""The evaluation is stream-ordered and free of host synchronisation, so it can be
captured in a CUDA graph: replaying (positions from device memory + evaluation) gives
the same results as direct evaluation of the same positions."""
import numpy as np
import pytest

import d3_systems as S
from d3_b200 import D3, OPT_PRECISION

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_graph_replay_matches_direct_evaluation(precision):
    import torch

    sys_ = S.triclinic_box(400, seed=12)
    kw = dict(rc=95.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)
    d = D3(sys_["Z"], len(sys_["Z"]), **kw)
    d.set_option(OPT_PRECISION, precision)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    d.compute()  # sizes the ATM list before capture
    pos = torch.tensor(sys_["pos"], dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        d.set_positions_device(pos.data_ptr(), stream.cuda_stream)
        d.compute_async(stream.cuda_stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        d.set_positions_device(pos.data_ptr(), stream.cuda_stream)
        d.compute_async(stream.cuda_stream)
    torch.cuda.synchronize()
    rng = np.random.default_rng(0)
    ref = D3(sys_["Z"], len(sys_["Z"]), **kw)
    ref.set_option(OPT_PRECISION, precision)
    ref.set_cell(sys_["cell"])
    cur = sys_["pos"].copy()
    for _ in range(3):
        step = rng.normal(0.0, 0.01, cur.shape)
        cur = cur + step
        with torch.cuda.stream(stream):
            pos.add_(torch.tensor(step, device="cuda"))
            graph.replay()
        torch.cuda.synchronize()
        e, f, s = d.fetch_results()
        ref.set_atoms(cur, sys_["Z"])
        e1, f1, s1 = ref.compute()
        # FP64: equal to rounding; FP32 arithmetic: last-bit differences of partial sums
        etol, ftol, stol = (1e-11, 1e-10, 1e-12) if precision == 0 else (1e-8, 1e-7, 1e-9)
        assert abs(e - e1) <= etol * abs(e1)
        assert np.abs(f - f1).max() <= ftol
        assert np.abs(s - s1).max() <= stol
    del graph
    ref.close()
    d.close()
