"""Sharded evaluation, host side: ShardedEvaluator's two all-reduces over a gloo process group of
two ranks on CPU. Each rank's handle is a stand-in whose two stages are known linear maps
(stage 1 writes a rank-specific part of dE/dCN; stage 2 maps the summed dE/dCN to a
rank-specific part of the results), so the expected sum is known exactly: the test checks
that stage 2 sees the dE/dCN of all ranks and that the results are summed over ranks."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

N = 7


class LinearStages:
    """Stand-in for a D3 (S = 1) or D3Batch (S > 1) handle: stage 1 writes G_r = a_r; stage 2
    writes out_r = B_r G + c_r over the 10 S + 3 N result values."""

    def __init__(self, rank, S=1):
        rng = np.random.default_rng(100 + rank + 10 * S)
        self.S = S
        self.a = rng.normal(size=N)
        self.B = rng.normal(size=(10 * S + 3 * N, N))
        self.c = rng.normal(size=10 * S + 3 * N)
        self.seen_G = None

    def shard_length(self):
        return N

    def shard_structures(self):
        return self.S

    def shard_begin(self, rank, world, G_ptr, stream):
        g = torch.from_numpy(self.a.copy())
        _write(G_ptr, g)

    def shard_end(self, G_ptr, out_ptr, stream):
        G = _read(G_ptr, N)
        self.seen_G = G.copy()
        S = self.S
        assert _BUFS[out_ptr].numel() == 10 * S + 3 * N  # the buffer the evaluator sized
        _write(out_ptr, torch.from_numpy(self.B @ G + self.c))


_BUFS = {}


def _write(ptr, t):
    _BUFS[ptr].copy_(t)


def _read(ptr, n):
    return _BUFS[ptr][:n].numpy().copy()


def _worker(rank, world, port, q, S=1):
    import torch.distributed as dist

    import d3_shard

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        h = LinearStages(rank, S)
        ev = d3_shard.ShardedEvaluator(h, device="cpu")
        _BUFS[ev.G.data_ptr()] = ev.G
        _BUFS[ev.out.data_ptr()] = ev.out
        e, f, s = ev.compute()
        q.put((rank, e, f, s, h.seen_G))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("S", [1, 3])
def test_two_rank_gloo_protocol(S):
    # S = 3: a batch handle; the results buffer must be sized from the handle
    world = 2
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, S)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, e, f, s, g = q.get(timeout=120)
        res[r] = (e, f, s, g)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    hs = [LinearStages(r, S) for r in range(world)]
    G = sum(h.a for h in hs)
    out = sum(h.B @ G + h.c for h in hs)
    for r in range(world):
        e, f, s, g = res[r]
        np.testing.assert_allclose(g, G, rtol=0, atol=1e-12)
        np.testing.assert_allclose(np.ravel(e), out[:S], rtol=0, atol=1e-12)
        np.testing.assert_allclose(np.ravel(f), out[S:S + 3 * N], rtol=0, atol=1e-12)
        np.testing.assert_allclose(np.ravel(s), out[S + 3 * N:S + 3 * N + 9 * S], rtol=0, atol=1e-12)


def test_structure_count_mismatch_is_rejected():
    # an explicit count that disagrees with the handle would size the buffer wrongly
    import torch.distributed as dist

    import d3_shard

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0, world_size=1)
    try:
        with pytest.raises(ValueError):
            d3_shard.ShardedEvaluator(LinearStages(0, 2), num_structures=1, device="cpu")
        ev = d3_shard.ShardedEvaluator(LinearStages(0, 2), device="cpu")
        assert ev.out.numel() == 10 * 2 + 3 * N
    finally:
        dist.destroy_process_group()
