"""Sharded evaluation of one structure over the ranks of a torch.distributed process group.

One process per GPU (NCCL over NVLink / NVSwitch). Every rank holds the same structure in
its own handle; d3_shard_begin computes the coordination numbers and C6 weights of every
atom and this rank's share (every world-th atom / ATM apex) of the two-body and ATM terms,
leaving this rank's part of dE/dCN; the ranks sum dE/dCN (all-reduce of n doubles), then
d3_shard_end runs the chain rule of this rank's share and the ranks sum the results
(all-reduce of S + 3n + 9S doubles: energies, forces, stresses). Those two all-reduces are
the only exchanges: positions are replicated, and the CN pass is cheap enough to repeat on
every rank instead of all-gathering it.

    dist.init_process_group("nccl", ...)
    d3 = D3(elements, n, rc=95.0, rc_cn=40.0, rc_atm=40.0)
    d3.set_cell(cell); d3.set_atoms(pos, Z)
    energy, forces, stress = ShardedEvaluator(d3).compute()
"""
class ShardedEvaluator:
    """Drives the two stages of a handle (anything with shard_length, shard_structures,
    shard_begin and shard_end) and the two all-reduces between and after them.

    The results buffer holds 10 S + 3 n doubles, S the structures of the handle (one for a
    D3 handle, the batch size for a D3Batch); S is taken from the handle, since
    d3_shard_end writes that many values whatever buffer it is given. `num_structures`,
    when given, must agree with it."""

    def __init__(self, handle, group=None, num_structures=None, device=None):
        import torch
        import torch.distributed as dist

        self.torch, self.dist = torch, dist
        self.h = handle
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.n = int(handle.shard_length())
        self.S = int(handle.shard_structures())
        if num_structures is not None and int(num_structures) != self.S:
            raise ValueError("num_structures=%d but the handle holds %d structures" % (num_structures, self.S))
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
        self.G = torch.zeros(self.n, dtype=torch.float64, device=device)
        self.out = torch.zeros(10 * self.S + 3 * self.n, dtype=torch.float64, device=device)

    def _stream(self):
        if self.G.is_cuda:
            return self.torch.cuda.current_stream().cuda_stream
        return None

    def compute_device(self):
        """Run the evaluation; the summed results stay in self.out (device)."""
        s = self._stream()
        self.h.shard_begin(self.rank, self.world, self.G.data_ptr(), s)
        self.dist.all_reduce(self.G, group=self.group)
        self.h.shard_end(self.G.data_ptr(), self.out.data_ptr(), s)
        self.dist.all_reduce(self.out, group=self.group)
        return self.out

    def compute(self):
        """Energies (eV), forces (eV/A, [n,3]) and stresses (eV/A^3, [S,3,3]); a single
        structure returns (float energy, forces, 3x3 stress)."""
        o = self.compute_device().cpu().numpy()
        S, n = self.S, self.n
        e = o[:S].copy()
        f = o[S:S + 3 * n].reshape(n, 3).copy()
        st = o[S + 3 * n:S + 3 * n + 9 * S].reshape(S, 3, 3).copy()
        if S == 1:
            return float(e[0]), f, st[0]
        return e, f, st

