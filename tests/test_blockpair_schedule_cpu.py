"""Index algebra of the block-pair ATM schedule (lasp-d3_b200/csrc/d3_atm32b.cuh, k_atm32b),
emulated lane by lane on the CPU: every unordered pair of entries of a block pair is visited
exactly once, and the y-side sums, which travel four lanes down per iteration as packed pairs
of steps and are gathered by three shuffles at the end, arrive at the right entry with the
contributions of exactly the x entries that visited it.

The kernel's own results are checked on the GPU against the mirror schedule and the FP64
oracle (tests/test_precision_gpu.py); this test pins the schedule's invariants, which hold
for any block pair, so that a change of the step or shift arithmetic fails here first."""
from collections import Counter

import pytest

LANES = 32


def emulate(diag):
    """Visits (x, y) of one block pair, and for each y the multiset of x's whose
    contributions the gather delivers to it (x, y: entry indices 0..31 of the blocks)."""
    s0, s1 = (1, 17) if diag else (0, 32)
    visits = []
    # ys[pq][c][lane]: the travelling y sums of step s + 2 pq + c, as multisets of x's
    ys = [[[Counter() for _ in range(LANES)] for _ in range(2)] for _ in range(2)]
    for s in range(s0, s1, 4):
        for L in range(LANES):
            for pq in range(2):
                k0 = (L + s + 2 * pq) & 31  # packed slot: entries k0 and k0 + 1 side by side
                for c in range(2):
                    t = s + 2 * pq + c
                    k = (k0 + c) & 31
                    if diag and not (t < 16 or L < 16):
                        continue
                    visits.append((L, k))
                    ys[pq][c][L][L] += 1
        # shift: lane L takes the sums of lane L + 4
        for pq in range(2):
            for c in range(2):
                ys[pq][c] = [ys[pq][c][(L + 4) & 31] for L in range(LANES)]
    gathered = {}
    for L in range(LANES):
        g = Counter(ys[0][0][L])
        g += ys[0][1][(L - 1) & 31]
        g += ys[1][0][(L - 2) & 31]
        g += ys[1][1][(L - 3) & 31]
        gathered[(L + s1) & 31] = g
    return visits, gathered


@pytest.mark.parametrize("diag", [False, True])
def test_every_pair_once_and_y_sums_reach_their_entry(diag):
    visits, gathered = emulate(diag)
    if diag:
        # unordered pairs of distinct entries, each once
        pairs = Counter(tuple(sorted(v)) for v in visits)
        assert all(x != y for x, y in visits)
        assert len(pairs) == LANES * (LANES - 1) // 2 and set(pairs.values()) == {1}
    else:
        pairs = Counter(visits)
        assert len(pairs) == LANES * LANES and set(pairs.values()) == {1}
    # the gather gives entry y exactly the x's that visited it, each once
    expect = {y: Counter() for y in range(LANES)}
    for x, y in visits:
        expect[y][x] += 1
    assert sorted(gathered) == list(range(LANES))
    for y in range(LANES):
        assert gathered[y] == expect[y], y


def test_packed_steps_fill_whole_iterations():
    """Four steps per iteration: 8 iterations off the diagonal, 4 on it (steps 1..16, the
    last of them on half the lanes), none cut short."""
    assert len(range(0, 32, 4)) * 4 == 32
    assert len(range(1, 17, 4)) * 4 == 16
