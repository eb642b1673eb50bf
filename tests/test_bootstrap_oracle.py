"""Bootstrap building blocks on the CPU: replicate generation, and the
interval/post-order form of the transfer distance (the batched kernel's
algorithm) against the oracle's TransferDisStream on bitsets."""
import numpy as np
import pytest

import oracle as O
from casphy_b200 import bootstrap as B
from casphy_b200 import synth


def test_make_replicates_shapes():
    off, cells, w = B.make_replicates(1000, 256, 7, 100, 400, seed=3)
    n = np.diff(off.astype(np.int64))
    assert len(n) == 7 and n.min() >= 100 and n.max() <= 400
    assert np.all(w.sum(axis=1) == 256) and np.all(w >= 0)
    for r in range(7):
        c = cells[off[r]:off[r + 1]]
        assert np.all(np.diff(c.astype(np.int64)) > 0) and c.max() < 1000


def _intervals(edge, ntip):
    edge = np.asarray(edge, dtype=np.int64)
    nn = len(edge) + 1
    kids = [[] for _ in range(nn)]
    is_child = np.zeros(nn, bool)
    for p, c in edge:
        kids[p].append(c)
        is_child[c] = True
    root = int(np.flatnonzero(~is_child)[0])
    rank = np.zeros(ntip, np.int64)
    lo, hi = np.zeros(nn, np.int64), np.zeros(nn, np.int64)
    order, stack, nxt = [], [root], 0
    while stack:
        v = stack.pop()
        order.append(v)
        if v < ntip:
            rank[v] = nxt
            nxt += 1
        else:
            stack.extend(reversed(kids[v]))
    for v in reversed(order):
        if v < ntip:
            lo[v] = hi[v] = rank[v]
        else:
            lo[v] = min(lo[c] for c in kids[v])
            hi[v] = max(hi[c] for c in kids[v])
    nodes = [v for v in range(ntip, nn) if v != root]
    return rank, lo[nodes], hi[nodes]


def _interval_transfer(full_edge, N, rep_edge, cells):
    rank, lo, hi = _intervals(full_edge, N)
    n = len(cells)
    r = rank[cells]
    M = (r[None, :] >= lo[:, None]) & (r[None, :] <= hi[:, None])  # clade x local tip
    nX = M.sum(axis=1)
    Y = B.clade_bits(rep_edge, n, (n + 31) // 32)
    Ym = np.unpackbits(Y.view(np.uint8), bitorder="little", axis=1)[:, :n].astype(bool)
    C = M.astype(np.int64) @ Ym.T.astype(np.int64)
    d = nX[:, None] + Ym.sum(axis=1)[None, :] - 2 * C
    dist = np.minimum(d, n - d)
    return dist.min(axis=1), np.minimum(nX, n - nX)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_interval_transfer_equals_transferdisstream(seed):
    rng = np.random.default_rng(seed)
    N = 150
    par, ch, _ = synth.yule_tree(N, 0.1, rng)
    full_edge = np.stack([par, ch], axis=1)
    ncol = (N + 31) // 32
    full_bits = B.clade_bits(full_edge, N, ncol)
    for n in (3, 40, 97):
        cells = np.sort(rng.choice(N, size=n, replace=False))
        p2, c2, _ = synth.yule_tree(n, 0.1, rng)
        rep_edge = np.stack([p2, c2], axis=1)
        xb = B.clade_bits(rep_edge, n, ncol, tip_map=cells)
        mask = np.zeros(ncol, np.uint32)
        np.bitwise_or.at(mask, cells // 32, (1 << (cells % 32)).astype(np.uint32))
        ymin, ysize, _, _ = O.transfer_dis(full_bits & mask, xb, n)
        y2, s2 = _interval_transfer(full_edge, N, rep_edge, cells)
        assert np.array_equal(ymin, y2) and np.array_equal(ysize, s2)


def test_plain_pipeline_runs_on_the_oracle():
    words = synth.binary_workload(120, 64, 8, 0.05, 0.05, seed=4)
    full_edge, _, _ = O.join_bit(words, None, 1)
    N = words.shape[0]
    full_bits = B.clade_bits(full_edge, N, (N + 31) // 32)
    off, cells, w = B.make_replicates(N, 64, 3, 30, 80, seed=5)
    for r in range(3):
        c = cells[off[r]:off[r + 1]]
        ymin, ysize = B.plain_replicate(O, words, full_bits, c, w[r])
        assert len(ymin) == N - 2 and np.all(ysize <= len(c) // 2)
