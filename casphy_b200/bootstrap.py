"""Bootstrap replicates and the plain (one replicate at a time) pipeline.

A replicate of the bit-coded matrix is a subset of cells (rows, in
increasing order) and integer site weights, the column multiplicities of a
resample with replacement (the binary route of the reference hands those to
joinEdgeBitReverse as the weight file, src/functions.cpp:4485-4492).  The
plain pipeline runs, per replicate, the join (casphy_join_bit), the clade
writer (internal nodes except the root as tip bitsets, nodeDesBig in
src/functions.cpp:1277-1366) and TransferDisStream (casphy_transfer_dis) of
the full-data tree's clades restricted to the replicate's cells against the
replicate tree's clades; support counts follow cal.abs
(R/bootstrap_functions.R:190-219).  casphy_bootstrap_bit computes the same
numbers for all replicates in one pass.
"""
from __future__ import annotations

import numpy as np


def make_replicates(ncell: int, nsite: int, nrep: int, nmin: int, nmax: int, seed: int):
    """Replicate r: n_r ~ U{nmin..nmax} distinct cells (sorted) and the
    multiplicities of nsite columns drawn with replacement.  Returns
    (offsets u32[nrep+1], cells u32[sum n_r], weights f64[nrep, nsite])."""
    rng = np.random.default_rng(seed)
    n = rng.integers(nmin, nmax + 1, size=nrep)
    cells = [np.sort(rng.choice(ncell, size=int(k), replace=False)) for k in n]
    weights = np.stack([np.bincount(rng.integers(0, nsite, size=nsite), minlength=nsite) for _ in range(nrep)])
    offsets = np.concatenate([[0], np.cumsum(n)]).astype(np.uint32)
    return offsets, np.concatenate(cells).astype(np.uint32), weights.astype(np.float64)


def clade_bits(edge, ntip: int, ncol: int, tip_map=None):
    """Tip bitsets (rows of ncol u32) of the internal nodes except the root, in
    increasing node id.  tip_map[i] is the bit of tip i (default i)."""
    edge = np.asarray(edge, dtype=np.int64).reshape(-1, 2)
    nn = len(edge) + 1
    tip_map = np.arange(ntip) if tip_map is None else np.asarray(tip_map, dtype=np.int64)
    kids = [[] for _ in range(nn)]
    is_child = np.zeros(nn, dtype=bool)
    for p, c in edge:
        kids[p].append(c)
        is_child[c] = True
    root = int(np.flatnonzero(~is_child)[0])
    bits = np.zeros((nn, ncol), dtype=np.uint32)
    bits[np.arange(ntip), tip_map // 32] = (1 << (tip_map % 32)).astype(np.uint32)
    order, stack = [], [root]
    while stack:
        v = stack.pop()
        order.append(v)
        stack.extend(kids[v])
    for v in reversed(order):
        if v >= ntip:
            bits[v] = np.bitwise_or.reduce(bits[kids[v]], axis=0)
    nodes = np.array([v for v in range(ntip, nn) if v != root], dtype=np.int64)
    return bits[nodes]


def plain_replicate(lib, words, full_bits, cells, weights, ancestral_type=1):
    """One replicate through join -> clades -> TransferDisStream.
    Returns (ymin, ysize) over the full-tree clades."""
    cells = np.asarray(cells, dtype=np.int64)
    n = len(cells)
    ncol = full_bits.shape[1]
    edge, _, _ = lib.join_bit(np.ascontiguousarray(words[cells]), weights, ancestral_type)
    xb = clade_bits(edge, n, ncol, tip_map=cells)
    mask = np.zeros(ncol, dtype=np.uint32)
    np.bitwise_or.at(mask, cells // 32, (1 << (cells % 32)).astype(np.uint32))
    yb = full_bits & mask
    ymin, ysize, _, _ = lib.transfer_dis(yb, xb, n)
    return ymin, ysize


def support_counts(ymin, ysize, threshold):
    ymin = np.asarray(ymin, dtype=np.float64)
    ysize = np.asarray(ysize, dtype=np.float64)
    return ((ysize > 0) & (ymin <= threshold * ysize)).sum(axis=0).astype(np.uint32)
