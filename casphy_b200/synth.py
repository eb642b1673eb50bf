"""Seeded synthetic inputs with the shapes of the benchmark workloads.

No public dataset is involved: every matrix is simulated from a seed so tests,
the bench and the golden fixtures see identical bytes.

Lineage model (indel and base-editor matrices): a complete binary division
tree of ``depth`` generations is grown from one unedited root cell; ``ncell``
of its ``2**depth`` leaves are sampled without replacement and shuffled.  On
every branch (one generation) each still-unedited site edits with
probability ``p_edit``; an indel site then takes an allele drawn from a Zipf
law over ``nallele`` alleles (weight k**-s), a base-editor site becomes 1.
Edits are irreversible.  Afterwards a fraction ``p_missing`` of entries is
set missing uniformly at random.  Only lineages with sampled descendants are
simulated, site block by site block, so 200,000 x 1,024 fits in host memory.

DNA model: a Yule (pure-birth) topology with Exponential(mean) branch
lengths and HKY85 substitutions (``kappa``, base frequencies ``pi``), then
gaps set uniformly at random.
"""
from __future__ import annotations

import numpy as np

from . import formats


def _zipf_p(nallele: int, s: float) -> np.ndarray:
    k = np.arange(1, nallele + 1, dtype=np.float64)
    p = k ** (-s)
    return p / p.sum()


def _lineage_plan(ncell: int, depth: int, rng: np.random.Generator):
    total = 1 << depth
    if ncell > total:
        raise ValueError(f"ncell={ncell} exceeds 2**depth={total}")
    leaves = np.sort(rng.choice(total, size=ncell, replace=False)).astype(np.int64)
    gens = []
    prev = np.zeros(1, dtype=np.int64)
    for g in range(1, depth + 1):
        cur = np.unique(leaves >> (depth - g))
        parent = np.searchsorted(prev, cur >> 1)
        gens.append(parent)
        prev = cur
    leaf_pos = np.searchsorted(prev, leaves)
    return gens, leaf_pos


def lineage_states(ncell: int, nsite: int, depth: int, p_edit: float,
                   nallele: int, zipf_s: float, p_missing: float, seed: int,
                   block: int = 64) -> np.ndarray:
    """Raw CRISPR states: int32 (ncell, nsite), -1 missing, 0 unedited,
    1..nallele allele.  nallele == 1 gives a 0/1 base-editor matrix."""
    rng = np.random.default_rng(seed)
    gens, leaf_pos = _lineage_plan(ncell, depth, rng)
    perm = rng.permutation(ncell)
    zp = _zipf_p(nallele, zipf_s) if nallele > 1 else None
    dtype = np.int16 if nallele < 32000 else np.int32
    out = np.empty((ncell, nsite), dtype=np.int32)
    for s0 in range(0, nsite, block):
        nb = min(block, nsite - s0)
        state = np.zeros((1, nb), dtype=dtype)
        for parent in gens:
            child = state[parent]
            hit = (rng.random(child.shape, dtype=np.float32) < p_edit) & (child == 0)
            nh = int(hit.sum())
            if nh:
                if zp is None:
                    child[hit] = 1
                else:
                    child[hit] = rng.choice(nallele, size=nh, p=zp).astype(dtype) + 1
            state = child
        out[:, s0:s0 + nb] = state[leaf_pos]
    out = out[perm]
    if p_missing > 0:
        miss = rng.random(out.shape, dtype=np.float32) < p_missing
        out[miss] = -1
    return out


def regularize(mat: np.ndarray) -> tuple[np.ndarray, int]:
    """R's ``regularize.mat(mat, mat)`` followed by ``+1L`` (R/CasPhy_functions
    .R:435-441, 610): per column, states are ranked within
    sort(unique(c(col, -1, 0))), giving 0 missing, 1 unedited, 2.. alleles.
    Returns (u32 codes, nState) with nState the largest allele count of any
    column (the row count of R's weight matrix, :583-585)."""
    m = np.asarray(mat)
    out = np.empty(m.shape, dtype=np.uint32)
    nstate = 1
    for i in range(m.shape[1]):
        col = m[:, i]
        u = np.unique(np.concatenate([col, np.array([-1, 0], dtype=col.dtype)]))
        out[:, i] = np.searchsorted(u, col).astype(np.uint32)
        nstate = max(nstate, len(u) - 2)
    return out, nstate


def indel_workload(ncell: int, nsite: int, depth: int, p_edit: float, nallele: int,
                   zipf_s: float, p_missing: float, seed: int):
    """Codes (u32, ncell x nsite), nState and unit weights (nState x nsite)."""
    raw = lineage_states(ncell, nsite, depth, p_edit, nallele, zipf_s, p_missing, seed)
    codes, nstate = regularize(raw)
    w = np.ones((nstate, nsite), dtype=np.float64)
    return codes, nstate, w


def binary_workload(ncell: int, nsite: int, depth: int, p_edit: float,
                    p_missing: float, seed: int):
    """Packed base-editor rows (u32, ncell x nsite/32); missing written as 0."""
    raw = lineage_states(ncell, nsite, depth, p_edit, 1, 1.0, p_missing, seed)
    bits = raw == 1
    return formats.pack_bits(bits)


# ---------------------------------------------------------------------------
# DNA (HKY85)

def hky85_P(t: float, kappa: float, pi: np.ndarray) -> np.ndarray:
    """HKY85 transition matrix, state order A, C, G, T, rate matrix scaled to
    one expected substitution per unit time (Hasegawa, Kishino & Yano 1985)."""
    Q = hky85_Q(kappa, pi)
    w, V = np.linalg.eig(Q)
    Vi = np.linalg.inv(V)
    return np.real(V @ np.diag(np.exp(w * t)) @ Vi)


def hky85_Q(kappa: float, pi: np.ndarray) -> np.ndarray:
    pi = np.asarray(pi, dtype=np.float64)
    Q = np.tile(pi, (4, 1))
    for i, j in ((0, 2), (2, 0), (1, 3), (3, 1)):  # transitions A<->G, C<->T
        Q[i, j] *= kappa
    np.fill_diagonal(Q, 0.0)
    np.fill_diagonal(Q, -Q.sum(axis=1))
    scale = -np.dot(pi, np.diag(Q))
    return Q / scale


def yule_tree(ntip: int, mean_bl: float, rng: np.random.Generator):
    """Random Yule topology.  Returns (parent, child, length) over 2*ntip-2
    edges listed parent-before-child; tips are 0..ntip-1, the root is ntip."""
    nn = 2 * ntip - 1
    parent_of = np.full(nn, -1, dtype=np.int64)
    leaves = [0]
    next_id = 1
    while len(leaves) < ntip:
        k = int(rng.integers(len(leaves)))
        v = leaves[k]
        parent_of[next_id] = v
        parent_of[next_id + 1] = v
        leaves[k] = next_id
        leaves.append(next_id + 1)
        next_id += 2
    is_leaf = np.zeros(nn, dtype=bool)
    is_leaf[np.array(leaves)] = True
    lab = np.empty(nn, dtype=np.int64)
    lab[np.array(leaves)] = np.arange(ntip)
    lab[~is_leaf] = ntip + np.arange(int((~is_leaf).sum()))
    ch = np.arange(1, nn)  # growth ids: a parent is always created first
    par = lab[parent_of[ch]]
    length = rng.exponential(mean_bl, size=len(ch))
    return par, lab[ch], length


def hky85_alignment(ntip: int, ncol: int, kappa: float, pi, mean_bl: float,
                    p_gap: float, seed: int):
    """Simulated alignment as uint8 states 0..3 (A,C,G,T) or 4 (gap), plus the
    tree (parent, child, length) it was simulated on."""
    rng = np.random.default_rng(seed)
    pi = np.asarray(pi, dtype=np.float64)
    par, ch, bl = yule_tree(ntip, mean_bl, rng)
    nn = 2 * ntip - 1
    seq = np.empty((nn, ncol), dtype=np.uint8)
    seq[ntip] = rng.choice(4, size=ncol, p=pi)
    for e in range(len(ch)):
        cum = np.cumsum(hky85_P(bl[e], kappa, pi), axis=1)
        u = rng.random(ncol)
        seq[ch[e]] = np.minimum((u[:, None] > cum[seq[par[e]]]).sum(axis=1), 3)
    tips = seq[:ntip].copy()
    if p_gap > 0:
        tips[rng.random(tips.shape) < p_gap] = 4
    return tips, (par, ch, bl)


def dna_to_fasta2bin(states: np.ndarray):
    """States 0..3 (A,C,G,T) / 4 gap -> fasta2bin codes after dropping
    invariant columns (cu/fasta2bin.cu:47-99): returns (u32 words, kept mask)."""
    lut = np.array([0x01, 0x04, 0x08, 0x02, 0x10], dtype=np.uint8)  # A C G T -
    codes = lut[states]
    # a column is variable if some base count is >0 and < number of rows seen
    # (a gap counts as a row seen but adds to no base count)
    n = states.shape[0]
    var = np.zeros(states.shape[1], dtype=bool)
    for b in range(4):
        cnt = (states == b).sum(axis=0)
        var |= (cnt > 0) & (cnt < n)
    return formats.encode_dna_codes(codes[:, var]), var


def dna_nibbles(states: np.ndarray) -> np.ndarray:
    """States 0..3 (A,C,G,T) / 4 gap -> the fasta2bin 4-bit nibble per site
    as u32 (A=1, T=2, C=4, G=8; a gap has an empty nibble = missing)."""
    lut = np.array([0x1, 0x4, 0x8, 0x2, 0x0], dtype=np.uint32)
    return lut[states]


def edit_alignment(ntip: int, nsite: int, rate: float, nallele: int, zipf_s: float,
                   mean_bl: float, p_missing: float, seed: int):
    """Irreversible CRISPR edits simulated on a Yule tree: the root is
    unedited, along an edge of length t an unedited site is edited with
    probability 1 - exp(-rate t) into allele a with Zipf(zipf_s) frequency,
    and edited sites never change.  Returns .tbmat-coded tips (u32: 0
    missing, 1 unedited, a+1 allele a) and the tree (parent, child, length)."""
    rng = np.random.default_rng(seed)
    par, ch, bl = yule_tree(ntip, mean_bl, rng)
    nn = 2 * ntip - 1
    q = 1.0 / np.arange(1, nallele + 1) ** zipf_s
    q /= q.sum()
    st = np.zeros((nn, nsite), dtype=np.int64)
    for e in range(len(ch)):
        s = st[par[e]].copy()
        hit = (s == 0) & (rng.random(nsite) < -np.expm1(-rate * bl[e]))
        s[hit] = 1 + rng.choice(nallele, size=int(hit.sum()), p=q)
        st[ch[e]] = s
    codes = (st[:ntip] + 1).astype(np.uint32)
    codes[rng.random(codes.shape) < p_missing] = 0
    return codes, (par, ch, bl)


def lineage_clades(ncell: int, depth: int, seed: int):
    """Clades of the true division tree behind ``lineage_states(ncell, ...,
    depth, ..., seed)``: for every generation, the sets of sampled cells
    sharing an ancestor there, without duplicates (unary lineages) and
    without the trivial sets (one cell, all cells).  Rows are tip bitsets of
    (ncell + 31) // 32 u32 words over the output row order."""
    rng = np.random.default_rng(seed)
    total = 1 << depth
    leaves = np.sort(rng.choice(total, size=ncell, replace=False)).astype(np.int64)
    perm = rng.permutation(ncell)
    leaf_of_row = leaves[perm]
    ncol = (ncell + 31) // 32
    seen, rows = set(), []
    word = np.arange(ncell) // 32
    bit = (1 << (np.arange(ncell) % 32)).astype(np.uint32)
    for g in range(1, depth + 1):
        pref = leaf_of_row >> (depth - g)
        order = np.argsort(pref, kind="stable")
        bounds = np.flatnonzero(np.diff(pref[order])) + 1
        for grp in np.split(order, bounds):
            if len(grp) <= 1 or len(grp) >= ncell:
                continue
            key = grp.tobytes()
            if key in seen:
                continue
            seen.add(key)
            r = np.zeros(ncol, dtype=np.uint32)
            np.bitwise_or.at(r, word[grp], bit[grp])
            rows.append(r)
    return np.array(rows, dtype=np.uint32).reshape(-1, ncol)


def neighbour_lists(ntip, seed):
    """Symmetric, ascending neighbour lists: tips in random clusters of 3-40,
    pairs inside a cluster linked with probability 0.6, each tip linked to one
    random tip elsewhere, and half the tips listing themselves (a radius list
    holds its own row when the row's self score reaches the radius).
    Returns (counts u32[ntip], concatenated idx u32)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(ntip)
    a, b = [], []
    pos = 0
    while pos < ntip:
        size = int(rng.integers(3, 41))
        members = perm[pos:pos + size]
        pos += size
        m = len(members)
        if m > 1:
            iu, ju = np.triu_indices(m, 1)
            keep = rng.random(len(iu)) < 0.6
            a.append(members[iu[keep]])
            b.append(members[ju[keep]])
    x = rng.integers(0, ntip, ntip)
    a.append(np.arange(ntip))
    b.append(x)
    a, b = np.concatenate(a), np.concatenate(b)
    ok = a != b
    a, b = a[ok], b[ok]
    selfs = np.flatnonzero(rng.random(ntip) < 0.5)
    rows = np.concatenate([a, b, selfs])
    cols = np.concatenate([b, a, selfs])
    key = np.unique(rows.astype(np.int64) * ntip + cols)
    rows, cols = key // ntip, key % ntip
    counts = np.bincount(rows, minlength=ntip).astype(np.uint32)
    return counts, cols.astype(np.uint32)
