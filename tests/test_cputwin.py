"""The reference's CPU implementations of the hot path (greedyJoinEdge2,
greedyJoinEdgeBitReverse, radiusWeightedParallel, radiusWeightedDNAParallel
of src/functions.cpp, compiled into oracle/_ref/libcputwin_ref.so) against
the oracle on seeded inputs.

The CPU joins are a different algorithm from the CUDA joins the oracle
restates (an N x N score cache with stale rows rescanned over higher node
indices only, against lazy per-row maxima rescanned over all live rows), so
they are compared by the clades of the trees they build; on these inputs the
two give the same tree.  The radius functions share the criterion (shared
weight >= radius) and are compared list for list."""
import os

import numpy as np
import pytest

import cputwin as T
import oracle as O
from casphy_b200 import synth

pytestmark = pytest.mark.skipif(not T.available(), reason="oracle/_ref/libcputwin_ref.so not built (make -C oracle ref)")


def clades(par, ch, ntip):
    kids = {}
    for p, c in zip(np.asarray(par).tolist(), np.asarray(ch).tolist()):
        kids.setdefault(p, []).append(c)
    allc = set(np.asarray(ch).tolist())
    root = [p for p in kids if p not in allc]
    assert len(root) == 1
    order, st = [], [root[0]]
    while st:
        v = st.pop()
        order.append(v)
        st.extend(kids.get(v, []))
    memo, out = {}, set()
    for v in reversed(order):
        if v < ntip:
            memo[v] = frozenset([v])
        else:
            s = frozenset().union(*[memo[c] for c in kids[v]])
            memo[v] = s
            out.add(s)
    assert len(memo) == 2 * ntip - 1 and len(out) == ntip - 1
    return out


def bitmap_lists(bm, n):
    bits = np.unpackbits(bm.view(np.uint8), axis=1, bitorder="little")[:, :n]
    return np.concatenate([np.nonzero(r)[0] for r in bits]).astype(np.uint32)


def test_indel_join_same_tree():
    """1,024 cells x 256 sites, 64 alleles Zipf(1.5), depth 12, p_edit 0.04,
    10% missing, unit weights."""
    codes, ns, w = synth.indel_workload(1024, 256, 12, 0.04, 64, 1.5, 0.10, 1)
    e = T.greedy_join_edge2(codes, ns, w)
    assert e.shape == (3 + 256, 2 * 1024 - 1)
    # the last column carries the root state only
    eo, _, _ = O.join_indel(codes, ns, w)
    assert clades(e[0, :-1], e[1, :-1], 1024) == clades(eo[:, 0], eo[:, 1], 1024)


@pytest.mark.parametrize("ancestral_type", [0, 1])
def test_bit_join_same_tree(ancestral_type):
    words = synth.binary_workload(1000, 512, 16, 0.03, 0.05, seed=7)
    e = T.greedy_join_edge_bit(words, ancestral_type=ancestral_type)
    eo, _, _ = O.join_bit(words, ancestral_type=ancestral_type)
    assert clades(e[0], e[1], 1000) == clades(eo[:, 0], eo[:, 1], 1000)


def test_radius_bit_same_lists():
    n = 1500
    words = synth.binary_workload(n, 512, 16, 0.03, 0.05, seed=23)
    c, bm = T.radius_weighted_rows(words, 4, 0, n, os.cpu_count() or 1)
    oc, oi = O.radius_bit(np.ascontiguousarray(words.T), np.ones(512), 4)
    assert np.array_equal(c, oc) and np.array_equal(bitmap_lists(bm, n), oi)
    # a row range is the same rows of the full result
    c2, bm2 = T.radius_weighted_rows(words, 4, 700, 900, 2)
    assert np.array_equal(c2, c[700:900]) and np.array_equal(bm2, bm[700:900])


def test_radius_dna_same_lists():
    n = 1200
    states, _ = synth.hky85_alignment(n, 1000, 4.0, [0.3, 0.2, 0.2, 0.3], 0.01, 0.02, seed=13)
    raw, var = synth.dna_to_fasta2bin(states)
    radius = int(var.sum()) - 60
    c, bm = T.radius_weighted_dna_rows(raw, radius, 0, n, os.cpu_count() or 1)
    oc, oi = O.radius_dna(raw, radius)
    assert oc.sum() > n  # neighbours beyond each row itself
    assert np.array_equal(c, oc) and np.array_equal(bitmap_lists(bm, n), oi)
