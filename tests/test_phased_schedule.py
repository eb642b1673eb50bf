"""The greedy joins in phases (oracle_join_indel_phased, oracle_join_bit_phased): batched early stale
rescans and two provably independent joins per phase give the same tree and
node states as the sequential joins (oracle_join_indel, oracle_join_bit), in fewer phases.  This
pins the schedule a parallel engine may use against the pinned oracle."""
import numpy as np
import pytest

import oracle as O
from casphy_b200 import synth

CASES = [
    # ncell, nsite, depth, p_edit, nallele, zipf, p_missing, seed, minSize, minRatio, weights
    (300, 64, 9, 0.05, 8, 1.5, 0.1, 1, 0, 2.0, "unit"),
    (1200, 128, 11, 0.03, 16, 1.3, 0.15, 7, 5, 1.5, "unit"),
    (800, 96, 10, 0.05, 12, 1.5, 0.1, 3, 0, 2.0, "f16"),
    (1500, 256, 11, 0.04, 32, 1.5, 0.1, 21, 0, 2.0, "unit"),
]


def _case(c):
    n, nsite, depth, pe, na, z, pm, seed, ms, mr, wk = c
    codes, nstate = synth.regularize(synth.lineage_states(n, nsite, depth, pe, na, z, pm, seed))
    rng = np.random.default_rng(seed)
    w = np.ones((nstate, nsite)) if wk == "unit" else rng.uniform(0.1, 2.0, (nstate, nsite))
    ts = rng.integers(1, 4, n).astype(np.uint32)
    return codes, nstate, w, ts, ms, mr


@pytest.mark.parametrize("c", CASES, ids=[f"{c[0]}cells-{c[10]}-minSize{c[8]}" for c in CASES])
def test_phased_join_gives_the_sequential_tree(c):
    codes, nstate, w, ts, ms, mr = _case(c)
    e0, s0, st0 = O.join_indel(codes, nstate, w, ts, ms, mr)
    seq_phases = int(st0[0] + st0[2])
    for max_batch, pairs in [(1, False), (8, False), (1, True), (8, True)]:
        e1, s1, st1 = O.join_indel_phased(codes, nstate, w, ts, ms, mr, max_batch, pairs)
        assert np.array_equal(e1, e0) and np.array_equal(s1, s0), (max_batch, pairs)
        assert int(st1[2]) == int(st0[2])  # every join made once
        if (max_batch, pairs) == (1, False):
            assert int(st1[3]) == seq_phases and int(st1[0]) == int(st0[0])
        else:
            assert int(st1[3]) < seq_phases
        if not pairs:
            assert int(st1[4]) == 0
    # both rules together: at least a quarter fewer phases on these trees
    assert int(st1[3]) <= 0.75 * seq_phases


def test_phased_join_rejects_a_zero_batch():
    codes, nstate, w, ts, ms, mr = _case(CASES[0])
    with pytest.raises(RuntimeError):
        O.join_indel_phased(codes, nstate, w, ts, ms, mr, 0, True)


BIT_CASES = [(400, 1, 0, "unit"), (400, 1, 1, "float"), (1500, 2, 0, "float"), (1500, 2, 1, "unit")]


@pytest.mark.parametrize("n,seed,atype,wk", BIT_CASES, ids=[f"{c[0]}cells-type{c[2]}-{c[3]}" for c in BIT_CASES])
def test_phased_bit_join_gives_the_sequential_tree(n, seed, atype, wk):
    """The same schedule on the bit model (joinEdgeBitReverse): the rules use
    only records, rescans and strict-improvement updates, which it shares."""
    words = synth.binary_workload(n, 256, 11, 0.03, 0.05, seed=seed)
    w = np.ones(256) if wk == "unit" else np.random.default_rng(seed).uniform(0.2, 3.0, 256)
    e0, s0, st0 = O.join_bit(words, w, atype)
    seq_phases = int(st0[0] + st0[2])
    for max_batch, pairs in [(1, False), (8, True)]:
        e1, s1, st1 = O.join_bit_phased(words, w, atype, max_batch, pairs)
        assert np.array_equal(e1, e0) and np.array_equal(s1, s0), (max_batch, pairs)
        if (max_batch, pairs) == (1, False):
            assert int(st1[3]) == seq_phases
    assert int(st1[3]) <= 0.75 * seq_phases


def test_phased_join_under_a_top2_table():
    """Deciding pairs from a table of each CTA range's top two records (16
    ranges here) gives up a pair only when a range's third best is hidden;
    the tree is still the sequential one."""
    codes, nstate, w, ts, ms, mr = _case(CASES[3])
    e0, s0, _ = O.join_indel(codes, nstate, w, ts, ms, mr)
    e1, s1, st1 = O.join_indel_phased(codes, nstate, w, ts, ms, mr, 8, True, 16)
    assert np.array_equal(e1, e0) and np.array_equal(s1, s0)
    _, _, full = O.join_indel_phased(codes, nstate, w, ts, ms, mr, 8, True, 0)
    assert int(full[5]) == 0  # with every record visible nothing is given up
    assert int(st1[4]) > 0 and int(st1[5]) < int(st1[4])
