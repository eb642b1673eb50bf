"""The oracle's column-scan engine for the indel join (the one that makes
the 200,000-cell oracle tree feasible) writes the same trees, node states
and join statistics as its row-wise engine, which is pinned byte for byte to
the reference joinEdgeIndel binaries."""
import contextlib
import ctypes
import json
import os

import numpy as np
import pytest

import golden_check
import oracle as O
from casphy_b200 import synth

HASHES = os.path.join(os.path.dirname(__file__), "golden", "scale_hashes.json")


@contextlib.contextmanager
def colscan():
    flag = ctypes.c_int.in_dll(O.lib(), "oracle_indel_colscan")
    flag.value = 1
    try:
        yield
    finally:
        flag.value = 0


def test_colscan_matches_reference_tools(golden):
    cases, ref = golden
    with colscan():
        bad = [m for _, ok, m in golden_check.iter_checks(cases, ref, kinds={"ji"}) if not ok]
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("seed,ncell,nsite,nallele,pm,weights,minsize", [
    (1, 2500, 193, 40, 0.1, "unit", False),
    (2, 1600, 86, 12, 0.3, "int", False),
    (3, 2200, 222, 60, 0.1, "unit", True),
    (4, 900, 520, 250, 0.15, "int", True),
    (5, 5200, 64, 8, 0.05, "unit", False),   # several compactions of the site-major copy
    (6, 3, 5, 2, 0.0, "unit", False),
])
def test_colscan_matches_rowwise(seed, ncell, nsite, nallele, pm, weights, minsize):
    rng = np.random.default_rng(seed)
    raw = synth.lineage_states(ncell, nsite, 13, 0.05, nallele, 1.4, pm, seed=seed)
    codes, ns = synth.regularize(raw)
    w = np.ones((ns, nsite)) if weights == "unit" else rng.integers(0, 4, size=(ns, nsite)).astype(float)
    kw = dict(tip_size=rng.integers(1, 30, ncell), min_size=8, min_ratio=1.5) if minsize else {}
    want = O.join_indel(codes, ns, w, **kw)
    with colscan():
        got = O.join_indel(codes, ns, w, **kw)
    for g, x in zip(got, want):
        assert np.array_equal(g, x)


def test_colscan_leaves_fractional_weights_to_binary16():
    """Non-integer weights keep the binary16 emulation under the flag."""
    rng = np.random.default_rng(9)
    raw = synth.lineage_states(400, 40, 10, 0.06, 10, 1.2, 0.05, seed=9)
    codes, ns = synth.regularize(raw)
    w = rng.uniform(0.01, 5.0, size=(ns, 40))
    want = O.join_indel(codes, ns, w)
    with colscan():
        got = O.join_indel(codes, ns, w)
    for g, x in zip(got, want):
        assert np.array_equal(g, x)


def test_scale_hash_20k_prefix_reproduces():
    """The committed 20,000-cell C5 prefix hash is what the oracle writes
    today (the generator and the oracle have not drifted)."""
    import hashlib
    import bench
    ref = json.load(open(HASHES))["c5_20k"]
    codes, ns, w = bench.gen_workload(20_000)
    with colscan():
        e, s, st = O.join_indel(codes, ns, w)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()  # noqa: E731
    assert sha(e) == ref["edge_sha256"] and sha(s) == ref["state_sha256"]
    assert int(st[0]) == ref["stale_recomputes"] and int(st[1]) == ref["pair_scores"]
