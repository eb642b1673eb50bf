"""The GPU joins at the benchmark's full sizes against the CPU oracle.

The oracle's trees for these workloads are stored as sha256 digests of the
edge list and the node-state rows (tests/golden/scale_hashes.json, written
by tests/golden/make_scale_hashes.py, which runs oracle/oracle.c on the same
seeded inputs).  Each test builds the input, runs the join through the C ABI
and compares digests, so a single differing byte anywhere in the 200,000-cell
tree fails it."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HASHES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "scale_hashes.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


@pytest.mark.parametrize("case,ncell", [("c5_20k", 20_000), ("c5_50k", 50_000), ("c5_200k", None)])
def test_c5_matches_oracle(gpu_lib, case, ncell):
    """joinEdgeIndel on the 200,000-cell x 1,024-site generator: its first
    20,000 and 50,000 cells, and the whole headline workload."""
    import bench
    ref = HASHES[case]
    codes, ns, w = bench.gen_workload(ncell)
    e, s, st = gpu_lib.join_indel(codes, ns, w)
    assert st["joins"] == ref["joins"]
    assert sha(e) == ref["edge_sha256"], "edge list differs from the oracle's"
    assert sha(s) == ref["state_sha256"], "node states differ from the oracle's"


@pytest.mark.parametrize("atype", [1, 0])
def test_c2_bit_join_matches_oracle(gpu_lib, atype):
    """joinEdgeBitReverse on the full 10,000 x 512 base-editor matrix, both
    ancestral rules."""
    from casphy_b200 import synth
    ref = HASHES[f"c2_bit_t{atype}"]
    words = synth.binary_workload(10_000, 512, 16, 0.03, 0.05, seed=23)
    e, s, st = gpu_lib.join_bit(words, None, atype)
    assert st["joins"] == ref["joins"]
    assert sha(e) == ref["edge_sha256"]
    assert sha(s) == ref["state_sha256"]
