"""joinEdgeIndel on the GPU (through the C ABI) against the reference bytes
and the CPU oracle."""
import numpy as np
import pytest

import golden_check
import oracle as O
from casphy_b200 import synth

pytestmark = pytest.mark.gpu


def test_golden_indel_joins(golden, gpu_lib, scan_path):
    cases, ref = golden
    bad = [m for name, ok, m in golden_check.iter_checks(cases, ref, impl=_Impl(gpu_lib), kinds={"ji"})
           if not ok]
    assert not bad, "\n".join(bad)


class _Impl:
    """Adapter so golden_check drives the GPU join and the oracle for the rest."""
    def __init__(self, L):
        self.L = L

    def join_indel(self, *a, **k):
        return self.L.join_indel(*a, **k)

    def __getattr__(self, name):
        return getattr(O, name)


@pytest.fixture(params=["bits", "dense"])
def scan_path(request, monkeypatch):
    """Run a test once per indel scan: allele bitsets (default) and the
    column-major code scan."""
    monkeypatch.setenv("CASPHY_INDEL_SCAN", request.param)
    return request.param


@pytest.mark.parametrize("seed,ncell,nsite,nallele,pm", [
    (101, 700, 96, 24, 0.1), (102, 1500, 40, 8, 0.3), (103, 64, 500, 200, 0.0), (104, 5000, 64, 16, 0.15)])
def test_random_indel_vs_oracle(gpu_lib, scan_path, stale_batch, seed, ncell, nsite, nallele, pm):
    raw = synth.lineage_states(ncell, nsite, 13, 0.05, nallele, 1.4, pm, seed=seed)
    codes, ns = synth.regularize(raw)
    w = np.ones((ns, nsite))
    e1, s1, st1 = gpu_lib.join_indel(codes, ns, w)
    assert st1["scan_path"] == (1 if scan_path == "bits" else 0)
    e0, s0, st0 = O.join_indel(codes, ns, w)
    assert np.array_equal(e1, e0)
    assert np.array_equal(s1, s0)
    if stale_batch == 1:
        # one rescan per phase: the reference loop's own counts
        assert st1["stale_recomputes"] == st0[0]
        assert st1["pair_scores"] == st0[1]
    else:
        # early rescans add rows, never remove one
        assert st1["stale_recomputes"] >= st0[0]


def test_half_path_random_weights(gpu_lib):
    rng = np.random.default_rng(7)
    raw = synth.lineage_states(900, 48, 11, 0.06, 10, 1.2, 0.05, seed=77)
    codes, ns = synth.regularize(raw)
    w = rng.uniform(0.01, 5.0, size=(ns, 48))
    e1, s1, st1 = gpu_lib.join_indel(codes, ns, w)
    assert st1["int_path"] == 0
    e0, s0, _ = O.join_indel(codes, ns, w)
    assert np.array_equal(e1, e0) and np.array_equal(s1, s0)


def test_integer_weights_and_min_size(gpu_lib, scan_path):
    rng = np.random.default_rng(8)
    raw = synth.lineage_states(800, 64, 11, 0.05, 12, 1.3, 0.1, seed=78)
    codes, ns = synth.regularize(raw)
    w = rng.integers(0, 4, size=(ns, 64)).astype(float)
    tip = rng.integers(1, 40, size=800)
    e1, s1, st1 = gpu_lib.join_indel(codes, ns, w, tip, 10, 1.5)
    assert st1["int_path"] == 1
    e0, s0, _ = O.join_indel(codes, ns, w, tip, 10, 1.5)
    assert np.array_equal(e1, e0) and np.array_equal(s1, s0)


def test_single_cell(gpu_lib):
    codes = np.array([[2, 1, 0, 3]], dtype=np.uint32)
    e, s, _ = gpu_lib.join_indel(codes, 2, np.ones((2, 4)))
    assert e.shape == (0, 2)
    assert np.array_equal(s, codes)


def test_rejects_codes_beyond_nstate(gpu_lib):
    codes = np.array([[2, 9], [3, 1]], dtype=np.uint32)
    with pytest.raises(gpu_lib.CasphyError) as ei:
        gpu_lib.join_indel(codes, 2, np.ones((2, 2)))
    assert ei.value.status == 2


def test_large_compaction_properties(gpu_lib, scan_path, stale_batch):
    """6,000 cells: exercises slot compaction; checked against the oracle."""
    raw = synth.lineage_states(6000, 96, 16, 0.03, 64, 1.3, 0.15, seed=55)
    codes, ns = synth.regularize(raw)
    w = np.ones((ns, 96))
    e1, s1, st1 = gpu_lib.join_indel(codes, ns, w)
    assert st1["compactions"] > 0
    e0, s0, st0 = O.join_indel(codes, ns, w)
    assert np.array_equal(e1, e0) and np.array_equal(s1, s0)


@pytest.mark.parametrize("name", ["w3k_unit", "w2k_int", "w1500_half"])
def test_reference_digests_at_1024_sites(gpu_lib, scan_path, name):
    """The GPU join (and nodeKeepIndel on the unit case) against the files
    the reference tools built with MAXCOL 1024 wrote for the same inputs."""
    import json
    import make_wide_golden as W
    ref = json.load(open(W.OUT))[name]
    codes, ns, w, out = W.case_inputs(name)
    e, s, _ = gpu_lib.join_indel(codes, ns, w)
    assert W.sha_bytes(W.edge2_file_bytes(e)) == ref["edge2"]
    assert W.sha_bytes(W.node_state2_file_bytes(s, *codes.shape)) == ref["nodeState2"]
    for cut in (1, 2):
        if f"retain{cut}" in ref:
            assert W.retain_digest(gpu_lib.node_keep(s, e, out, cut)) == ref[f"retain{cut}"]


def test_stale_batches_cut_phases(gpu_lib, monkeypatch):
    """Batched rescans: the same tree in fewer phases than one rescan per
    phase (5,000 cells of the 200k generator's settings)."""
    raw = synth.lineage_states(5000, 256, 20, 0.02, 256, 1.3, 0.15, seed=57)
    codes, ns = synth.regularize(raw)
    w = np.ones((ns, 256))
    res = {}
    for b in ("1", "8"):
        monkeypatch.setenv("CASPHY_STALE_BATCH", b)
        res[b] = gpu_lib.join_indel(codes, ns, w)
    (e1, s1, st1), (e8, s8, st8) = res["1"], res["8"]
    assert np.array_equal(e1, e8) and np.array_equal(s1, s8)
    assert st8["phases"] < 0.9 * st1["phases"]
