"""Batched bootstrap (casphy_bootstrap_bit) against the plain pipeline run
one replicate at a time: identical replicate trees, identical per-replicate
TransferDisStream values and identical support counts."""
import numpy as np
import pytest

import oracle as O
from casphy_b200 import bootstrap as B
from casphy_b200 import synth

pytestmark = pytest.mark.gpu


def _case(ncell, nbin, nrep, nmin, nmax, seed):
    words = synth.binary_workload(ncell, nbin * 32, 12, 0.03, 0.05, seed=seed)
    full_edge, _, _ = O.join_bit(words, None, 1)
    off, cells, w = B.make_replicates(ncell, nbin * 32, nrep, nmin, nmax, seed=seed + 1)
    return words, full_edge, off, cells, w


def _raw_to_clades(raw, n, cells, ncol):
    e = raw.reshape(-1, 2)
    return B.clade_bits(e, n, ncol, tip_map=cells)


@pytest.mark.parametrize("ncell,nbin,nrep,nmin,nmax,seed", [
    (300, 2, 9, 2, 300, 1),
    (900, 4, 24, 150, 900, 2),
    (2500, 16, 6, 2000, 2500, 3),
])
def test_batched_equals_sequential(gpu_lib, ncell, nbin, nrep, nmin, nmax, seed):
    words, full_edge, off, cells, w = _case(ncell, nbin, nrep, nmin, nmax, seed)
    thr = 0.05
    got = gpu_lib.bootstrap_bit(words, full_edge, off, cells, w, threshold=thr, raw_edges=True)
    ncol = (ncell + 31) // 32
    full_bits = B.clade_bits(full_edge, ncell, ncol)
    ymin = np.zeros_like(got["ymin"])
    ysize = np.zeros_like(got["ysize"])
    for r in range(nrep):
        c = cells[off[r]:off[r + 1]]
        ymin[r], ysize[r] = B.plain_replicate(gpu_lib, words, full_bits, c, w[r])
        # the replicate tree is the tree of the single join
        edge, _, _ = gpu_lib.join_bit(np.ascontiguousarray(words[c]), w[r], 1)
        a = B.clade_bits(edge, len(c), ncol, tip_map=c)
        b = _raw_to_clades(got["raw_edges"][r], len(c), c, ncol)
        assert np.array_equal(np.unique(a, axis=0), np.unique(b, axis=0)), f"replicate {r} tree differs"
    assert np.array_equal(got["ymin"], ymin)
    assert np.array_equal(got["ysize"], ysize)
    assert np.array_equal(got["support"], B.support_counts(ymin, ysize, thr))
    assert got["stats"]["graph"] == 1  # the pass ran as one captured CUDA graph
    st = got["stats"]
    assert st["join_ms"] > 0 and st["total_ms"] >= st["prep_ms"] + st["join_ms"]  # event nodes time the graph
    if nmin >= 2000:
        # the same replicates joined by groups of 4 CTAs give the same trees and values
        import os
        os.environ["CASPHY_BS_GROUP"] = "4"
        try:
            grouped = gpu_lib.bootstrap_bit(words, full_edge, off, cells, w, threshold=thr, raw_edges=True)
        finally:
            del os.environ["CASPHY_BS_GROUP"]
        assert grouped["stats"]["max_ctas_per_rep"] == 4
        assert np.array_equal(grouped["ymin"], ymin) and np.array_equal(grouped["ysize"], ysize)
        for r in range(nrep):
            assert np.array_equal(grouped["raw_edges"][r], got["raw_edges"][r])


def test_oracle_pipeline_agrees_on_a_replicate(gpu_lib):
    words, full_edge, off, cells, w = _case(400, 2, 3, 100, 400, 7)
    got = gpu_lib.bootstrap_bit(words, full_edge, off, cells, w)
    full_bits = B.clade_bits(full_edge, 400, (400 + 31) // 32)
    for r in range(3):
        c = cells[off[r]:off[r + 1]]
        ymin, ysize = B.plain_replicate(O, words, full_bits, c, w[r])
        assert np.array_equal(got["ymin"][r], ymin) and np.array_equal(got["ysize"][r], ysize)


def test_bad_replicates_raise(gpu_lib):
    words, full_edge, off, cells, w = _case(200, 2, 2, 50, 100, 9)
    bad = cells.copy()
    bad[1] = bad[0]
    with pytest.raises(gpu_lib.CasphyError):
        gpu_lib.bootstrap_bit(words, full_edge, off, bad, w)
    with pytest.raises(gpu_lib.CasphyError):
        gpu_lib.bootstrap_bit(words, full_edge, off, cells, w + 0.5)


def test_weights_beyond_the_row_use_planes(gpu_lib):
    """Weights that sum past the site count (here doubled multiplicities)
    cannot be laid out as repeated columns; the bit-plane path must give the
    plain pipeline's values too."""
    words, full_edge, off, cells, w = _case(600, 4, 5, 200, 600, 9)
    w2 = 2 * w
    got = gpu_lib.bootstrap_bit(words, full_edge, off, cells, w2)
    full_bits = B.clade_bits(full_edge, 600, (600 + 31) // 32)
    for r in range(5):
        c = cells[off[r]:off[r + 1]]
        ymin, ysize = B.plain_replicate(gpu_lib, words, full_bits, c, w2[r])
        assert np.array_equal(got["ymin"][r], ymin) and np.array_equal(got["ysize"][r], ysize)
