"""nodeKeep, radius search, tryRadius and TransferDis on the GPU against the
reference bytes (golden fixtures) and the oracle (random and edge cases)."""
import numpy as np
import pytest

import golden_check
import oracle as O
from casphy_b200 import formats, synth

pytestmark = pytest.mark.gpu


class _GpuAll:
    """GPU implementation for every tool except the joins, which come from the
    oracle so these tests isolate the tools under test."""
    def __init__(self, L):
        self.L = L

    def __getattr__(self, name):
        if name in ("join_indel", "join_bit"):
            return getattr(O, name)
        return getattr(self.L, name)


@pytest.mark.parametrize("kinds", [{"ji"}, {"jb"}, {"dna"}, {"td"}])
def test_golden_tools(golden, gpu_lib, kinds):
    cases, ref = golden
    bad = [m for name, ok, m in golden_check.iter_checks(cases, ref, impl=_GpuAll(gpu_lib), kinds=kinds)
           if not ok and not name.startswith(("ji/", "jb/"))]
    assert not bad, "\n".join(bad)


def test_node_keep_random(gpu_lib):
    raw = synth.lineage_states(900, 96, 11, 0.05, 16, 1.3, 0.1, seed=301)
    codes, ns = synth.regularize(raw)
    e, s, _ = O.join_indel(codes[:700], ns, np.ones((ns, 96)))
    for cut in (0, 1, 2, 5):
        assert np.array_equal(gpu_lib.node_keep(s, e, codes[700:], cut), O.node_keep(s, e, codes[700:], cut))
    # no out-group rows: every tested node is kept
    assert np.array_equal(gpu_lib.node_keep(s, e, np.zeros((0, 96), np.uint32), 3),
                          O.node_keep(s, e, np.zeros((0, 96), np.uint32), 3))


@pytest.mark.parametrize("radius", [1, 5, 9, 0, -2])
def test_radius_bit_random(gpu_lib, radius):
    words = synth.binary_workload(1500, 200, 12, 0.05, 0.05, seed=302)  # ntip not a multiple of 32
    bmat = np.ascontiguousarray(words.T)
    w = np.ones(bmat.shape[0] * 32)
    c1, i1 = gpu_lib.radius_bit(bmat, w, radius)
    c0, i0 = O.radius_bit(bmat, w, radius)
    assert np.array_equal(c1, c0) and np.array_equal(i1, i0)
    q = np.array([0, 1, 1499, 700, 700], dtype=np.uint32)
    assert np.array_equal(gpu_lib.try_radius_bit(bmat, w, radius, q), O.try_radius_bit(bmat, w, radius, q))


def test_radius_bit_float_weights(gpu_lib):
    rng = np.random.default_rng(3)
    words = synth.binary_workload(700, 128, 12, 0.05, 0.05, seed=303)
    bmat = np.ascontiguousarray(words.T)
    w = rng.uniform(0.1, 2.0, size=128)
    c1, i1 = gpu_lib.radius_bit(bmat, w, 4)
    c0, i0 = O.radius_bit(bmat, w, 4)
    assert np.array_equal(c1, c0) and np.array_equal(i1, i0)


@pytest.mark.parametrize("radius", [0, 150, 300, 390])
def test_radius_dna_random(gpu_lib, radius):
    tips, _ = synth.hky85_alignment(900, 500, 4.0, [0.3, 0.2, 0.2, 0.3], 0.01, 0.02, seed=304)
    raw, _ = synth.dna_to_fasta2bin(tips)
    c1, i1 = gpu_lib.radius_dna(raw, radius)
    c0, i0 = O.radius_dna(raw, radius)
    assert np.array_equal(c1, c0) and np.array_equal(i1, i0)
    q = np.arange(0, 900, 37, dtype=np.uint32)
    assert np.array_equal(gpu_lib.try_radius_dna(raw, radius, q), O.try_radius_dna(raw, radius, q))


def test_radius_dna_ambiguity_codes(gpu_lib):
    """IUPAC ambiguity codes (several nibble bits) intersect any base they
    include; 1,001 columns leave a ragged last block of positions."""
    tips, _ = synth.hky85_alignment(700, 1001, 4.0, [0.3, 0.2, 0.2, 0.3], 0.05, 0.05, seed=305)
    raw, var = synth.dna_to_fasta2bin(tips)
    rng = np.random.default_rng(6)
    b = raw.view(np.uint8).copy()
    m = (rng.random(b.shape) < 0.03) & (b > 0) & (b < 0x10)
    b[m] = rng.choice([3, 5, 6, 9, 10, 12, 7, 15], size=int(m.sum())).astype(np.uint8)
    raw = b.view(np.uint32).reshape(raw.shape)
    for radius in (int(var.sum()) - 60, int(var.sum()) // 2):
        c1, i1 = gpu_lib.radius_dna(raw, radius)
        c0, i0 = O.radius_dna(raw, radius)
        assert np.array_equal(c1, c0) and np.array_equal(i1, i0)
        q = np.arange(0, 700, 29, dtype=np.uint32)
        assert np.array_equal(gpu_lib.try_radius_dna(raw, radius, q), O.try_radius_dna(raw, radius, q))


@pytest.mark.parametrize("ny,nx,ntip", [(1, 1, 40), (13, 7, 40), (300, 211, 1000), (64, 64, 2048)])
def test_transfer_dis_random(gpu_lib, ny, nx, ntip):
    rng = np.random.default_rng(ny * 7 + nx)
    nb = (ntip + 31) // 32
    y = rng.integers(0, 2**32, size=(ny, nb), dtype=np.uint64).astype(np.uint32)
    x = rng.integers(0, 2**32, size=(nx, nb), dtype=np.uint64).astype(np.uint32)
    if ntip % 32:  # clear padding bits on most rows, keep some set
        keep = np.uint32((1 << (ntip % 32)) - 1)
        y[::2, -1] &= keep
        x[1::2, -1] &= keep
    got = gpu_lib.transfer_dis(y, x, ntip)
    want = O.transfer_dis(y, x, ntip)
    for g, w_ in zip(got, want):
        assert np.array_equal(g, w_)


def test_radius_row_ranges_concatenate_to_full_lists(gpu_lib):
    from casphy_b200 import synth
    words = synth.binary_workload(700, 128, 10, 0.05, 0.05, seed=31)
    bmat = np.ascontiguousarray(words.T)
    w = np.ones(128)
    fc, fi = gpu_lib.radius_bit(bmat, w, 3)
    parts = [gpu_lib.radius_bit_rows(bmat, w, 3, lo, hi) for lo, hi in ((0, 33), (33, 400), (400, 700))]
    assert np.array_equal(np.concatenate([p[0] for p in parts]), fc)
    assert np.array_equal(np.concatenate([p[1] for p in parts]), fi)
    raw, var = synth.dna_to_fasta2bin(synth.hky85_alignment(500, 300, 4.0, [.3, .2, .2, .3], 0.02, 0.02, seed=32)[0])
    r = int(var.sum()) - 10
    dc, di = gpu_lib.radius_dna(raw, r)
    parts = [gpu_lib.radius_dna_rows(raw, r, lo, hi) for lo, hi in ((0, 250), (250, 251), (251, 500))]
    assert np.array_equal(np.concatenate([p[0] for p in parts]), dc)
    assert np.array_equal(np.concatenate([p[1] for p in parts]), di)


def test_radius_lists_outgrowing_the_guess(gpu_lib):
    """Radius 0 makes every pair a neighbour: the row-range call's guessed
    buffer (64 per row) is too small and it searches again into an exact one;
    the full call's library-allocated lists come from one search.  Both equal
    the oracle's."""
    from casphy_b200 import synth
    words = synth.binary_workload(1500, 64, 11, 0.05, 0.05, seed=32)
    bmat = np.ascontiguousarray(words.T)
    w = np.ones(64)
    c0, i0 = O.radius_bit(bmat, w, 0)
    c1, i1 = gpu_lib.radius_bit(bmat, w, 0)
    c2, i2 = gpu_lib.radius_bit_rows(bmat, w, 0, 0, 1500)
    assert int(c0.sum()) == 1500 * 1500
    assert np.array_equal(c1, c0) and np.array_equal(i1, i0)
    assert np.array_equal(c2, c0) and np.array_equal(i2, i0)
    del i1  # the library's list buffer is released with the array
