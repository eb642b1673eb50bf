"""File formats, bit packing, R-compatible regularisation and the seeded
synthetic generators."""
import numpy as np

from casphy_b200 import formats, synth


def test_matrix_file_roundtrip(tmp_path):
    m = np.arange(12, dtype=np.uint32).reshape(3, 4)
    formats.write_mat(tmp_path / "m", m)
    raw = np.fromfile(tmp_path / "m", dtype=np.uint32)
    assert list(raw[:2]) == [3, 4]
    assert np.array_equal(formats.read_mat(tmp_path / "m"), m)


def test_pack_bits_layout():
    bits = np.zeros((2, 40), dtype=bool)
    bits[0, 0] = bits[0, 33] = bits[1, 31] = True
    w = formats.pack_bits(bits)
    assert w.shape == (2, 2)
    assert w[0, 0] == 1 and w[0, 1] == 2 and w[1, 0] == 1 << 31
    assert np.array_equal(formats.unpack_bits(w, 40), bits)
    u = formats.pack_u64(w)
    assert u[0, 0] == (1 | (2 << 32))


def test_regularize_matches_r_semantics():
    # R: tmp <- sort(unique(c(col,-1,0))); match(col,tmp) - 2 ; then +1
    col = np.array([[5], [-1], [0], [9], [5], [2]], dtype=np.int32)
    codes, ns = synth.regularize(col)
    assert codes[:, 0].tolist() == [3, 0, 1, 4, 3, 2]
    assert ns == 3


def test_generators_are_deterministic():
    a = synth.lineage_states(300, 40, 10, 0.05, 16, 1.5, 0.1, seed=9)
    b = synth.lineage_states(300, 40, 10, 0.05, 16, 1.5, 0.1, seed=9)
    assert np.array_equal(a, b)
    assert a.min() >= -1 and a.max() <= 16
    assert 0.05 < (a == -1).mean() < 0.15


def test_irreversible_edits_follow_tree():
    # with no missing data, every allele column is consistent with a tree: a
    # cell's edited sites are a superset of its sampled ancestor lineage's
    s = synth.lineage_states(64, 32, 6, 0.1, 8, 1.0, 0.0, seed=1)
    assert (s >= 0).all()


def test_hky85_rows_are_stochastic():
    P = synth.hky85_P(0.05, 4.0, np.array([0.3, 0.2, 0.2, 0.3]))
    assert np.allclose(P.sum(axis=1), 1.0)
    assert (P > 0).all()


def test_fasta2bin_encoding_drops_invariant_columns():
    st = np.array([[0, 1, 2, 4], [0, 3, 2, 4], [0, 1, 2, 2]], dtype=np.uint8)
    words, keep = synth.dna_to_fasta2bin(st)
    assert keep.tolist() == [False, True, False, True]
    assert words.shape == (3, 1)
    assert words[0, 0] == (0x04 | (0x10 << 8))
