"""Parsimony change counts per edge (ancestralBitReverse, charAncestralEC):
the oracle against the outputs of the reference's own functions
(tests/golden/parsimony_reference.npz), and the GPU against both."""
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _cases():
    z = np.load(os.path.join(HERE, "golden", "parsimony_reference.npz"))
    out = {}
    for k in z.files:
        kind, name, field = k.split("/")
        if kind in ("pb", "pc"):
            out.setdefault((kind, name), {})[field] = z[k]
    return sorted(out.items())


def _run(mod, kind, c):
    nnode = int(c["nnode"][0])
    if kind == "pb":
        return mod.ancestral_bit(c["words"], c["edge"], nnode)
    return mod.ancestral_char(c["mat"], c["edge"], c["tips"], float(c["rule"][0]), float(c["rule"][1]), nnode)


@pytest.mark.parametrize("key,c", _cases(), ids=lambda x: "/".join(x) if isinstance(x, tuple) else "")
def test_oracle_matches_reference(key, c):
    state, ln = _run(O, key[0], c)
    assert np.array_equal(state, c["state"]) and np.array_equal(ln, c["len"])


@pytest.mark.gpu
@pytest.mark.parametrize("key,c", _cases(), ids=lambda x: "/".join(x) if isinstance(x, tuple) else "")
def test_gpu_matches_reference(gpu_lib, key, c):
    state, ln = _run(gpu_lib, key[0], c)
    assert np.array_equal(state, c["state"]) and np.array_equal(ln, c["len"])


@pytest.mark.gpu
def test_gpu_matches_oracle_on_join_trees(gpu_lib):
    from casphy_b200 import synth
    words = synth.binary_workload(20_000, 512, 16, 0.03, 0.05, seed=41)
    edge, _, _ = gpu_lib.join_bit(words, None, 1)
    for mod_out in (gpu_lib.ancestral_bit(words, edge),):
        want = O.ancestral_bit(words, edge)
        assert np.array_equal(mod_out[0], want[0]) and np.array_equal(mod_out[1], want[1])
    raw = synth.lineage_states(20_000, 256, 16, 0.03, 64, 1.5, 0.1, seed=42)
    codes, ns = synth.regularize(raw)
    e2, _, _ = gpu_lib.join_indel(codes, ns, np.ones((ns, 256)))
    tips = np.random.default_rng(3).integers(1, 20, 20_000)
    got = gpu_lib.ancestral_char(raw, e2, tips, 10, 2)
    want = O.ancestral_char(raw, e2, tips, 10, 2)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


@pytest.mark.gpu
def test_gpu_rejects_unordered_edges(gpu_lib):
    from casphy_b200 import synth
    words = synth.binary_workload(50, 64, 8, 0.05, 0.05, seed=43)
    edge, _, _ = gpu_lib.join_bit(words, None, 1)
    with pytest.raises(gpu_lib.CasphyError):
        gpu_lib.ancestral_bit(words, edge[::-1])


def _nd_cases():
    z = np.load(os.path.join(HERE, "golden", "parsimony_reference.npz"))
    names = sorted(set(k.split("/")[1] for k in z.files if k.startswith("nd/")))
    out = []
    for n in names:
        ntip, nnode = (int(x) for x in z[f"nd/{n}/ntip"])
        raw = z[f"nd/{n}/file"]
        out.append((n, z[f"nd/{n}/edge"], ntip, nnode, raw[:2], raw[2:].reshape(-1, raw[1]), z[f"nd/{n}/sizes"]))
    return out


@pytest.mark.parametrize("name,edge,ntip,nnode,hdr,rows,sizes", _nd_cases(), ids=[c[0] for c in _nd_cases()])
def test_node_des_oracle_matches_reference(name, edge, ntip, nnode, hdr, rows, sizes):
    r, s = O.node_des(edge, ntip, nnode)
    assert tuple(hdr) == (nnode - 1, (ntip - 1) // 32 + 1)
    assert np.array_equal(r, rows) and np.array_equal(s, sizes)


@pytest.mark.gpu
@pytest.mark.parametrize("name,edge,ntip,nnode,hdr,rows,sizes", _nd_cases(), ids=[c[0] for c in _nd_cases()])
def test_node_des_gpu_matches_reference(gpu_lib, name, edge, ntip, nnode, hdr, rows, sizes):
    r, s = gpu_lib.node_des(edge, ntip, nnode)
    assert np.array_equal(r, rows) and np.array_equal(s, sizes)


@pytest.mark.gpu
def test_node_des_gpu_on_a_large_join_tree(gpu_lib):
    from casphy_b200 import bootstrap as B
    from casphy_b200 import synth
    words = synth.binary_workload(30_000, 256, 16, 0.03, 0.05, seed=44)
    edge, _, _ = gpu_lib.join_bit(words, None, 1)
    r, s = gpu_lib.node_des(edge, 30_000)
    ro, so = O.node_des(edge, 30_000)
    assert np.array_equal(r, ro) and np.array_equal(s, so)
    # the same set of clades as the package's clade bitsets (all internal nodes but the root)
    cb = B.clade_bits(edge, 30_000, (30_000 + 31) // 32)
    assert np.array_equal(np.unique(r, axis=0), np.unique(cb, axis=0))
