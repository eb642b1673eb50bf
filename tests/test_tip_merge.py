"""tipMerge: the oracle and the GPU path against the .member files of the
reference executable (tests/golden/tipmerge_reference.npz, made by
make_tipmerge_golden.py), and the drop-in executable on one case."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import make_tipmerge_golden as G
import oracle as O
from casphy_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "..", "casphy_b200", "bin", "tipMerge")


def _cases():
    z = np.load(os.path.join(HERE, "golden", "tipmerge_reference.npz"))
    out = []
    for name, _, _, _ in G.CASES:
        ntip, seed = (int(x) for x in z[f"tm/{name}/params"])
        out.append((name, ntip, seed, float(z[f"tm/{name}/pshared"][0]), z[f"tm/{name}/member"]))
    return out


@pytest.mark.parametrize("name,ntip,seed,p,want", _cases(), ids=[c[0] for c in G.CASES])
def test_oracle_matches_reference(name, ntip, seed, p, want):
    counts, idx = synth.neighbour_lists(ntip, seed)
    assert np.array_equal(O.tip_merge(counts, idx, p), want)


@pytest.mark.gpu
@pytest.mark.parametrize("name,ntip,seed,p,want", _cases(), ids=[c[0] for c in G.CASES])
def test_gpu_matches_reference(gpu_lib, name, ntip, seed, p, want):
    counts, idx = synth.neighbour_lists(ntip, seed)
    assert np.array_equal(gpu_lib.tip_merge(counts, idx, p), want)


@pytest.mark.gpu
def test_dropin_writes_the_reference_member_file(gpu_lib):
    name, ntip, seed, p, want = _cases()[2]
    counts, idx = synth.neighbour_lists(ntip, seed)
    assert np.array_equal(G.run_tool(BIN, counts, idx, p), want)


@pytest.mark.gpu
def test_gpu_on_radius_lists_matches_oracle(gpu_lib):
    from casphy_b200 import synth
    states, _ = synth.hky85_alignment(3000, 400, 4.0, [.3, .2, .2, .3], 0.01, 0.02, seed=51)
    raw, var = synth.dna_to_fasta2bin(states)
    counts, idx = gpu_lib.radius_dna(raw, int(var.sum()) - 25)
    for p in (0.2, 0.5):
        assert np.array_equal(gpu_lib.tip_merge(counts, idx, p), O.tip_merge(counts, idx, p))


@pytest.mark.gpu
def test_too_many_neighbours(gpu_lib):
    n = 1024 * 1024 + 2
    counts = np.zeros(n, np.uint32)
    counts[0] = n - 1
    idx = np.arange(1, n, dtype=np.uint32)
    with pytest.raises(gpu_lib.CasphyError):
        gpu_lib.tip_merge(counts, idx, 0.5)
