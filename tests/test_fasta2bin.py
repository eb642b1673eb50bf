"""fasta2bin: the Python restatement and the GPU drop-in against the outputs
of the reference's own fasta2bin (tests/golden/fasta_reference.npz)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import fasta as F

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "..", "casphy_b200", "bin", "fasta2bin")


def _cases():
    z = np.load(os.path.join(HERE, "golden", "fasta_reference.npz"))
    names = sorted(set(k.split("/")[1] for k in z.files))
    return [(n, z[f"fa/{n}/fasta"].tobytes().decode(), z[f"fa/{n}/bin"], z[f"fa/{n}/names"].tobytes().decode(),
             z[f"fa/{n}/positions"].tobytes().decode()) for n in names]


@pytest.mark.parametrize("name,text,bin_,names,pos", _cases(), ids=[c[0] for c in _cases()])
def test_restatement_matches_reference(name, text, bin_, names, pos):
    b, n, p = F.convert(text)
    assert np.array_equal(b, bin_) and n == names and p == pos


@pytest.mark.gpu
@pytest.mark.parametrize("name,text,bin_,names,pos", _cases(), ids=[c[0] for c in _cases()])
def test_dropin_matches_reference(gpu_lib, name, text, bin_, names, pos):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "in.fasta")
        with open(src, "w") as f:
            f.write(text)
        subprocess.run([BIN, src, os.path.join(d, "out")], check=True, stdout=subprocess.DEVNULL)
        got = np.fromfile(os.path.join(d, "out.bin"), dtype=np.uint32)
        with open(os.path.join(d, "out_names.txt")) as f:
            gn = f.read()
        with open(os.path.join(d, "out_positions.txt")) as f:
            gp = f.read()
    assert np.array_equal(got, bin_) and gn == names and gp == pos
