"""The drop-in executables (casphy_b200/bin) run on the golden inputs write
the same files, byte for byte, as the reference executables did."""
import os

import numpy as np
import pytest

import make_golden
import oracle as O

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(__file__), "..", "casphy_b200", "bin")


@pytest.fixture(scope="module")
def tool_outputs(gpu_lib):
    """Every golden case run through the drop-in executables."""
    return make_golden.run_tools(BIN)


def test_dropin_outputs_match_reference_files(golden, tool_outputs):
    cases, ref = golden
    got = tool_outputs
    checked, bad = 0, []
    for key, want in sorted(ref.items()):
        if key not in got:
            bad.append(f"missing {key}")
            continue
        have = got[key]
        if key.startswith(("trb/", "trd/")):
            # rows are drawn with rand(); check the counts for the drawn rows
            kind, name, _ = key.split("/")
            nrep = int(have[1])
            q, cnt = have[2:2 + nrep], have[2 + nrep:]
            c = cases[("jb" if kind == "trb" else "dna", name)]
            if kind == "trb":
                bmat = np.ascontiguousarray(c["words"].T)
                exp = O.try_radius_bit(bmat, c["w"], 4, q)
            else:
                exp = O.try_radius_dna(c["raw"], int(c["lvalid"][0]) - 20, q)
            ok = np.array_equal(cnt, exp)
        else:
            ok = have.shape == want.shape and np.array_equal(have, want)
        checked += 1
        if not ok:
            bad.append(f"differs: {key}")
    assert checked > 50
    assert not bad, "\n".join(bad)


def test_felsenstein_resampler_matches_reference_files(golden, tool_outputs):
    """`Felsenstein <prefix> 7` (cu/Felsenstein.cu:56-66): the mt19937 column
    draw (.idx) and the gathered matrix (.bin) equal the reference tool's
    files byte for byte on both alignments."""
    _, ref = golden
    got = tool_outputs
    keys = sorted(k for k in ref if k.startswith("fs/"))
    assert len(keys) == 4
    for key in keys:
        assert key in got, f"drop-in wrote no {key}"
        assert got[key].shape == ref[key].shape and np.array_equal(got[key], ref[key]), key
