"""The CPU oracle reproduces the reference tools' output bytes on every
golden case (outputs generated by running the reference executables, built
from the CasPhy sources, on a B200; see tests/golden/make_golden.py)."""
import ctypes

import numpy as np
import pytest

import golden_check
import oracle as O


def test_oracle_matches_reference_tools(golden):
    cases, ref = golden
    bad = [m for _, ok, m in golden_check.iter_checks(cases, ref) if not ok]
    assert not bad, "\n".join(bad)


def test_oracle_f16_emulation_matches_reference(golden):
    """The binary16 path (forced) gives the same bytes as the integer path on
    unit-weight cases and matches the non-integer-weight golden case."""
    cases, ref = golden
    flag = ctypes.c_int.in_dll(O.lib(), "oracle_force_f16")
    flag.value = 1
    try:
        bad = [m for _, ok, m in golden_check.iter_checks(cases, ref, kinds={"ji"}) if not ok]
    finally:
        flag.value = 0
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("seed", range(3))
def test_binary16_helpers_match_numpy(seed):
    rng = np.random.default_rng(seed)
    L = O.lib()
    xs = np.concatenate([rng.normal(0, 1, 2000), rng.uniform(-70000, 70000, 2000),
                         rng.uniform(-1e-6, 1e-6, 2000), [0.0, -0.0, 65504.0, 65520.0, 2049.0, 2050.0]])
    for x in xs:
        assert L.oracle_f64_to_f16(float(x)) == int(np.float16(x).view(np.uint16))
    h = rng.integers(0, 0x7C00, size=3000).astype(np.uint16)
    for a, b in zip(h[::2], h[1::2]):
        want = (np.float64(np.uint16(a).view(np.float16)) + np.float64(np.uint16(b).view(np.float16)))
        assert L.oracle_f16_add(int(a), int(b)) == int(np.float16(want).view(np.uint16))


def test_oracle_matches_reference_at_1024_sites():
    """The oracle against the reference joinEdgeIndel / nodeKeepIndel built
    with MAXCOL 1024, on three 1,024-site cases of the 200k generator's
    settings (unit, integer and fractional weights; digests in
    tests/golden/wide_reference.json)."""
    import json
    import os
    import make_wide_golden as W
    ref = json.load(open(W.OUT))
    for name in W.CASES:
        got = W.oracle_digests(name)
        for k, v in ref[name].items():
            assert got[k] == v, f"{name}/{k}"
