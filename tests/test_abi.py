"""libcasphy.so exports every entry point include/casphy.h declares; the
drop-in executables follow the reference tools' error conventions.  No GPU
compute happens here."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
LIB = os.path.join(ROOT, "casphy_b200", "libcasphy.so")
BIN = os.path.join(ROOT, "casphy_b200", "bin")


def _declared():
    txt = open(os.path.join(ROOT, "include", "casphy.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(casphy_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "casphy_b200"), "-j8"], check=True)
    return ctypes.CDLL(LIB)


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(lib):
    lib.casphy_strerror.restype = ctypes.c_char_p
    assert lib.casphy_strerror(0) == b"ok"
    assert lib.casphy_strerror(5) == b"device-side wait timed out"
    assert lib.casphy_abi_version() == 2


def test_no_gpu_is_an_error_not_a_fallback(lib):
    if lib.casphy_device_count() > 0:
        pytest.skip("a GPU is visible")
    import casphy_b200.lib as L
    with pytest.raises(L.CasphyError) as ei:
        L.join_indel(np.array([[2, 1], [2, 1]], np.uint32), 1, np.ones((1, 2)))
    assert ei.value.status == 7


def _exe(name):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        subprocess.run(["make", "-C", os.path.join(ROOT, "casphy_b200"), "-j8"], check=True)
    return exe


# tool, argv after the prefix, the reference's message for a missing input,
# whether the reference prints its device count first, and where it does so
MISSING = [
    ("joinEdgeIndel", ["w", "2", "0", "2"], "No tbmat input.", False, "cu/joinEdgeIndel.cu:263-266"),
    ("joinEdgeBitReverse", ["w", "1"], "No tbmat input.", False, "cu/joinEdgeBitReverse.cu:301-304"),
    ("nodeKeepIndel", ["1"], "No nodeState input.", False, "cu/nodeKeepIndel.cu:66-69"),
    ("nodeKeepBit", ["1"], "No nodeState input.", False, "cu/nodeKeepBit.cu:107-110"),
    ("radiusNeighbor", ["4"], "No bmat input.", True, "cu/radiusNeighbor.cu:175,183-186"),
    ("radiusNeighborDNA", ["4"], "No bmat input.", True, "cu/radiusNeighborDNA.cu:124,131-135"),
    ("tryRadius", ["4", "3"], "No bmat input.", False, "cu/tryRadius.cu:68-72"),
    ("tryRadiusDNA", ["4", "3"], "No bmat input.", False, "cu/tryRadiusDNA.cu:93-97"),
    ("Felsenstein", ["7"], "No input.", False, "cu/Felsenstein.cu:94-97"),
    ("tipMerge", ["0.4"], "No nNeighbor input.", True, "cu/tipMerge.cu:149,156-159"),
]


@pytest.mark.parametrize("tool,args,msg,devline,where", MISSING, ids=[m[0] for m in MISSING])
def test_drop_in_missing_input_prints_and_returns_zero(tmp_path, tool, args, msg, devline, where):
    r = subprocess.run([_exe(tool), str(tmp_path / "nothing")] + args, capture_output=True, text=True)
    lines = r.stdout.strip().splitlines()
    assert r.returncode == 0, where
    assert lines[-1] == msg, where
    if devline:
        assert len(lines) == 2 and re.fullmatch(r"\d+ devices detected", lines[0]), where
    else:
        assert len(lines) == 1, where
    assert sorted(os.listdir(tmp_path)) == []


def test_transfer_dis_missing_input_is_an_error(tmp_path):
    """The reference reads the header without checking the fopen result
    (cu/TransferDisStream.cu:141-146) and crashes; the drop-in reports the
    error and exits non-zero, writing nothing."""
    r = subprocess.run([_exe("TransferDisStream"), str(tmp_path / "y"), str(tmp_path / "x"),
                        str(tmp_path / "out"), "10"], capture_output=True, text=True)
    assert r.returncode != 0
    assert "cannot open input" in r.stderr
    assert sorted(os.listdir(tmp_path)) == []
