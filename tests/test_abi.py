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


def test_drop_in_missing_input_prints_and_returns_zero(tmp_path):
    exe = os.path.join(BIN, "joinEdgeIndel")
    if not os.path.exists(exe):
        subprocess.run(["make", "-C", os.path.join(ROOT, "casphy_b200"), "-j8"], check=True)
    r = subprocess.run([exe, str(tmp_path / "nothing"), str(tmp_path / "w"), "2", "0", "2"],
                       capture_output=True, text=True)
    assert r.returncode == 0
    assert r.stdout.strip() == "No tbmat input."
    assert not (tmp_path / "nothing.edge2").exists()
