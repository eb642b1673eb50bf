"""The fasta2bin drop-in's host side (FASTA reading, names, valid-base counts,
error messages) on the CPU: the executable's source is compiled against a stub
of the library whose encoder returns the sequence matrix it was given, and the
result is compared with the Python restatement of the reference's reader
(oracle/fasta.py, cu/fasta2bin.cu:120-183)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import fasta as F

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..")
TOOLS = os.path.join(ROOT, "casphy_b200", "csrc", "tools")

# The stub stands in for libcasphy: no device work, the .bin body is the
# row-major letter matrix and every column is reported variable.
STUB = r"""
#include <cstdint>
#include <cstring>
#include "casphy.h"
extern "C" int casphy_device_count(void) { return 1; }
extern "C" int casphy_set_device(int) { return 0; }
extern "C" const char* casphy_strerror(int) { return "stub"; }
extern "C" const char* casphy_last_error(void) { return ""; }
extern "C" int casphy_fasta_encode(uint32_t nseq, uint32_t len, const char* seqs, uint8_t* variable,
                                   uint32_t* nkeep, uint32_t* bin_out, uint64_t cap) {
    memset(variable, 1, len);
    *nkeep = len;
    const size_t n = (size_t)nseq * len;
    memset(bin_out, 0, cap * 4);
    if (n > cap * 4) return 1;
    memcpy(bin_out, seqs, n);
    return 0;
}
"""


@pytest.fixture(scope="module")
def tool(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("f2b")
    stub = d / "stub.cpp"
    stub.write_text(STUB)
    exe = d / "fasta2bin_stub"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", TOOLS, "-o", str(exe),
                    os.path.join(TOOLS, "fasta2bin.cpp"), os.path.join(TOOLS, "toolio.cpp"), str(stub), "-pthread"],
                   check=True)
    return str(exe)


def _run(tool, tmp_path, text: bytes):
    src = tmp_path / "in.fasta"
    src.write_bytes(text)
    out = tmp_path / "out"
    r = subprocess.run([tool, str(src), str(out)], capture_output=True)
    files = {}
    for ext in (".bin", "_names.txt"):
        p = tmp_path / ("out" + ext)
        files[ext] = p.read_bytes() if p.exists() else None
    return r, files


def _golden_texts():
    z = np.load(os.path.join(HERE, "golden", "fasta_reference.npz"))
    names = sorted(set(k.split("/")[1] for k in z.files))
    return [(n, z[f"fa/{n}/fasta"].tobytes()) for n in names]


EDGE = [
    ("crlf", b">a x\r\nAC GT\r\nACGT\r\n>b\r\nACGT\r\nNNnn\r\n"),
    ("no_final_newline", b">a\nACGT\n>b\nAC.T"),
    ("blank_lines_and_empty_header", b"\n\n>a\n\nAC\n\nGT\n\n>empty\n>b\nACGT\n\n"),
    ("letters_before_first_header", b"ACGT\n>a\nACGT\n"),
    ("names_with_tabs", b">\t  name1\tmore\nACGT\n>   \nACGT\n>x\n A C G T \n"),
    ("lower_case_and_ambiguity", b">s1\nacgtRYKM\n>s2\nNNNN-.-.\n"),
]


@pytest.mark.parametrize("name,text", _golden_texts() + EDGE, ids=[c[0] for c in _golden_texts() + EDGE])
def test_reader_matches_restatement(tool, tmp_path, name, text):
    r, files = _run(tool, tmp_path, text)
    assert r.returncode == 0, r.stderr
    names, seqs = F.parse(text.decode())
    n, L = len(seqs), len(seqs[0])
    body = np.frombuffer(files[".bin"], dtype=np.uint32)
    assert body[0] == n and body[1] == (L + 3) // 4
    mat = body[2:].view(np.uint8)[: n * L]
    assert mat.tobytes() == "".join(seqs).encode()
    valid = [sum(1 for c in s if c.upper() not in "-.N") for s in seqs]
    want = "SequenceName,ValidBaseCount\n" + "".join(f"{a},{v}\n" for a, v in zip(names, valid))
    assert files["_names.txt"].decode() == want


@pytest.mark.parametrize("text,msg", [
    (b"", b"Error: No valid sequences found in file"),
    (b">a\n>b\n", b"Error: No valid sequences found in file"),
    (b">a\nACGT\n>b\nACG\n", b"Error: All sequences must have the same length for variant filtering"),
], ids=["empty", "headers_only", "ragged"])
def test_reader_errors(tool, tmp_path, text, msg):
    r, files = _run(tool, tmp_path, text)
    assert r.returncode == 1 and msg in r.stderr
    assert files[".bin"] is None


def test_missing_file(tool, tmp_path):
    r = subprocess.run([tool, str(tmp_path / "absent.fasta"), str(tmp_path / "o")], capture_output=True)
    assert r.returncode == 1 and b"Error: Cannot open file:" in r.stderr
