"""Readers and writers for the files CasPhy's R package and CUDA tools exchange.

All files are little-endian.  A *matrix file* is ``u32 dim[2]`` followed by
``dim[0]`` rows of ``dim[1]`` u32 values; the R writer ``write.mat2bin``
(R/CasPhy_functions.R:1551-1585) stores ``rev(dim(m))`` and the column-major
data of ``m``, so a file written from an R matrix with one column per cell
has one row per cell here.  Weight files are raw float64 with no header
(R/CasPhy_functions.R:606,609).  ``.idx`` is a headerless run of u32 and
``.retainNode`` is text with one id per line (cu/nodeKeepIndel.cu:149).
"""
from __future__ import annotations

import os
import numpy as np

U32 = np.dtype("<u4")


def write_mat(path: str | os.PathLike, mat: np.ndarray) -> None:
    """Write a 2-D matrix file (header = rows, cols)."""
    m = np.ascontiguousarray(mat, dtype=U32)
    if m.ndim != 2:
        raise ValueError("write_mat expects a 2-D array")
    with open(path, "wb") as f:
        np.array(m.shape, dtype=U32).tofile(f)
        m.tofile(f)


def read_mat(path: str | os.PathLike) -> np.ndarray:
    """Read a matrix file into a (dim0, dim1) u32 array."""
    raw = np.fromfile(path, dtype=U32)
    if raw.size < 2:
        raise ValueError(f"{path}: truncated header")
    r, c = int(raw[0]), int(raw[1])
    body = raw[2:]
    if body.size < r * c:
        raise ValueError(f"{path}: expected {r}x{c} values, found {body.size}")
    return body[: r * c].reshape(r, c)


def read_header(path: str | os.PathLike) -> tuple[int, int]:
    raw = np.fromfile(path, dtype=U32, count=2)
    return int(raw[0]), int(raw[1])


def write_f64(path: str | os.PathLike, arr: np.ndarray) -> None:
    np.ascontiguousarray(arr, dtype="<f8").tofile(path)


def read_f64(path: str | os.PathLike, count: int = -1) -> np.ndarray:
    return np.fromfile(path, dtype="<f8", count=count)


def read_idx(path: str | os.PathLike) -> np.ndarray:
    return np.fromfile(path, dtype=U32)


def read_retain(path: str | os.PathLike) -> np.ndarray:
    with open(path) as f:
        return np.array([int(x) for x in f.read().split()], dtype=U32)


def write_retain(path: str | os.PathLike, nodes) -> None:
    with open(path, "w") as f:
        for n in nodes:
            f.write(f"{int(n)}\n")


# ---------------------------------------------------------------------------
# packing helpers

def pack_bits(bits: np.ndarray) -> np.ndarray:
    """(n, nsite) bool -> (n, ceil(nsite/32)) u32; bit j of word k is site 32k+j
    (src/functions.cpp:54-68)."""
    bits = np.asarray(bits, dtype=bool)
    n, nsite = bits.shape
    nbin = (nsite + 31) // 32
    pad = np.zeros((n, nbin * 32), dtype=bool)
    pad[:, :nsite] = bits
    b8 = np.packbits(pad.reshape(n, nbin * 4, 8), axis=2, bitorder="little").reshape(n, nbin * 4)
    return b8.view("<u4").reshape(n, nbin).copy()


def unpack_bits(words: np.ndarray, nsite: int | None = None) -> np.ndarray:
    w = np.ascontiguousarray(words, dtype=U32)
    n, nbin = w.shape
    b = np.unpackbits(w.view(np.uint8).reshape(n, nbin * 4), axis=1, bitorder="little").astype(bool)
    return b if nsite is None else b[:, :nsite]


def pack_u64(words32: np.ndarray) -> np.ndarray:
    """Little-endian view of u32 word pairs as u64 (bit indices are kept)."""
    w = np.ascontiguousarray(words32, dtype=U32)
    n, nbin = w.shape
    if nbin % 2:
        w = np.concatenate([w, np.zeros((n, 1), dtype=U32)], axis=1)
    return w.view("<u8").copy()


# fasta2bin's 8-bit IUPAC codes (cu/fasta2bin.cu:12-33)
IUPAC = {
    "A": 0x01, "T": 0x02, "U": 0x02, "C": 0x04, "G": 0x08,
    "W": 0x03, "M": 0x05, "R": 0x09, "Y": 0x06, "K": 0x0A, "S": 0x0C,
    "H": 0x07, "D": 0x0B, "V": 0x0D, "B": 0x0E, "N": 0x0F,
}
GAP_CODE = 0x10


def encode_dna_codes(codes8: np.ndarray) -> np.ndarray:
    """(n, L) uint8 codes -> (n, ceil(L/4)) u32 words, code of base 4i+j in byte j
    (cu/fasta2bin.cu:189-210)."""
    c = np.asarray(codes8, dtype=np.uint8)
    n, L = c.shape
    nb = (L + 3) // 4
    pad = np.zeros((n, nb * 4), dtype=np.uint8)
    pad[:, :L] = c
    return pad.view("<u4").reshape(n, nb).copy()
