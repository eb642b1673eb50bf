"""ctypes access to the reference's CPU implementations of the hot path,
compiled from src/functions.cpp into oracle/_ref/libcputwin_ref.so
(make -C oracle ref).  Test infrastructure: the timed CPU baseline beside the
B200 path and a cross-check of tree validity, never part of the product.

    greedy_join_edge2          src/functions.cpp:1880-2017 (phy.join, indel)
    greedy_join_edge_bit       src/functions.cpp:3316-3461 (phy.join, bit)
    radius_weighted_rows       src/functions.cpp:1825-1857 per row, rows in parallel
    radius_weighted_dna_rows   src/functions.cpp:4021-4036 per row, rows in parallel
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcputwin_ref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        u32, i32 = C.c_uint32, C.c_int
        L.ref_greedy_join_edge2.argtypes = [u32, u32, P, u32, P, P, i32, C.c_float, P]
        L.ref_greedy_join_edge_bit_reverse.argtypes = [u32, u32, P, P, i32, P]
        L.ref_radius_weighted_rows.argtypes = [u32, u32, P, i32, P, C.c_float, u32, u32, i32, P]
        L.ref_radius_weighted_dna_rows.argtypes = [u32, u32, P, P, C.c_float, u32, u32, i32, P]
        for f in (L.ref_greedy_join_edge2, L.ref_greedy_join_edge_bit_reverse, L.ref_radius_weighted_rows,
                  L.ref_radius_weighted_dna_rows):
            f.restype = i32
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def greedy_join_edge2(codes, nstate, weight, tip_size=None, min_size=0, min_ratio=2.0, want_edge=True):
    """greedyJoinEdge2 on regularised codes (ncell x nsite; 0 missing, 1
    unedited, 2.. alleles), as phy.join calls it: mat = t(codes - 1), weight
    nstate x nsite.  Returns the (3 + nsite) x (2 ncell - 1) edge matrix
    (rows: parent, child, change count, child states) or None."""
    codes = np.asarray(codes)
    ncell, nsite = codes.shape
    mat = np.ascontiguousarray(codes.astype(np.int32) - 1)  # ncell x nsite row-major == nsite x ncell col-major
    w = np.asfortranarray(np.asarray(weight, dtype=np.float64).reshape(nstate, nsite))
    ts = np.ascontiguousarray(np.ones(ncell, np.int32) if tip_size is None else np.asarray(tip_size, np.int32))
    out = np.zeros((2 * ncell - 1, 3 + nsite), dtype=np.int32) if want_edge else None
    rc = lib().ref_greedy_join_edge2(ncell, nsite, _p(mat), nstate, w.ctypes.data_as(C.c_void_p), _p(ts),
                                     int(min_size), float(min_ratio), _p(out) if want_edge else None)
    if rc:
        raise RuntimeError(f"ref_greedy_join_edge2 returned {rc}")
    return out.T if want_edge else None


def greedy_join_edge_bit(words, weight=None, ancestral_type=0, want_edge=True):
    """greedyJoinEdgeBitReverse on packed rows (ncell x nbin uint32 words).
    Returns the 2 x (2 ncell - 2) edge matrix (0-based parent, child) or None."""
    words = np.ascontiguousarray(words, dtype=np.uint32)
    ncell, nbin = words.shape
    w = np.ascontiguousarray(np.ones(32 * nbin) if weight is None else np.asarray(weight, np.float64))
    out = np.zeros((2 * ncell - 2, 2), dtype=np.int32) if want_edge else None
    rc = lib().ref_greedy_join_edge_bit_reverse(ncell, nbin, _p(words), _p(w), int(ancestral_type),
                                                _p(out) if want_edge else None)
    if rc:
        raise RuntimeError(f"ref_greedy_join_edge_bit_reverse returned {rc}")
    return out.T if want_edge else None


def radius_weighted_rows(words, radius, row0, row1, nthreads, weight=None):
    """radiusWeightedParallel for rows [row0, row1) of packed rows (ncell x
    nword).  Returns (counts, bitmaps (rows x nbin uint32))."""
    words = np.asarray(words, dtype=np.uint32)
    ncell, nword = words.shape
    mat = np.asfortranarray(words)
    max_char = max(1, int(np.unpackbits(words.view(np.uint8), axis=1).sum(axis=1).max()))
    w = np.ascontiguousarray(np.ones(32 * nword) if weight is None else np.asarray(weight, np.float64))
    nb = (ncell + 31) // 32
    out = np.zeros((row1 - row0, nb + 1), dtype=np.uint32)
    rc = lib().ref_radius_weighted_rows(ncell, nword, mat.ctypes.data_as(C.c_void_p), max_char, _p(w),
                                        float(radius), row0, row1, int(nthreads), _p(out))
    if rc:
        raise RuntimeError(f"ref_radius_weighted_rows returned {rc}")
    return out[:, 0].copy(), out[:, 1:].copy()


def radius_weighted_dna_rows(ints, radius, row0, row1, nthreads, weight=None):
    """radiusWeightedDNAParallel for rows [row0, row1) of fasta2bin rows
    (nseq x nint words, four columns per word, one code byte each), which is
    the matrix R hands it (nint x nseq column-major)."""
    ints = np.ascontiguousarray(ints, dtype=np.uint32)
    nseq, nint = ints.shape
    w = np.ascontiguousarray(np.ones(4 * nint) if weight is None else np.asarray(weight, np.float64))
    nb = (nseq + 31) // 32
    out = np.zeros((row1 - row0, nb + 1), dtype=np.uint32)
    rc = lib().ref_radius_weighted_dna_rows(nseq, nint, _p(ints), _p(w), float(radius), row0, row1,
                                            int(nthreads), _p(out))
    if rc:
        raise RuntimeError(f"ref_radius_weighted_dna_rows returned {rc}")
    return out[:, 0].copy(), out[:, 1:].copy()
