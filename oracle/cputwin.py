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


def _lib_ac():
    L = lib()
    if not getattr(L, "_ac", False):
        P, u32, i32 = C.c_void_p, C.c_uint32, C.c_int
        L.ref_approx_compare.argtypes = [u32, u32, u32, P, u32, P, u32, P, u32, i32, C.c_float, P, P]
        L.ref_approx_compare.restype = i32
        L.ref_approx_compare_many.argtypes = [u32, u32, u32, P, u32, P, u32, P, P, P, P, P, i32, C.c_float, i32,
                                              P, P]
        L.ref_approx_compare_many.restype = i32
        L._ac = True
    return L


def approx_compare(clade_rows, ntip, edge1, edge2, nnode2=None, cache_size=8192, threshold=0.1):
    """approximateCompare2_AVX2 of one query tree.  clade_rows: the reference
    tree's nodeDesBig rows ((nnode1 - 1) x nbin, file order); edge1, edge2:
    0-based (parent, child) pairs in cladewise order (tips 0.., root ntip).
    Returns (ref2qry nnode1 x 2, qry2ref nnode2 x 3), 1-based nodes as R sees
    them; raises when the function runs out of cache."""
    clade = np.ascontiguousarray(clade_rows, dtype=np.int32)
    nnode1 = clade.shape[0] + 1
    nbin = clade.shape[1]
    e1 = np.ascontiguousarray(np.asarray(edge1).reshape(-1, 2) + 1, dtype=np.int32)
    e2 = np.ascontiguousarray(np.asarray(edge2).reshape(-1, 2) + 1, dtype=np.int32)
    nnode2 = int(e2.max()) - ntip if nnode2 is None else int(nnode2)
    r = np.zeros((2, nnode1), np.int32)
    q = np.zeros((3, nnode2), np.int32)
    rc = _lib_ac().ref_approx_compare(ntip, nnode1, nbin, _p(clade), len(e1), _p(e1), len(e2), _p(e2), nnode2,
                                      int(cache_size), float(threshold), _p(r), _p(q))
    if rc:
        raise RuntimeError("approximateCompare2_AVX2 ran out of cache")
    return r.T.copy(), q.T.copy()


def approx_compare_many(clade_rows, ntip, edge1, edges2, nthreads, cache_size=8192, threshold=0.1):
    """approx_compare over a list of query trees, trees spread over threads.
    Returns (ref2qry distances ntree x nnode1, number of trees out of cache)."""
    clade = np.ascontiguousarray(clade_rows, dtype=np.int32)
    nnode1 = clade.shape[0] + 1
    nbin = clade.shape[1]
    e1 = np.ascontiguousarray(np.asarray(edge1).reshape(-1, 2) + 1, dtype=np.int32)
    es = [np.asarray(e).reshape(-1, 2) for e in edges2]
    ne = np.array([len(e) for e in es], np.uint32)
    nn = np.array([int(e.max()) + 1 - ntip for e in es], np.uint32)
    off = np.zeros(len(es), np.uint64)
    off[1:] = np.cumsum(ne[:-1].astype(np.uint64))
    allE = np.ascontiguousarray(np.concatenate(es) + 1, dtype=np.int32)
    r = np.zeros((len(es), 2, nnode1), np.int32)
    bad = _lib_ac().ref_approx_compare_many(ntip, nnode1, nbin, _p(clade), len(e1), _p(e1), len(es), _p(off),
                                            _p(ne), _p(allE), _p(nn), None, int(cache_size), float(threshold),
                                            int(nthreads), _p(r), None)
    return r[:, 1, :].copy(), int(bad)
