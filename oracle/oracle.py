"""ctypes binding of the CPU oracle (oracle.c) -- TEST INFRASTRUCTURE.

Imported only by tests/, __graft_entry__.smoke() (as the checker) and
bench.py's CPU legs.  Builds liboracle.so with `make -C oracle` when it is
missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = C.CDLL(path)
        u32, i32, f32, i = C.c_uint32, C.c_int32, C.c_float, C.c_int
        L.oracle_f64_to_f16.argtypes = [C.c_double]
        L.oracle_f64_to_f16.restype = C.c_uint16
        L.oracle_f16_to_f64.argtypes = [C.c_uint16]
        L.oracle_f16_to_f64.restype = C.c_double
        L.oracle_f16_add.argtypes = [C.c_uint16, C.c_uint16]
        L.oracle_f16_add.restype = C.c_uint16
        L.oracle_join_indel.argtypes = [u32, u32, _u32p, u32, _f64p, _u32p, u32, f32,
                                        _u32p, _u32p, _u64p, i]
        L.oracle_join_indel_phased.argtypes = [u32, u32, _u32p, u32, _f64p, _u32p, u32, f32, u32, i, u32,
                                               _u32p, _u32p, _u64p, i]
        L.oracle_join_bit.argtypes = [u32, u32, _u32p, _f64p, i, _u32p, _u32p, _u64p, i]
        L.oracle_join_bit_phased.argtypes = [u32, u32, _u32p, _f64p, i, u32, i, u32, _u32p, _u32p, _u64p, i]
        for name in ("oracle_node_keep_indel", "oracle_node_keep_bit"):
            getattr(L, name).argtypes = [u32, u32, _u32p, u32, _u32p, u32, _u32p, u32,
                                         _u32p, C.POINTER(u32)]
        L.oracle_radius_bit.argtypes = [u32, u32, _u32p, _f64p, i32, _u32p, C.c_void_p,
                                        C.c_uint64, C.POINTER(C.c_uint64), i]
        L.oracle_radius_dna.argtypes = [u32, u32, _u32p, u32, _u32p, C.c_void_p,
                                        C.c_uint64, C.POINTER(C.c_uint64), i]
        L.oracle_try_radius_bit.argtypes = [u32, u32, _u32p, _f64p, i32, u32, _u32p, _u32p, i]
        L.oracle_try_radius_dna.argtypes = [u32, u32, _u32p, u32, u32, _u32p, _u32p, i]
        L.oracle_transfer_dis.argtypes = [u32, u32, u32, u32, _u32p, _u32p, _u32p, _u32p,
                                          _u32p, _u32p, i]
        _LIB = L
    return _LIB


def _chk(st, what):
    if st != 0:
        raise RuntimeError(f"oracle {what} failed with status {st}")


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def join_indel(codes, nstate, w, tip_size=None, min_size=0, min_ratio=2.0, nthreads=0):
    codes = _u32(codes)
    ntip, ncol = codes.shape
    w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
    ts = _u32(np.ones(ntip) if tip_size is None else tip_size)
    nedge = 2 * ntip - 2
    edge = np.zeros(max(nedge, 1) * 2, dtype=np.uint32)
    state = np.zeros(max(ntip - 1, 1) * ncol, dtype=np.uint32)
    stats = np.zeros(3, dtype=np.uint64)
    _chk(lib().oracle_join_indel(ntip, ncol, codes, nstate, w, ts, min_size, min_ratio,
                                 edge, state, stats, nthreads or os.cpu_count()), "join_indel")
    return edge[: 2 * nedge].reshape(nedge, 2), state.reshape(-1, ncol), stats


def join_indel_phased(codes, nstate, w, tip_size=None, min_size=0, min_ratio=2.0, max_batch=8, pair_joins=True,
                      table_ctas=0, nthreads=0, ride=False):
    """The indel join in phases (oracle_join_indel_phased); stats adds
    [3] phases, [4] phases with two joins, [5] pairs a top-2 table over
    `table_ctas` ranges could not vouch for and [6] joins made in a rescan
    phase because the best fresh record was still the decision after the
    rescans (`ride`)."""
    codes = _u32(codes)
    ntip, ncol = codes.shape
    w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
    ts = _u32(np.ones(ntip) if tip_size is None else tip_size)
    nedge = 2 * ntip - 2
    edge = np.zeros(max(nedge, 1) * 2, dtype=np.uint32)
    state = np.zeros(max(ntip - 1, 1) * ncol, dtype=np.uint32)
    stats = np.zeros(7, dtype=np.uint64)
    _chk(lib().oracle_join_indel_phased(ntip, ncol, codes, nstate, w, ts, min_size, min_ratio, max_batch,
                                        (1 if pair_joins else 0) | (2 if ride else 0), table_ctas, edge, state, stats,
                                        nthreads or os.cpu_count()),
         "join_indel_phased")
    return edge[: 2 * nedge].reshape(nedge, 2), state.reshape(-1, ncol), stats


def join_bit(words, w=None, ancestral_type=1, nthreads=0):
    words = _u32(words)
    ntip, nbin = words.shape
    w = np.ones(nbin * 32) if w is None else w
    w = np.ascontiguousarray(w, dtype=np.float64)
    nedge = 2 * ntip - 2
    edge = np.zeros(max(nedge, 1) * 2, dtype=np.uint32)
    state = np.zeros(max(ntip - 1, 1) * nbin, dtype=np.uint32)
    stats = np.zeros(3, dtype=np.uint64)
    _chk(lib().oracle_join_bit(ntip, nbin, words, w, ancestral_type, edge, state, stats,
                               nthreads or os.cpu_count()), "join_bit")
    return edge[: 2 * nedge].reshape(nedge, 2), state.reshape(-1, nbin), stats


def node_keep(node_state, edge, outmat, cutoff, bit=False):
    node_state, edge, outmat = _u32(node_state), _u32(edge), _u32(outmat)
    nnode, ncol = node_state.shape
    out = np.zeros(max(edge.shape[0], 1), dtype=np.uint32)
    n = C.c_uint32(0)
    f = lib().oracle_node_keep_bit if bit else lib().oracle_node_keep_indel
    _chk(f(nnode, ncol, node_state, edge.shape[0], edge.reshape(-1), outmat.shape[0],
           outmat.reshape(-1) if outmat.size else np.zeros(1, np.uint32), cutoff, out,
           C.byref(n)), "node_keep")
    return out[: n.value].copy()


def radius_bit(bmat, w, radius, nthreads=0):
    """bmat: (nrow words, ntip) word-plane-major.  Returns (counts, idx)."""
    bmat = _u32(bmat)
    nrow, ntip = bmat.shape
    w = np.ascontiguousarray(w, dtype=np.float64)
    counts = np.zeros(ntip, dtype=np.uint32)
    tot = C.c_uint64(0)
    L = lib()
    nt = nthreads or os.cpu_count()
    _chk(L.oracle_radius_bit(nrow, ntip, bmat, w, radius, counts, None, 0, C.byref(tot), nt), "radius")
    idx = np.zeros(max(tot.value, 1), dtype=np.uint32)
    _chk(L.oracle_radius_bit(nrow, ntip, bmat, w, radius, counts, idx.ctypes.data_as(C.c_void_p),
                             tot.value, C.byref(tot), nt), "radius")
    return counts, idx[: tot.value]


def radius_dna(raw, radius, nthreads=0):
    raw = _u32(raw)
    ntip, nb = raw.shape
    counts = np.zeros(ntip, dtype=np.uint32)
    tot = C.c_uint64(0)
    L = lib()
    nt = nthreads or os.cpu_count()
    _chk(L.oracle_radius_dna(ntip, nb, raw, radius, counts, None, 0, C.byref(tot), nt), "radius_dna")
    idx = np.zeros(max(tot.value, 1), dtype=np.uint32)
    _chk(L.oracle_radius_dna(ntip, nb, raw, radius, counts, idx.ctypes.data_as(C.c_void_p),
                             tot.value, C.byref(tot), nt), "radius_dna")
    return counts, idx[: tot.value]


def try_radius_bit(bmat, w, radius, qidx, nthreads=0):
    bmat, qidx = _u32(bmat), _u32(qidx)
    nrow, ntip = bmat.shape
    counts = np.zeros(len(qidx), dtype=np.uint32)
    _chk(lib().oracle_try_radius_bit(nrow, ntip, bmat, np.ascontiguousarray(w, dtype=np.float64),
                                     radius, len(qidx), qidx, counts, nthreads or os.cpu_count()),
         "try_radius")
    return counts


def try_radius_dna(raw, radius, qidx, nthreads=0):
    raw, qidx = _u32(raw), _u32(qidx)
    counts = np.zeros(len(qidx), dtype=np.uint32)
    _chk(lib().oracle_try_radius_dna(raw.shape[0], raw.shape[1], raw, radius, len(qidx), qidx,
                                     counts, nthreads or os.cpu_count()), "try_radius_dna")
    return counts


def transfer_dis(y, x, ntip, nthreads=0):
    y, x = _u32(y), _u32(x)
    ny, ncol = y.shape
    nx = x.shape[0]
    ymin, ysize = np.zeros(ny, np.uint32), np.zeros(ny, np.uint32)
    xmin, xsize = np.zeros(nx, np.uint32), np.zeros(nx, np.uint32)
    _chk(lib().oracle_transfer_dis(ny, nx, ncol, ntip, y, x, ymin, ysize, xmin, xsize,
                                   nthreads or os.cpu_count()), "transfer_dis")
    return ymin, ysize, xmin, xsize


def ancestral_bit(mat, edge, nnode=None):
    mat = _u32(mat)
    ntip, nbin = mat.shape
    edge = _u32(edge).reshape(-1, 2)
    nnode = int(edge.max()) + 1 - ntip if nnode is None else int(nnode)
    state = np.zeros((nnode, nbin), np.uint32)
    bis = np.zeros((nnode, nbin), np.uint32)
    ln = np.zeros(len(edge), np.uint32)
    L = lib()
    _chk(L.oracle_ancestral_bit(C.c_uint32(ntip), C.c_uint32(nnode), C.c_uint32(nbin),
                                mat.ctypes.data_as(C.c_void_p), C.c_uint32(len(edge)),
                                np.ascontiguousarray(edge.reshape(-1)).ctypes.data_as(C.c_void_p),
                                state.ctypes.data_as(C.c_void_p), bis.ctypes.data_as(C.c_void_p),
                                ln.ctypes.data_as(C.c_void_p)), "ancestral_bit")
    return state, ln


def ancestral_char(mat, edge, tip_size=None, min_size=0.0, min_ratio=0.0, nnode=None):
    mat = np.ascontiguousarray(mat, dtype=np.int32)
    ntip, nsite = mat.shape
    edge = _u32(edge).reshape(-1, 2)
    nnode = int(edge.max()) + 1 - ntip if nnode is None else int(nnode)
    tips = _u32(np.ones(ntip) if tip_size is None else tip_size)
    state = np.zeros((nnode, nsite), np.int32)
    ln = np.zeros(len(edge), np.uint32)
    L = lib()
    _chk(L.oracle_ancestral_char(C.c_uint32(ntip), C.c_uint32(nnode), C.c_uint32(nsite),
                                 mat.ctypes.data_as(C.c_void_p), C.c_uint32(len(edge)),
                                 np.ascontiguousarray(edge.reshape(-1)).ctypes.data_as(C.c_void_p),
                                 tips.ctypes.data_as(C.c_void_p), C.c_float(min_size),
                                 C.c_float(min_ratio), state.ctypes.data_as(C.c_void_p),
                                 ln.ctypes.data_as(C.c_void_p)), "ancestral_char")
    return state, ln


def tip_merge(counts, idx, pshared):
    counts = _u32(counts)
    idx = _u32(idx)
    member = np.zeros(max(len(counts), 1), np.int32)
    _chk(lib().oracle_tip_merge(C.c_uint32(len(counts)), counts.ctypes.data_as(C.c_void_p),
                                idx.ctypes.data_as(C.c_void_p), C.c_double(pshared),
                                member.ctypes.data_as(C.c_void_p)), "tip_merge")
    return member[: len(counts)]


def node_des(edge, ntip, nnode=None):
    edge = _u32(edge).reshape(-1, 2)
    nnode = int(edge.max()) + 1 - ntip if nnode is None else int(nnode)
    nbin = (ntip - 1) // 32 + 1
    rows = np.zeros((max(nnode - 1, 1), nbin), np.uint32)
    sizes = np.zeros(max(nnode - 1, 1), np.int32)
    _chk(lib().oracle_node_des(C.c_uint32(ntip), C.c_uint32(nnode), C.c_uint32(len(edge)),
                               np.ascontiguousarray(edge.reshape(-1)).ctypes.data_as(C.c_void_p),
                               rows.ctypes.data_as(C.c_void_p), sizes.ctypes.data_as(C.c_void_p)), "node_des")
    return rows[: nnode - 1], sizes[: nnode - 1]


def approx_compare(clade_rows, ntip, edge1, edge2, nnode2=None, cache_size=8192, threshold=0.1):
    """approximateCompare2_AVX2 restated: clade_rows = the reference tree's
    nodeDesBig rows ((nnode1 - 1) x nbin), edges 0-based cladewise.  Returns
    (ref2qry nnode1 x 2, qry2ref nnode2 x 3) as the reference's matrices."""
    clade = _u32(clade_rows)
    nnode1, nbin = clade.shape[0] + 1, clade.shape[1]
    e1 = _u32(np.asarray(edge1).reshape(-1, 2))
    e2 = _u32(np.asarray(edge2).reshape(-1, 2))
    nnode2 = int(e2.max()) + 1 - ntip if nnode2 is None else int(nnode2)
    r = np.zeros((nnode1, 2), np.int32)
    q = np.zeros((nnode2, 3), np.int32)
    P = C.c_void_p
    f = lib().oracle_approx_compare
    f.argtypes = [C.c_uint32] * 3 + [P, C.c_uint32, P, C.c_uint32, P, C.c_uint32, C.c_uint32, C.c_float, P, P]
    f.restype = C.c_int
    _chk(f(ntip, nnode1, nbin, clade.ctypes.data_as(P), len(e1), e1.ctypes.data_as(P), len(e2),
           e2.ctypes.data_as(P), nnode2, int(cache_size), float(threshold), r.ctypes.data_as(P),
           q.ctypes.data_as(P)), "approx_compare")
    return r, q


def join_bit_phased(words, w=None, ancestral_type=1, max_batch=8, pair_joins=True, table_ctas=0, nthreads=0,
                    ride=False):
    """The bit join in phases (oracle_join_bit_phased); stats adds [3] phases,
    [4] phases with two joins, [5] pairs a top-2 table over `table_ctas`
    ranges could not vouch for and [6] joins made in a rescan phase
    (`ride`)."""
    words = _u32(words)
    ntip, nbin = words.shape
    w = np.ones(nbin * 32) if w is None else w
    w = np.ascontiguousarray(w, dtype=np.float64)
    nedge = 2 * ntip - 2
    edge = np.zeros(max(nedge, 1) * 2, dtype=np.uint32)
    state = np.zeros(max(ntip - 1, 1) * nbin, dtype=np.uint32)
    stats = np.zeros(7, dtype=np.uint64)
    _chk(lib().oracle_join_bit_phased(ntip, nbin, words, w, ancestral_type, max_batch,
                                      (1 if pair_joins else 0) | (2 if ride else 0),
                                      table_ctas, edge, state, stats, nthreads or os.cpu_count()), "join_bit_phased")
    return edge[: 2 * nedge].reshape(nedge, 2), state.reshape(-1, nbin), stats


def _fel_edge(edge):
    e = _u32(edge).reshape(-1, 2)
    return e, e.shape[0]


def loglik_hky85(edge, t, codes, kappa, pi, weights=None, nthreads=0):
    """FP64 HKY85 log-likelihood (oracle_loglik_hky85); codes: (ntip, nsite)
    fasta2bin nibbles, edge (nedge, 2) parent/child."""
    e, ne = _fel_edge(edge)
    codes = _u32(codes)
    ntip, nsite = codes.shape
    ll = C.c_double(0)
    t = np.ascontiguousarray(t, dtype=np.float64)
    pi = np.ascontiguousarray(pi, dtype=np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    L = lib()
    L.oracle_loglik_hky85.argtypes = [C.c_uint32, C.c_uint32, _u32p, _f64p, C.c_uint32, _u32p, C.c_void_p,
                                      C.c_double, _f64p, C.POINTER(C.c_double), C.c_int]
    _chk(L.oracle_loglik_hky85(ntip, ne, e.reshape(-1), t, nsite, codes, None if w is None else w.ctypes.data,
                               kappa, pi, C.byref(ll), nthreads or os.cpu_count()), "loglik_hky85")
    return ll.value


def tip_allele_freqs(codes, nallele):
    """Per-site allele frequencies from the tips' allele counts, uniform over
    the nallele alleles where a site has none (the library's default):
    (nsite, nallele + 1), column 0 unused."""
    codes = np.asarray(codes)
    nsite = codes.shape[1]
    q = np.zeros((nsite, nallele + 1))
    for s in range(nsite):
        col = codes[:, s].astype(np.int64)
        cnt = np.bincount(col[col >= 2] - 1, minlength=nallele + 1)[: nallele + 1].astype(np.float64)
        tot = cnt[1:].sum()
        q[s, 1:] = cnt[1:] / tot if tot > 0 else 1.0 / nallele
    return q


def loglik_irreversible(edge, t, codes, nallele, q, rate, weights=None, nthreads=0):
    """FP64 irreversible-edit log-likelihood in the compact form
    (oracle_loglik_irreversible); codes: (ntip, nsite) .tbmat codes."""
    e, ne = _fel_edge(edge)
    codes = _u32(codes)
    ntip, nsite = codes.shape
    ll = C.c_double(0)
    t = np.ascontiguousarray(t, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    assert q.shape == (nsite, nallele + 1)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    L = lib()
    L.oracle_loglik_irreversible.argtypes = [C.c_uint32, C.c_uint32, _u32p, _f64p, C.c_uint32, _u32p, C.c_void_p,
                                             C.c_uint32, _f64p, C.c_double, C.POINTER(C.c_double), C.c_int]
    _chk(L.oracle_loglik_irreversible(ntip, ne, e.reshape(-1), t, nsite, codes,
                                      None if w is None else w.ctypes.data, nallele, q, rate, C.byref(ll),
                                      nthreads or os.cpu_count()), "loglik_irreversible")
    return ll.value
