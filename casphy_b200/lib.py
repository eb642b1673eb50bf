"""ctypes binding of libcasphy.so (the sm_100a implementation).

The functions mirror the reference tools' computations and return numpy
arrays holding exactly the bytes those tools write (without file headers).
There is no CPU fallback: if libcasphy.so is missing or no GPU is visible the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcasphy.so")
_LIB = None

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class JoinStats(C.Structure):
    _fields_ = [("joins", C.c_uint64), ("stale_recomputes", C.c_uint64), ("pair_scores", C.c_uint64),
                ("compactions", C.c_uint64), ("kernel_launches", C.c_uint64), ("int_path", C.c_uint32),
                ("scan_path", C.c_uint32), ("init_scan_ms", C.c_double), ("join_loop_ms", C.c_double),
                ("total_ms", C.c_double), ("alg_bytes_init", C.c_uint64), ("alg_bytes_join", C.c_uint64),
                ("phases", C.c_uint64), ("refreshes", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ }


class FelModel(C.Structure):
    _fields_ = [("model", C.c_uint32), ("nallele", C.c_uint32), ("kappa", C.c_double),
                ("pi", C.c_double * 4), ("rate", C.c_double), ("allele_freq", C.c_void_p),
                ("mem_budget", C.c_uint64)]


class BloptStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("evaluations", C.c_uint32), ("site_chunks", C.c_uint32),
                ("levels_inside", C.c_uint32), ("levels_outside", C.c_uint32), ("reserved", C.c_uint32),
                ("loglik_start", C.c_double), ("loglik_end", C.c_double), ("seconds", C.c_double),
                ("launches_per_eval", C.c_uint64), ("eval_seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class BootstrapStats(C.Structure):
    _fields_ = [("nrep", C.c_uint32), ("nclade", C.c_uint32), ("prep_ms", C.c_double), ("join_ms", C.c_double),
                ("transfer_ms", C.c_double), ("total_ms", C.c_double), ("kernel_launches", C.c_uint64),
                ("join_phases", C.c_uint64), ("max_ctas_per_rep", C.c_uint32), ("tuned", C.c_uint32),
                ("join_longest_ms", C.c_double), ("join_busy_ms", C.c_double), ("cost_alpha_us", C.c_double),
                ("cost_beta_us", C.c_double), ("cost_gamma_us", C.c_double), ("graph", C.c_uint32),
                ("reserved", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


MODEL_HKY85, MODEL_IRREVERSIBLE = 0, 1
GRAD_ADJOINT, GRAD_CENTRAL_DIFF = 0, 1


class CasphyError(RuntimeError):
    def __init__(self, status, what):
        lib = _LIB
        msg = lib.casphy_strerror(status).decode() if lib else str(status)
        last = lib.casphy_last_error().decode() if lib else ""
        super().__init__(f"{what}: status {status} ({msg}) {last}")
        self.status = status


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `make -C casphy_b200` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        u32, f32, vp = C.c_uint32, C.c_float, C.c_void_p
        L.casphy_strerror.restype = C.c_char_p
        L.casphy_strerror.argtypes = [C.c_int]
        L.casphy_last_error.restype = C.c_char_p
        L.casphy_abi_version.restype = C.c_int
        L.casphy_join_indel.argtypes = [u32, u32, _u32p, u32, _f64p, _u32p, u32, f32, _u32p, _u32p,
                                        C.POINTER(JoinStats)]
        L.casphy_join_indel_dev.argtypes = [u32, u32, vp, u32, _f64p, _u32p, u32, f32, _u32p, vp,
                                            C.POINTER(JoinStats), vp]
        for name in ("casphy_node_keep_indel", "casphy_node_keep_bit"):
            getattr(L, name).argtypes = [u32, u32, _u32p, u32, _u32p, u32, _u32p, u32, _u32p, C.POINTER(u32)]
        L.casphy_radius_bit.argtypes = [u32, u32, _u32p, _f64p, C.c_int32, _u32p, vp, C.c_uint64,
                                        C.POINTER(C.c_uint64)]
        L.casphy_radius_dna.argtypes = [u32, u32, _u32p, u32, _u32p, vp, C.c_uint64, C.POINTER(C.c_uint64)]
        _pp = C.POINTER(C.POINTER(C.c_uint32))
        L.casphy_radius_bit_lists.argtypes = [u32, u32, _u32p, _f64p, C.c_int32, _u32p, _pp, C.POINTER(C.c_uint64)]
        L.casphy_radius_dna_lists.argtypes = [u32, u32, _u32p, u32, _u32p, _pp, C.POINTER(C.c_uint64)]
        L.casphy_free.argtypes = [vp]
        L.casphy_free.restype = None
        L.casphy_radius_bit_rows.argtypes = [u32, u32, _u32p, _f64p, C.c_int32, u32, u32, _u32p, vp, C.c_uint64,
                                             C.POINTER(C.c_uint64)]
        L.casphy_radius_dna_rows.argtypes = [u32, u32, _u32p, u32, u32, u32, _u32p, vp, C.c_uint64,
                                             C.POINTER(C.c_uint64)]
        L.casphy_try_radius_bit.argtypes = [u32, u32, _u32p, _f64p, C.c_int32, u32, _u32p, _u32p]
        L.casphy_try_radius_dna.argtypes = [u32, u32, _u32p, u32, u32, _u32p, _u32p]
        L.casphy_transfer_dis.argtypes = [u32, u32, u32, u32, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p]
        L.casphy_resample_columns.argtypes = [u32, u32, _u32p, u32, _u32p, _u32p]
        L.casphy_felsenstein_loglik.argtypes = [u32, u32, _u32p, _f64p, u32, _u32p, vp, C.POINTER(FelModel),
                                                C.POINTER(C.c_double), vp]
        L.casphy_felsenstein_optimize.argtypes = [u32, u32, _u32p, _f64p, u32, _u32p, vp, C.POINTER(FelModel),
                                                  C.c_int, u32, C.c_double, C.POINTER(BloptStats)]
        L.casphy_bootstrap_bit.argtypes = [u32, u32, _u32p, _u32p, u32, _u32p, _u32p, _f64p, C.c_int, C.c_double,
                                           _u32p, vp, vp, vp, C.POINTER(BootstrapStats)]
        _i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        L.casphy_ancestral_bit.argtypes = [u32, u32, u32, _u32p, u32, _u32p, vp, _u32p]
        L.casphy_ancestral_char.argtypes = [u32, u32, u32, _i32p, u32, _u32p, _u32p, C.c_float, C.c_float, vp, _u32p]
        L.casphy_fasta_encode.argtypes = [u32, u32, C.c_char_p, vp, C.POINTER(u32), vp, C.c_uint64]
        L.casphy_node_des.argtypes = [u32, u32, u32, _u32p, _u32p, _i32p]
        L.casphy_tip_merge.argtypes = [u32, _u32p, vp, C.c_double, _i32p]
        L.casphy_approx_compare.argtypes = [u32, u32, _u32p, u32, _u32p, u32, vp, vp, u32, f32, vp, vp, _i32p]
        L.casphy_cal_abs.argtypes = [u32, u32, _u32p, u32, vp, vp, C.c_double, vp, _i32p]
        if hasattr(L, "casphy_join_bit"):
            L.casphy_join_bit.argtypes = [u32, u32, _u32p, _f64p, C.c_int, _u32p, _u32p, C.POINTER(JoinStats)]
            L.casphy_join_bit_dev.argtypes = [u32, u32, vp, _f64p, C.c_int, _u32p, vp, C.POINTER(JoinStats), vp]
        _LIB = L
    return _LIB


def _chk(st, what):
    if st != 0:
        raise CasphyError(st, what)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def join_indel(codes, nstate, w, tip_size=None, min_size=0, min_ratio=2.0, return_stats=False):
    """joinEdgeIndel on the GPU.  Returns (edge (2N-2, 2), nodeState (N-1, ncol), stats)."""
    codes = _u32(codes)
    ntip, ncol = codes.shape
    w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1)
    ts = _u32(np.ones(ntip) if tip_size is None else tip_size)
    nedge = 2 * ntip - 2
    edge = np.zeros(max(nedge, 1) * 2, dtype=np.uint32)
    state = np.zeros(max(ntip - 1, 1) * ncol, dtype=np.uint32)
    st = JoinStats()
    _chk(lib().casphy_join_indel(ntip, ncol, codes, nstate, w, ts, min_size, min_ratio, edge, state,
                                 C.byref(st)), "casphy_join_indel")
    return edge[: 2 * nedge].reshape(nedge, 2), state.reshape(-1, ncol), st.as_dict()


def join_bit(words, w=None, ancestral_type=1):
    words = _u32(words)
    ntip, nbin = words.shape
    w = np.ones(nbin * 32) if w is None else w
    w = np.ascontiguousarray(w, dtype=np.float64)
    nedge = 2 * ntip - 2
    edge = np.zeros(max(nedge, 1) * 2, dtype=np.uint32)
    state = np.zeros(max(ntip - 1, 1) * nbin, dtype=np.uint32)
    st = JoinStats()
    _chk(lib().casphy_join_bit(ntip, nbin, words, w, ancestral_type, edge, state, C.byref(st)),
         "casphy_join_bit")
    return edge[: 2 * nedge].reshape(nedge, 2), state.reshape(-1, nbin), st.as_dict()


def node_keep(node_state, edge, outmat, cutoff, bit=False):
    """nodeKeepIndel / nodeKeepBit: retained node ids in .retainNode order."""
    node_state, edge, outmat = _u32(node_state), _u32(edge), _u32(outmat)
    nnode, ncol = node_state.shape
    out = np.zeros(max(edge.shape[0], 1), dtype=np.uint32)
    n = C.c_uint32(0)
    f = lib().casphy_node_keep_bit if bit else lib().casphy_node_keep_indel
    om = outmat.reshape(-1) if outmat.size else np.zeros(1, np.uint32)
    _chk(f(nnode, ncol, node_state, edge.shape[0], edge.reshape(-1), outmat.shape[0] if outmat.size else 0, om,
           cutoff, out, C.byref(n)), "casphy_node_keep")
    return out[: n.value].copy()


def _lists(call, ntip):
    """Counts and lists in one search when they fit a guessed buffer (64 per
    row); a second search only when they do not."""
    counts = np.zeros(max(ntip, 1), dtype=np.uint32)
    tot = C.c_uint64(0)
    idx = np.empty(max(64 * ntip, 1 << 16), dtype=np.uint32)
    st = call(counts, idx.ctypes.data_as(C.c_void_p), idx.size, C.byref(tot))
    if st == 2 and tot.value > idx.size:  # CASPHY_ERANGE: the lists need a bigger buffer
        idx = np.empty(tot.value, dtype=np.uint32)
        st = call(counts, idx.ctypes.data_as(C.c_void_p), idx.size, C.byref(tot))
    _chk(st, "casphy_radius")
    return counts[:ntip], (idx if idx.size == tot.value else idx[: tot.value].copy())


def _lists_owned(call, ntip):
    """One search; the lists stay in the library's exact-size host buffer,
    viewed without a copy and released with casphy_free when the array goes."""
    import weakref
    counts = np.zeros(max(ntip, 1), dtype=np.uint32)
    tot = C.c_uint64(0)
    ptr = C.POINTER(C.c_uint32)()
    _chk(call(counts, C.byref(ptr), C.byref(tot)), "casphy_radius")
    n = tot.value
    idx = np.ctypeslib.as_array(ptr, shape=(max(n, 1),))
    weakref.finalize(idx.base, lib().casphy_free, C.cast(ptr, C.c_void_p))
    return counts[:ntip], idx[:n]


def radius_bit(bmat, w, radius):
    """radiusNeighbor: bmat (nrow words, ntip) word-plane-major -> (counts, idx)."""
    bmat = _u32(bmat)
    nrow, ntip = bmat.shape
    w = np.ascontiguousarray(w, dtype=np.float64)
    return _lists_owned(lambda c, p, t: lib().casphy_radius_bit_lists(nrow, ntip, bmat, w, int(radius), c, p, t),
                        ntip)


def radius_dna(raw, radius):
    """radiusNeighborDNA on fasta2bin rows -> (counts, idx)."""
    raw = _u32(raw)
    ntip, nb = raw.shape
    return _lists_owned(lambda c, p, t: lib().casphy_radius_dna_lists(ntip, nb, raw, int(radius), c, p, t), ntip)


def radius_bit_rows(bmat, w, radius, row_begin, row_end):
    """radiusNeighbor lists of query rows [row_begin, row_end) only."""
    bmat = _u32(bmat)
    nrow, ntip = bmat.shape
    w = np.ascontiguousarray(w, dtype=np.float64)
    return _lists(lambda c, i, cap, t: lib().casphy_radius_bit_rows(nrow, ntip, bmat, w, int(radius), row_begin,
                                                                    row_end, c, i, cap, t), row_end - row_begin)


def radius_dna_rows(raw, radius, row_begin, row_end):
    """radiusNeighborDNA lists of query rows [row_begin, row_end) only."""
    raw = _u32(raw)
    ntip, nb = raw.shape
    return _lists(lambda c, i, cap, t: lib().casphy_radius_dna_rows(ntip, nb, raw, int(radius), row_begin, row_end,
                                                                    c, i, cap, t), row_end - row_begin)


def try_radius_bit(bmat, w, radius, qidx):
    bmat, qidx = _u32(bmat), _u32(qidx)
    nrow, ntip = bmat.shape
    counts = np.zeros(len(qidx), dtype=np.uint32)
    _chk(lib().casphy_try_radius_bit(nrow, ntip, bmat, np.ascontiguousarray(w, dtype=np.float64), int(radius),
                                     len(qidx), qidx, counts), "casphy_try_radius_bit")
    return counts


def try_radius_dna(raw, radius, qidx):
    raw, qidx = _u32(raw), _u32(qidx)
    counts = np.zeros(len(qidx), dtype=np.uint32)
    _chk(lib().casphy_try_radius_dna(raw.shape[0], raw.shape[1], raw, int(radius), len(qidx), qidx, counts),
         "casphy_try_radius_dna")
    return counts


def transfer_dis(y, x, ntip):
    """TransferDisStream -> (ymin, ysize, xmin, xsize)."""
    y, x = _u32(y), _u32(x)
    ny, ncol = y.shape
    nx = x.shape[0]
    ymin, ysize = np.zeros(max(ny, 1), np.uint32), np.zeros(max(ny, 1), np.uint32)
    xmin, xsize = np.zeros(max(nx, 1), np.uint32), np.zeros(max(nx, 1), np.uint32)
    _chk(lib().casphy_transfer_dis(ny, nx, ncol, ntip, y, x, ymin, ysize, xmin, xsize), "casphy_transfer_dis")
    return ymin[:ny], ysize[:ny], xmin[:nx], xsize[:nx]


def resample_columns(raw, idx):
    """Felsenstein bootstrap gather: byte idx[4i+j] of every row of the
    fasta2bin body `raw` (ntip x nbin u32) into byte j of word i."""
    raw, idx = _u32(raw), _u32(idx)
    ntip, nbin = raw.shape
    out = np.zeros((ntip, (len(idx) + 3) // 4), np.uint32)
    _chk(lib().casphy_resample_columns(ntip, nbin, raw, len(idx), idx, out), "casphy_resample_columns")
    return out


def _fel_model(model, kappa, pi, rate, nallele, allele_freq, mem_budget):
    m = FelModel()
    m.model = {"hky85": MODEL_HKY85, "irreversible": MODEL_IRREVERSIBLE}[model]
    m.nallele = int(nallele)
    m.kappa = float(kappa)
    for i, v in enumerate(pi):
        m.pi[i] = float(v)
    m.rate = float(rate)
    keep = None
    if allele_freq is not None:
        keep = np.ascontiguousarray(allele_freq, dtype=np.float64)
        m.allele_freq = keep.ctypes.data
    m.mem_budget = int(mem_budget)
    return m, keep


def _fel_args(edge, brlen, codes, weights):
    edge = _u32(edge).reshape(-1, 2)
    brlen = np.ascontiguousarray(brlen, dtype=np.float64)
    codes = _u32(codes)
    ntip, nsite = codes.shape
    wk = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    return edge, brlen, codes, ntip, nsite, wk


def felsenstein_loglik(edge, brlen, codes, model="hky85", kappa=2.0, pi=(0.25, 0.25, 0.25, 0.25), rate=1.0,
                       nallele=1, allele_freq=None, weights=None, grad=False, mem_budget=0):
    """log L of the tree (.edge2 rows, tips 0..ntip-1) and, with grad=True,
    d log L / d brlen by the adjoint pass."""
    edge, brlen, codes, ntip, nsite, wk = _fel_args(edge, brlen, codes, weights)
    m, _keep = _fel_model(model, kappa, pi, rate, nallele, allele_freq, mem_budget)
    ll = C.c_double(0)
    g = np.zeros(len(brlen)) if grad else None
    _chk(lib().casphy_felsenstein_loglik(ntip, len(edge), edge, brlen, nsite, codes,
                                         None if wk is None else wk.ctypes.data, C.byref(m), C.byref(ll),
                                         None if g is None else g.ctypes.data), "casphy_felsenstein_loglik")
    return (ll.value, g) if grad else ll.value


def felsenstein_optimize(edge, brlen, codes, model="hky85", kappa=2.0, pi=(0.25, 0.25, 0.25, 0.25), rate=1.0,
                         nallele=1, allele_freq=None, weights=None, gradient="adjoint", max_iter=200,
                         rel_tol=1e-9, mem_budget=0):
    """L-BFGS branch lengths; returns (optimised brlen, stats dict)."""
    edge, brlen, codes, ntip, nsite, wk = _fel_args(edge, brlen, codes, weights)
    m, _keep = _fel_model(model, kappa, pi, rate, nallele, allele_freq, mem_budget)
    t = brlen.copy()
    st = BloptStats()
    mode = {"adjoint": GRAD_ADJOINT, "central_diff": GRAD_CENTRAL_DIFF}[gradient]
    _chk(lib().casphy_felsenstein_optimize(ntip, len(edge), edge, t, nsite, codes,
                                           None if wk is None else wk.ctypes.data, C.byref(m), mode, max_iter,
                                           rel_tol, C.byref(st)), "casphy_felsenstein_optimize")
    return t, st.as_dict()


def bootstrap_bit(words, full_edge, offsets, cells, weights, ancestral_type=1, threshold=0.05, matrices=True,
                  raw_edges=False):
    """Batched bootstrap: returns dict(support, ymin, ysize, raw_edges, stats)."""
    words = _u32(words)
    ntip, nbin = words.shape
    edge = _u32(full_edge).reshape(-1, 2)
    offsets, cells = _u32(offsets), _u32(cells)
    nrep = len(offsets) - 1
    weights = np.ascontiguousarray(weights, dtype=np.float64).reshape(nrep, nbin * 32)
    nX = ntip - 2
    support = np.zeros(max(nX, 1), np.uint32)
    ymin = np.zeros((nrep, nX), np.uint32) if matrices else None
    ysize = np.zeros((nrep, nX), np.uint32) if matrices else None
    n = np.diff(offsets.astype(np.int64))
    raw = np.zeros(int((4 * (n - 1)).sum()), np.uint32) if raw_edges else None
    st = BootstrapStats()
    ptr = lambda a: None if a is None else a.ctypes.data
    _chk(lib().casphy_bootstrap_bit(ntip, nbin, words, edge, nrep, offsets, cells, weights.reshape(-1),
                                    1 if ancestral_type else 0, float(threshold), support, ptr(ymin), ptr(ysize),
                                    ptr(raw), C.byref(st)), "casphy_bootstrap_bit")
    out = {"support": support[:nX], "ymin": ymin, "ysize": ysize, "stats": st.as_dict()}
    if raw_edges:
        out["raw_edges"] = np.split(raw, np.cumsum(4 * (n - 1))[:-1])
    return out


def ancestral_bit(mat, edge, nnode=None):
    """ancestralBitReverse: (node states nnode x nbin, edge lengths)."""
    mat = _u32(mat)
    ntip, nbin = mat.shape
    edge = _u32(edge).reshape(-1, 2)
    nnode = int(edge.max()) + 1 - ntip if nnode is None else int(nnode)
    state = np.zeros((nnode, nbin), np.uint32)
    ln = np.zeros(len(edge), np.uint32)
    _chk(lib().casphy_ancestral_bit(ntip, nnode, nbin, mat, len(edge), edge.reshape(-1), state.ctypes.data, ln),
         "casphy_ancestral_bit")
    return state, ln


def ancestral_char(mat, edge, tip_size=None, min_size=0.0, min_ratio=0.0, nnode=None):
    """charAncestralEC on int32 states (-1 unknown): (node states, edge lengths)."""
    mat = np.ascontiguousarray(mat, dtype=np.int32)
    ntip, nsite = mat.shape
    edge = _u32(edge).reshape(-1, 2)
    nnode = int(edge.max()) + 1 - ntip if nnode is None else int(nnode)
    tips = _u32(np.ones(ntip) if tip_size is None else tip_size)
    state = np.zeros((nnode, nsite), np.int32)
    ln = np.zeros(len(edge), np.uint32)
    _chk(lib().casphy_ancestral_char(ntip, nnode, nsite, mat, len(edge), edge.reshape(-1), tips, float(min_size),
                                     float(min_ratio), state.ctypes.data, ln), "casphy_ancestral_char")
    return state, ln


def tip_merge(counts, idx, pshared):
    """tipMerge: .member categories from radius lists (counts, concatenated idx)."""
    counts = _u32(counts)
    idx = _u32(idx)
    member = np.zeros(max(len(counts), 1), np.int32)
    _chk(lib().casphy_tip_merge(len(counts), counts, idx.ctypes.data if idx.size else None, float(pshared), member),
         "casphy_tip_merge")
    return member[: len(counts)]


def node_des(edge, ntip, nnode=None):
    """nodeDesBig: (clade rows (nnode-1) x nbin in file order, sizes as returned)."""
    edge = _u32(edge).reshape(-1, 2)
    nnode = int(edge.max()) + 1 - ntip if nnode is None else int(nnode)
    nbin = (ntip - 1) // 32 + 1
    rows = np.zeros((max(nnode - 1, 1), nbin), np.uint32)
    sizes = np.zeros(max(nnode - 1, 1), np.int32)
    _chk(lib().casphy_node_des(ntip, nnode, len(edge), edge.reshape(-1), rows, sizes), "casphy_node_des")
    return rows[: nnode - 1], sizes[: nnode - 1]


def _query_trees(edges2):
    es = [_u32(np.asarray(e)).reshape(-1, 2) for e in edges2]
    off = np.zeros(len(es) + 1, np.uint64)
    off[1:] = np.cumsum([len(e) for e in es])
    flat = np.ascontiguousarray(np.concatenate(es) if es else np.zeros((1, 2), np.uint32), dtype=np.uint32)
    return es, off, flat


def approx_compare(clade_rows, ntip, edge1, edges2, cache_size=8192, threshold=0.1):
    """approximateCompare2_AVX2 of each query tree (0-based cladewise edges)
    against the reference tree (edge1, clade rows from node_des).  Returns
    (ref2qry list of nnode1 x 2, qry2ref list of nnode2 x 3, status array)."""
    clade = _u32(clade_rows)
    nnode1 = clade.shape[0] + 1
    e1 = _u32(edge1).reshape(-1, 2)
    es, off, flat = _query_trees(edges2)
    nt = len(es)
    nn2 = [len(e) - ntip + 1 for e in es]
    r = np.zeros((max(nt, 1), nnode1, 2), np.int32)
    q = np.zeros((max(sum(nn2), 1), 3), np.int32)
    status = np.zeros(max(nt, 1), np.int32)
    _chk(lib().casphy_approx_compare(ntip, nnode1, clade.reshape(-1), len(e1), e1.reshape(-1), nt, off.ctypes.data,
                                     flat.ctypes.data, int(cache_size), float(threshold), r.ctypes.data,
                                     q.ctypes.data, status), "casphy_approx_compare")
    qs, o = [], 0
    for n in nn2:
        qs.append(q[o:o + n].copy())
        o += n
    return [r[t].copy() for t in range(nt)], qs, status[:nt].copy()


def cal_abs(edge1, ntip, edges2, threshold=0.05):
    """cal.abs: (support, node_size) of every internal node of the reference
    tree (0-based cladewise edges) over the query trees."""
    e1 = _u32(edge1).reshape(-1, 2)
    nnode1 = len(e1) - ntip + 1
    es, off, flat = _query_trees(edges2)
    sup = np.zeros(nnode1, np.float64)
    size = np.zeros(nnode1, np.int32)
    _chk(lib().casphy_cal_abs(ntip, len(e1), e1.reshape(-1), len(es), off.ctypes.data, flat.ctypes.data,
                              float(threshold), sup.ctypes.data, size), "casphy_cal_abs")
    return sup, size


def fasta_encode(seqs):
    """fasta2bin's column classification and encoding of equal-length
    sequences (bytes or str): (variable flags u8[len], .bin body u32 rows)."""
    rows = [x.encode() if isinstance(x, str) else bytes(x) for x in seqs]
    nseq, length = len(rows), len(rows[0])
    buf = b"".join(rows)
    var = np.zeros(length, np.uint8)
    nkeep = C.c_uint32(0)
    out = np.zeros(max(nseq * ((length + 3) // 4), 1), np.uint32)
    _chk(lib().casphy_fasta_encode(nseq, length, buf, var.ctypes.data, C.byref(nkeep), out.ctypes.data, out.size),
         "casphy_fasta_encode")
    nw = (nkeep.value + 3) // 4
    return var, out[: nseq * nw].reshape(nseq, nw)
