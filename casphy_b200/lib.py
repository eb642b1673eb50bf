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
