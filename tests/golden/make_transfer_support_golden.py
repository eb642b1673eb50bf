"""Golden fixtures for the clade matching approximateCompare2_AVX2 and the
transfer support cal.abs builds from it, produced by the reference's own
functions (src/functions.cpp: approximateCompare2_AVX2 in
oracle/_ref/libcputwin_ref.so, nodeDesBig in oracle/_ref/libparsimony_ref.so;
make -C oracle ref).

    python tests/golden/make_transfer_support_golden.py   # writes transfer_support_reference.npz

Cases: a greedy-join reference tree against join trees of column-resampled
data (the bootstrap use), multifurcating trees against collapsed and
unrelated ones, Yule trees against unrelated Yule trees at a wide threshold,
and a cache too small for some of the query trees.  Per case the fixture
holds the trees (0-based cladewise edges), the nodeDesBig clade rows and
sizes of the reference tree, and per query tree and threshold the two
matrices the function returns (or the out-of-cache flag).  The cal.abs
support column is derived from them as R does (distance / node size <=
threshold, averaged over trees) by the tests.
"""
import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), HERE]

from casphy_b200 import synth  # noqa: E402
from make_parsimony_golden import collapse, preorder, relabel  # noqa: E402


def node_des_ref(edge, ntip):
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libparsimony_ref.so"))
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    lib.ref_node_des_big.argtypes = [C.c_uint32] * 3 + [u32p, C.c_char_p, C.c_int, i32p]
    nnode = len(edge) - ntip + 1
    sizes = np.zeros(max(nnode - 1, 1), np.int32)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "clades.bk")
        lib.ref_node_des_big(ntip, nnode, len(edge), np.ascontiguousarray(edge.reshape(-1), dtype=np.uint32),
                             path.encode(), 0, sizes)
        rows = np.fromfile(path, dtype=np.uint32)
    nbin = (ntip - 1) // 32 + 1
    return rows.reshape(nnode - 1, nbin), sizes[: nnode - 1]


def peak_open(edge, ntip):
    """Most open rows the reference's cache holds for this query tree."""
    open_, n, peak = set(), 0, 0
    for p, c in np.asarray(edge)[::-1]:
        if p not in open_:
            open_.add(p)
            n += 1
            peak = max(peak, n)
        if c >= ntip:
            open_.discard(c)
            n -= 1
    return peak


def resampled_join(words, rng):
    import oracle as O
    nsite = words.shape[1] * 32
    bits = np.unpackbits(words.view(np.uint8), axis=1, bitorder="little")[:, :nsite]
    cols = rng.integers(0, nsite, nsite)
    wb = np.ascontiguousarray(np.packbits(bits[:, cols], axis=1, bitorder="little")).view(np.uint32)
    e, _, _ = O.join_bit(np.ascontiguousarray(wb), None, 1)
    return np.ascontiguousarray(e, dtype=np.uint32)


def yule(ntip, rng, frac=0.0):
    par, ch, _ = synth.yule_tree(ntip, 0.1, rng)
    e = preorder(par, ch, ntip)
    if frac:
        e = collapse(e, ntip, frac, rng)
    return np.ascontiguousarray(relabel(e, ntip)[0], dtype=np.uint32)


def main():
    import oracle as O
    import cputwin as T
    rng = np.random.default_rng(77)
    res = {}

    def case(name, ntip, ref, queries, thresholds, cache=8192):
        rows, sizes = node_des_ref(ref, ntip)
        res[f"{name}/ntip"] = np.array([ntip, cache], np.uint32)
        res[f"{name}/ref"] = ref
        res[f"{name}/rows"] = rows
        res[f"{name}/sizes"] = sizes
        res[f"{name}/thr"] = np.array(thresholds, np.float64)
        for q, e in enumerate(queries):
            res[f"{name}/q{q}/edge"] = e
            for k, thr in enumerate(thresholds):
                try:
                    r2q, q2r = T.approx_compare(rows, ntip, ref, e, cache_size=cache, threshold=thr)
                    res[f"{name}/q{q}/t{k}/ref2qry"] = r2q
                    res[f"{name}/q{q}/t{k}/qry2ref"] = q2r
                except RuntimeError:
                    res[f"{name}/q{q}/t{k}/out_of_cache"] = np.array([1], np.uint8)

    words = synth.binary_workload(600, 256, 12, 0.04, 0.05, seed=31)
    ref, _, _ = O.join_bit(words, None, 1)
    ref = np.ascontiguousarray(ref, dtype=np.uint32)
    boot = [resampled_join(words, rng) for _ in range(5)]
    # cal.abs passes threshold + 0.05 as binary32: 0.05 -> 0.1, 0.3 -> 0.35
    case("join600", 600, ref, boot, [float(np.float32(0.05 + 0.05)), float(np.float32(0.3 + 0.05))])
    m = yule(400, rng, 0.4)
    mq = [m, np.ascontiguousarray(relabel(collapse(m, 400, 0.3, rng), 400)[0], dtype=np.uint32),
          yule(400, rng, 0.4), yule(400, rng)]
    case("multi400", 400, m, mq, [0.1, 0.25])
    y = yule(300, rng)
    case("yule300", 300, y, [yule(300, rng) for _ in range(3)], [0.55])
    peaks = sorted(peak_open(e, 600) for e in boot)
    case("cache600", 600, ref, boot, [0.1], cache=peaks[len(peaks) // 2])
    out = os.path.join(HERE, "transfer_support_reference.npz")
    np.savez_compressed(out, **res)
    print(f"wrote {out} ({len(res)} arrays)")


if __name__ == "__main__":
    main()
