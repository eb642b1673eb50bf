"""Golden fixtures for the parsimony edge lengths (ancestralBitReverse,
charAncestralEC of src/functions.cpp) and the clade rows of nodeDesBig,
produced by the reference's own functions compiled into
oracle/_ref/libparsimony_ref.so (make -C oracle ref).

    python tests/golden/make_parsimony_golden.py   # writes parsimony_reference.npz

Cases: seeded bit and indel matrices on greedy-join trees, Yule trees and
multifurcating trees (internal edges collapsed, so the child order of the
bottom-up pass matters), with unit and uneven tip sizes and both size rules.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

from casphy_b200 import synth  # noqa: E402


def preorder(par, ch, ntip):
    """Edges re-listed in DFS pre-order from the root (an ape cladewise edge matrix)."""
    par, ch = np.asarray(par), np.asarray(ch)
    kids = {}
    for p, c in zip(par, ch):
        kids.setdefault(int(p), []).append(int(c))
    isc = set(int(c) for c in ch)
    root = [int(p) for p in par if int(p) not in isc][0]
    out, stack = [], [root]
    while stack:
        v = stack.pop()
        for c in reversed(kids.get(v, [])):
            out.append((v, c))
            stack.append(c)
    return np.array(out, dtype=np.uint32)


def relabel(edge, ntip):
    """Internal nodes renumbered ntip, ntip+1, ... in order of first appearance (root first)."""
    m, nxt = {}, ntip
    out = edge.copy()
    for i, (p, c) in enumerate(edge):
        for j, v in ((0, p), (1, c)):
            if v >= ntip:
                if v not in m:
                    m[v] = nxt
                    nxt += 1
                out[i, j] = m[v]
    return out, nxt - ntip


def collapse(edge, ntip, frac, rng):
    """Collapse a fraction of internal edges (children join the grandparent)."""
    edge = [tuple(map(int, e)) for e in edge]
    parent = {c: p for p, c in edge}
    internal = [c for p, c in edge if c >= ntip]
    drop = set(rng.choice(internal, size=int(frac * len(internal)), replace=False).tolist()) if internal else set()

    def up(v):
        while v in drop:
            v = parent[v]
        return v
    new = [(up(p), c) for p, c in edge if c not in drop]
    return preorder([p for p, _ in new], [c for _, c in new], ntip)


def trees(ntip, rng, kind):
    if kind == "yule":
        par, ch, _ = synth.yule_tree(ntip, 0.1, rng)
        e = preorder(par, ch, ntip)
    elif kind == "multi":
        par, ch, _ = synth.yule_tree(ntip, 0.1, rng)
        e = collapse(preorder(par, ch, ntip), ntip, 0.4, rng)
    else:
        raise ValueError(kind)
    return relabel(e, ntip)


def main():
    import oracle as O
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libparsimony_ref.so"))
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    lib.ref_ancestral_bit.argtypes = [C.c_uint32] * 3 + [u32p, C.c_uint32, u32p, u32p, u32p]
    lib.ref_ancestral_char.argtypes = [C.c_uint32] * 3 + [i32p, C.c_uint32, u32p, u32p, C.c_float, C.c_float,
                                                           i32p, u32p]
    lib.ref_node_des_big.argtypes = [C.c_uint32] * 3 + [u32p, C.c_char_p, C.c_int, i32p]

    def node_des(edge, ntip, nnode, name):
        import tempfile
        sizes = np.zeros(max(nnode - 1, 1), np.int32)
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "clades.bin")
            lib.ref_node_des_big(ntip, nnode, len(edge), np.ascontiguousarray(edge.reshape(-1)), path.encode(), 1,
                                 sizes)
            raw = np.fromfile(path, dtype=np.uint32)
        res[f"nd/{name}/edge"] = edge
        res[f"nd/{name}/ntip"] = np.array([ntip, nnode], np.uint32)
        res[f"nd/{name}/file"] = raw
        res[f"nd/{name}/sizes"] = sizes[: nnode - 1]
    rng = np.random.default_rng(2024)
    res = {}
    # bit matrices
    for name, ntip, nbin, kind in (("b50y", 50, 1, "yule"), ("b300m", 300, 3, "multi"), ("b1000j", 1000, 16, "join"),
                                   ("b700m", 700, 5, "multi")):
        words = synth.binary_workload(ntip, nbin * 32, 12, 0.05, 0.05, seed=int(rng.integers(1 << 30)))
        if kind == "join":
            e0, _, _ = O.join_bit(words, None, 1)
            edge, nnode = np.ascontiguousarray(e0, dtype=np.uint32), ntip - 1
        else:
            edge, nnode = trees(ntip, rng, kind)
        state = np.zeros(nnode * nbin, np.uint32)
        ln = np.zeros(len(edge), np.uint32)
        lib.ref_ancestral_bit(ntip, nnode, nbin, np.ascontiguousarray(words), len(edge),
                              np.ascontiguousarray(edge.reshape(-1)), state, ln)
        res[f"pb/{name}/words"] = words
        res[f"pb/{name}/edge"] = edge
        res[f"pb/{name}/nnode"] = np.array([nnode], np.uint32)
        res[f"pb/{name}/state"] = state.reshape(nnode, nbin)
        res[f"pb/{name}/len"] = ln
        node_des(edge, ntip, nnode, name)
    # indel matrices (raw states: -1 missing, 0 unedited, alleles >= 1)
    for name, ntip, nsite, kind, ms, mr, uneven in (("c60y", 60, 40, "yule", 0.0, 0.0, False),
                                                   ("c500m", 500, 128, "multi", 0.0, 0.0, False),
                                                   ("c800j", 800, 96, "join", 0.0, 0.0, False),
                                                   ("c400r", 400, 64, "multi", 10.0, 2.0, True)):
        raw = synth.lineage_states(ntip, nsite, 12, 0.05, 16, 1.5, 0.1, seed=int(rng.integers(1 << 30)))
        if kind == "join":
            codes, ns = synth.regularize(raw)
            e0, _, _ = O.join_indel(codes, ns, np.ones((ns, nsite)))
            edge, nnode = np.ascontiguousarray(e0, dtype=np.uint32), ntip - 1
        else:
            edge, nnode = trees(ntip, rng, kind)
        tips = (rng.integers(1, 30, size=ntip) if uneven else np.ones(ntip)).astype(np.uint32)
        mat = np.ascontiguousarray(raw, dtype=np.int32)
        state = np.zeros(nnode * nsite, np.int32)
        ln = np.zeros(len(edge), np.uint32)
        lib.ref_ancestral_char(ntip, nnode, nsite, mat, len(edge), np.ascontiguousarray(edge.reshape(-1)), tips,
                               ms, mr, state, ln)
        res[f"pc/{name}/mat"] = mat
        res[f"pc/{name}/edge"] = edge
        res[f"pc/{name}/nnode"] = np.array([nnode], np.uint32)
        res[f"pc/{name}/tips"] = tips
        res[f"pc/{name}/rule"] = np.array([ms, mr], np.float32)
        res[f"pc/{name}/state"] = state.reshape(nnode, nsite)
        res[f"pc/{name}/len"] = ln
    for name, ntip in (("y3000", 3000), ("y33", 33)):
        edge, nnode = trees(ntip, rng, "yule")
        node_des(edge, ntip, nnode, name)
    path = os.path.join(HERE, "parsimony_reference.npz")
    np.savez_compressed(path, **res)
    print(f"wrote {path} ({len(res)} arrays)")


if __name__ == "__main__":
    main()
