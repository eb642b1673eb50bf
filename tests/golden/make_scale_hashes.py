"""Oracle hashes of the full-size joins, for the parity tests and the bench.

    python tests/golden/make_scale_hashes.py [CASE ...]

Runs the CPU oracle (oracle/oracle.c) on the seeded synthetic workloads the
benchmark measures and writes, per case, the sha256 of the edge list and of
the node-state rows (little-endian u32, exactly the arrays the C ABI
returns) together with the oracle's join statistics, into
tests/golden/scale_hashes.json.  Existing entries for other cases are kept.

Cases:
  c5_200k      joinEdgeIndel on the 200,000-cell x 1,024-site indel workload
               (bench.gen_workload(): 256 alleles Zipf(1.3), Yule depth 20,
               p_edit 0.02, 15 % missing, unit weights, minSize 0, minRatio 2)
  c5_50k       the same generator cut to its first 50,000 cells
  c5_20k       the same generator cut to its first 20,000 cells
  c2_bit_t1    joinEdgeBitReverse, ancestralType 1, on the 10,000-cell x
               512-site base-editor matrix (synth.binary_workload seed 23)
  c2_bit_t0    the same with ancestralType 0

The indel cases use the oracle's column-scan engine (oracle_indel_colscan,
integer weights), which the CPU tests check against the row-wise engine
that is pinned to the reference binaries; the full 200k tree takes about
15 minutes on 8 cores.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

OUT = os.path.join(HERE, "scale_hashes.json")

C2_SEED = 23


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def c5_inputs(ncell=None):
    import bench
    return bench.gen_workload(ncell)


def c2_words():
    from casphy_b200 import synth
    return synth.binary_workload(10_000, 512, 16, 0.03, 0.05, seed=C2_SEED)


CASES = {
    "c5_200k": ("indel", None),
    "c5_50k": ("indel", 50_000),
    "c5_20k": ("indel", 20_000),
    "c2_bit_t1": ("bit", 1),
    "c2_bit_t0": ("bit", 0),
}


def run_case(name):
    import oracle as O
    kind, arg = CASES[name]
    if kind == "indel":
        codes, ns, w = c5_inputs(arg)
        flag = ctypes.c_int.in_dll(O.lib(), "oracle_indel_colscan")
        flag.value = 1
        t = time.time()
        try:
            e, s, st = O.join_indel(codes, ns, w, nthreads=os.cpu_count())
        finally:
            flag.value = 0
        desc = (f"joinEdgeIndel, first {codes.shape[0]} cells of the 200000 x 1024 indel generator "
                f"(nState {ns}), unit weights, minSize 0, minRatio 2")
    else:
        words = c2_words()
        t = time.time()
        e, s, st = O.join_bit(words, None, arg, nthreads=os.cpu_count())
        desc = f"joinEdgeBitReverse ancestralType {arg}, 10000 x 512 base-editor matrix (seed {C2_SEED}), unit weights"
    return {
        "workload": desc,
        "ntip": int(e.shape[0] // 2 + 1),
        "edge_sha256": sha(e),
        "state_sha256": sha(s),
        "stale_recomputes": int(st[0]),
        "pair_scores": int(st[1]),
        "joins": int(st[2]),
        "oracle_s": round(time.time() - t, 1),
    }


def main(argv):
    names = argv or list(CASES)
    table = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for name in names:
        if name not in CASES:
            raise SystemExit(f"unknown case {name}; known: {', '.join(CASES)}")
        table[name] = run_case(name)
        print(name, table[name], flush=True)
        with open(OUT, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
            f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:])
