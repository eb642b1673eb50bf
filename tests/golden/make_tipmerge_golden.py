"""Golden fixtures for tipMerge (cu/tipMerge.cu): seeded neighbour lists in
the radiusNeighbor output format, run through the reference executable built
from its own source (oracle/_ref/tipMerge, make -C oracle ref).

    python tests/golden/make_tipmerge_golden.py [out.npz]   # on a GPU box; default tipmerge_reference.npz

The lists are regenerated from their parameters by neighbour_lists(), so the
fixture stores only the parameters and the reference's .member values.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))

sys.path[:0] = [ROOT]
from casphy_b200.synth import neighbour_lists  # noqa: E402

# (name, ntip, seed, pShared): the last case has more than 131072 tips, so
# the reference's chunked visiting order is exercised
CASES = [("t300", 300, 1, 0.5), ("t2k", 2000, 2, 0.3), ("t5k", 5000, 3, 0.6), ("t5kb", 5000, 3, 0.2),
         ("t140k", 140_000, 4, 0.4)]


def write_inputs(d, name, counts, idx):
    with open(os.path.join(d, name + ".nNeighbor"), "wb") as f:
        np.array([1, len(counts)], np.uint32).tofile(f)
        counts.tofile(f)
    idx.tofile(os.path.join(d, name + ".idx"))


def read_member(path):
    with open(path) as f:
        return np.array([int(x) for x in f.read().split()], dtype=np.int32)


def run_tool(tool, counts, idx, pshared):
    with tempfile.TemporaryDirectory() as d:
        write_inputs(d, "c", counts, idx)
        subprocess.run([tool, os.path.join(d, "c"), repr(pshared)], check=True, stdout=subprocess.DEVNULL)
        return read_member(os.path.join(d, "c.member"))


def main():
    tool = os.path.join(ROOT, "oracle", "_ref", "tipMerge")
    res = {}
    for name, ntip, seed, p in CASES:
        counts, idx = neighbour_lists(ntip, seed)
        res[f"tm/{name}/params"] = np.array([ntip, seed], np.int64)
        res[f"tm/{name}/pshared"] = np.array([p], np.float64)
        res[f"tm/{name}/member"] = run_tool(tool, counts, idx, p)
        print(name, "categories", int(res[f"tm/{name}/member"].max()) + 1, flush=True)
    path = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "tipmerge_reference.npz")
    np.savez_compressed(path, **res)
    print("wrote", path)


if __name__ == "__main__":
    main()
