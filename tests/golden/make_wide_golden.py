"""Golden digests of the reference joinEdgeIndel at 1,024 sites.

The reference tool keeps the query row in a 1000-entry constant array
(`#define MAXCOL 1000` in cu/joinEdgeIndel.cu and cu/nodeKeepIndel.cu), so
the 1,024-site workloads run only through the builds with MAXCOL 1024 that
oracle/Makefile makes (oracle/_ref/joinEdgeIndel_MAXCOL1024,
oracle/_ref/nodeKeepIndel_MAXCOL1024).  The inputs are regenerated from
their seeds, so only sha256 digests of the reference's output files are
stored.

    python tests/golden/make_wide_golden.py run-ref OUTDIR   (needs a GPU)
        runs the reference builds on every case and writes
        OUTDIR/wide_reference.json
    python tests/golden/make_wide_golden.py collect OUTDIR
        checks the CPU oracle against those digests and, when every file
        matches, installs tests/golden/wide_reference.json
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from casphy_b200 import formats, synth  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.join(HERE, "wide_reference.json")

# name: (cells kept as the tree, out-group cells, seed, weight kind)
CASES = {
    "w3k_unit": (3000, 256, 41, "unit"),
    "w2k_int": (2000, 0, 42, "int"),      # weights 0..2: the largest sum is 2,048, the exact-integer limit
    "w1500_half": (1500, 0, 43, "half"),  # fractional weights: binary16 sums over 1,024 sites
}


def case_inputs(name):
    """(codes, nState, w, out-group codes) of a wide case: the 200,000-cell
    generator's settings (256 alleles Zipf(1.3), Yule depth 20, p_edit 0.02,
    15 % missing) at 1,024 sites."""
    ncell, nout, seed, wk = CASES[name]
    raw = synth.lineage_states(ncell + nout, 1024, 20, 0.02, 256, 1.3, 0.15, seed=seed)
    codes, ns = synth.regularize(raw)
    rng = np.random.default_rng(seed)
    if wk == "unit":
        w = np.ones((ns, 1024))
    elif wk == "int":
        w = rng.integers(0, 3, size=(ns, 1024)).astype(np.float64)
    else:
        w = rng.uniform(0.05, 2.0, size=(ns, 1024)).round(3)
    return np.ascontiguousarray(codes[:ncell]), ns, w, np.ascontiguousarray(codes[ncell:])


def sha_bytes(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def edge2_file_bytes(edge) -> bytes:
    e = np.asarray(edge, dtype="<u4").reshape(-1, 2)
    return np.concatenate([np.array([e.shape[0], 2], "<u4"), e.reshape(-1)]).tobytes()


def node_state2_file_bytes(state, ntip, ncol) -> bytes:
    s = np.asarray(state, dtype="<u4").reshape(-1)
    return np.concatenate([np.array([ntip - 1, ncol], "<u4"), s]).tobytes()


def retain_digest(ids) -> str:
    return sha_bytes(np.asarray(ids, dtype="<u4").tobytes())


def run_ref(outdir):
    os.makedirs(outdir, exist_ok=True)
    ji = os.path.join(REF_BIN, "joinEdgeIndel_MAXCOL1024")
    nk = os.path.join(REF_BIN, "nodeKeepIndel_MAXCOL1024")
    res = {}
    with tempfile.TemporaryDirectory() as d:
        p = lambda n: os.path.join(d, n)  # noqa: E731
        for name in CASES:
            codes, ns, w, out = case_inputs(name)
            formats.write_mat(p(name + ".tbmat"), codes)
            formats.write_mat(p(name + ".tipSize"), np.ones((codes.shape[0], 1), np.uint32))
            formats.write_f64(p(name + ".w"), w)
            r = subprocess.run([ji, name, name + ".w", str(ns), "0", "2.0"], cwd=d, stdout=subprocess.PIPE,
                               stderr=subprocess.STDOUT, timeout=1200)
            if r.returncode != 0:
                raise RuntimeError(f"reference joinEdgeIndel exited {r.returncode}: {r.stdout[-400:]!r}")
            ent = {"edge2": sha_bytes(open(p(name + ".edge2"), "rb").read()),
                   "nodeState2": sha_bytes(open(p(name + ".nodeState2"), "rb").read())}
            if out.shape[0]:
                formats.write_mat(p(name + ".tboutmat"), out)
                for cut in (1, 2):
                    subprocess.run([nk, name, str(cut)], cwd=d, check=True, stdout=subprocess.DEVNULL, timeout=600)
                    ent[f"retain{cut}"] = retain_digest(formats.read_retain(p(name + ".retainNode")))
            res[name] = ent
            print(name, ent, flush=True)
    with open(os.path.join(outdir, "wide_reference.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


def oracle_digests(name):
    import oracle as O
    codes, ns, w, out = case_inputs(name)
    e, s, _ = O.join_indel(codes, ns, w)
    ntip, ncol = codes.shape
    ent = {"edge2": sha_bytes(edge2_file_bytes(e)), "nodeState2": sha_bytes(node_state2_file_bytes(s, ntip, ncol))}
    if out.shape[0]:
        for cut in (1, 2):
            ent[f"retain{cut}"] = retain_digest(O.node_keep(s, e, out, cut))
    return ent


def collect(outdir):
    ref = json.load(open(os.path.join(outdir, "wide_reference.json")))
    bad = []
    for name in CASES:
        got = oracle_digests(name)
        for k, v in ref[name].items():
            print(name, k, "ok" if got.get(k) == v else "MISMATCH", flush=True)
            if got.get(k) != v:
                bad.append(f"{name}/{k}")
    if bad:
        raise SystemExit("oracle differs from the reference on " + ", ".join(bad))
    shutil.copyfile(os.path.join(outdir, "wide_reference.json"), OUT)
    print(f"installed {OUT}")


if __name__ == "__main__":
    cmd = sys.argv[1] if len(sys.argv) > 1 else ""
    if cmd == "run-ref" and len(sys.argv) > 2:
        run_ref(sys.argv[2])
    elif cmd == "collect" and len(sys.argv) > 2:
        collect(sys.argv[2])
    else:
        print(__doc__)
        sys.exit(2)
