"""Golden fixtures for the parity tests, produced by the reference tools.

Three steps (the second needs a GPU, the others do not):

  python tests/golden/make_golden.py prepare
      Builds every input case (seeded synthetic matrices, the CasPhy package
      data sets mat1k / mat_binary read from their .rda files, and the
      run1_1024 example alignment run through the reference fasta2bin) and
      stores them in tests/golden/cases.npz.  Reads the CasPhy source tree
      (REF env var, else a checkout named reference beside this repository)
      for the .rda/.fasta fixtures.

  python tests/golden/make_golden.py run-ref OUTDIR
      Writes each case as the reference file set, runs the reference tools
      compiled into oracle/_ref/ (see oracle/Makefile) and stores every output
      file in OUTDIR/reference_outputs.npz.

  python tests/golden/make_golden.py collect OUTDIR
      Checks the CPU oracle against those outputs and, if every case matches
      byte for byte, installs tests/golden/reference_outputs.npz.
"""
from __future__ import annotations

import gzip
import io
import os
import struct
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
CASES = os.path.join(HERE, "cases.npz")
OUTPUTS = os.path.join(HERE, "reference_outputs.npz")


# ---------------------------------------------------------------------------
# minimal reader for R's XDR serialisation (.rda = "RDX3\n" + gzip'd stream)

class _RReader:
    def __init__(self, buf: bytes):
        self.b = io.BytesIO(buf)
        self.refs = []

    def i(self):
        return struct.unpack(">i", self.b.read(4))[0]

    def item(self):
        flags = self.i()
        t = flags & 0xFF
        has_attr, has_tag = flags & (1 << 9), flags & (1 << 10)
        if t == 254:  # NILVALUE
            return None
        if t == 255:  # REFSXP
            k = flags >> 8
            return self.refs[(k or self.i()) - 1]
        if t == 1:  # SYMSXP
            s = self.item()
            self.refs.append(s)
            return s
        if t in (2, 17):  # LISTSXP / ATTRLISTSXP
            attr = self.item() if has_attr else None
            tag = self.item() if has_tag else None
            car = self.item()
            cdr = self.item()
            out = [(tag, car)]
            if isinstance(cdr, list):
                out += cdr
            del attr
            return out
        if t == 9:  # CHARSXP
            n = self.i()
            return None if n == -1 else self.b.read(n).decode("latin1")
        if t in (10, 13):  # LGLSXP / INTSXP
            n = self.i()
            v = np.frombuffer(self.b.read(4 * n), dtype=">i4").astype(np.int32)
        elif t == 14:  # REALSXP
            n = self.i()
            v = np.frombuffer(self.b.read(8 * n), dtype=">f8").astype(np.float64)
        elif t == 16:  # STRSXP
            n = self.i()
            v = [self.item() for _ in range(n)]
        elif t == 19:  # VECSXP
            n = self.i()
            v = [self.item() for _ in range(n)]
        else:
            raise ValueError(f"unsupported R type {t}")
        attrs = dict(self.item()) if has_attr else {}
        if "dim" in attrs and isinstance(v, np.ndarray):
            d = attrs["dim"]
            v = v.reshape(tuple(int(x) for x in d[::-1])).T  # column-major
        return v


def read_rda(path: str) -> dict:
    raw = gzip.open(path).read()
    assert raw[:5] == b"RDX3\n" and raw[5:7] == b"X\n", path
    r = _RReader(raw[7:])
    ver = r.i()
    r.i(), r.i()
    if ver == 3:
        n = r.i()
        r.b.read(n)
    return dict(r.item())


# ---------------------------------------------------------------------------
# case construction

def _clades(par, ch, ntip):
    """Clade bitsets (one row per internal node except the root) in the
    nodeDesBig row layout: ceil(ntip/32) u32 words, bit t = tip t."""
    nn = 2 * ntip - 1
    kids = [[] for _ in range(nn)]
    for p, c in zip(par, ch):
        kids[p].append(c)
    nb = (ntip + 31) // 32
    rows = {}
    order = []
    stack = [ntip]
    while stack:
        v = stack.pop()
        order.append(v)
        stack.extend(kids[v])
    for v in reversed(order):
        if v < ntip:
            continue
        m = np.zeros(nb, dtype=np.uint32)
        for c in kids[v]:
            if c < ntip:
                m[c // 32] |= np.uint32(1 << (c % 32))
            else:
                m |= rows[c]
        rows[v] = m
    return np.array([rows[v] for v in range(ntip + 1, nn)], dtype=np.uint32)


def prepare(ref_tree: str):
    rng = np.random.default_rng(2024)
    C = {}

    def indel(name, codes, nstate, w, tip=None, min_size=0, min_ratio=2.0):
        C[f"ji/{name}/codes"] = np.ascontiguousarray(codes, dtype=np.uint32)
        C[f"ji/{name}/w"] = np.ascontiguousarray(w, dtype=np.float64).reshape(nstate, -1)
        C[f"ji/{name}/tip"] = np.ones(codes.shape[0], np.uint32) if tip is None else tip.astype(np.uint32)
        C[f"ji/{name}/args"] = np.array([nstate, min_size], dtype=np.int64)
        C[f"ji/{name}/ratio"] = np.array([min_ratio], dtype=np.float64)

    # config-1 workload, with 256 extra cells kept as the out-group
    raw = synth.lineage_states(1280, 256, 12, 0.04, 64, 1.5, 0.10, seed=11)
    codes, ns = synth.regularize(raw)
    indel("c1", codes[:1024], ns, np.ones((ns, 256)))
    C["nk/c1/outmat"] = codes[1024:]
    # CasPhy's packaged mat1k data set (1000 cells x 30 sites)
    if ref_tree:
        m = read_rda(os.path.join(ref_tree, "data", "mat1k.rda"))["mat1k"]
        codes_m, ns_m = synth.regularize(m.astype(np.int32))
        indel("mat1k", codes_m[:900], ns_m, np.ones((ns_m, codes_m.shape[1])))
        C["nk/mat1k/outmat"] = codes_m[900:]
    # non-integer weights: exercises the binary16 accumulation order
    raw = synth.lineage_states(300, 64, 10, 0.06, 12, 1.2, 0.08, seed=12)
    codes, ns = synth.regularize(raw)
    indel("halfw", codes, ns, rng.uniform(0.05, 3.0, size=(ns, 64)).round(3))
    # minSize / minRatio rule with non-unit tip sizes
    raw = synth.lineage_states(400, 128, 11, 0.05, 32, 1.5, 0.10, seed=13)
    codes, ns = synth.regularize(raw)
    indel("minsize", codes, ns, np.ones((ns, 128)), tip=rng.integers(1, 30, size=400),
          min_size=8, min_ratio=1.5)
    # many duplicate rows: tie-breaking
    proto = synth.lineage_states(6, 16, 4, 0.2, 4, 1.0, 0.0, seed=14)
    codes, ns = synth.regularize(proto[rng.integers(0, 6, size=64)])
    indel("ties", codes, ns, np.ones((ns, 16)))
    for n in (2, 3):
        raw = synth.lineage_states(n, 8, 3, 0.3, 3, 1.0, 0.0, seed=15 + n)
        codes, ns = synth.regularize(raw)
        indel(f"tiny{n}", codes, ns, np.ones((ns, 8)))

    # binary join + nodeKeepBit + radius
    words = synth.binary_workload(2300, 512, 16, 0.03, 0.05, seed=21)
    C["jb/bin2k/words"] = words[:2000]
    C["jb/bin2k/w"] = np.ones(512)
    C["nkb/bin2k/outmat"] = words[2000:]
    w96 = rng.uniform(0.1, 2.0, size=96).round(2)
    C["jb/bhalf/words"] = synth.binary_workload(300, 96, 10, 0.06, 0.05, seed=22)
    C["jb/bhalf/w"] = w96
    if ref_tree:
        mb = read_rda(os.path.join(ref_tree, "data", "mat_binary.rda"))["mat_binary"]
        C["jb/matbin/words"] = formats.pack_bits(np.asarray(mb) != 0)
        C["jb/matbin/w"] = np.ones(C["jb/matbin/words"].shape[1] * 32)

    # DNA radius inputs
    tips, _ = synth.hky85_alignment(1000, 400, 4.0, [0.3, 0.2, 0.2, 0.3], 0.01, 0.02, seed=31)
    raw_dna, keep = synth.dna_to_fasta2bin(tips)
    C["dna/hky/raw"] = raw_dna
    C["dna/hky/lvalid"] = np.array([int(keep.sum())])
    if ref_tree:
        with tempfile.TemporaryDirectory() as d:
            subprocess.run([os.path.join(REF_BIN, "fasta2bin"),
                            os.path.join(ref_tree, "examples", "run1_1024.fasta"),
                            os.path.join(d, "run1")], check=True, stdout=subprocess.DEVNULL)
            C["dna/run1/raw"] = formats.read_mat(os.path.join(d, "run1.bin"))
            pos = open(os.path.join(d, "run1_positions.txt")).read().splitlines()[1:]
            C["dna/run1/lvalid"] = np.array([sum(p.endswith("Yes") for p in pos)])
            C["f2b/run1/names"] = np.frombuffer(open(os.path.join(d, "run1_names.txt"), "rb").read(), np.uint8)
            C["f2b/run1/positions"] = np.frombuffer(open(os.path.join(d, "run1_positions.txt"), "rb").read(), np.uint8)

    # TransferDis clade sets from two random trees (ntip not a multiple of 32,
    # row counts not multiples of 8) plus a copy with stray padding bits
    ntip = 700
    pa, ca, _ = synth.yule_tree(ntip, 1.0, rng)
    pb, cb, _ = synth.yule_tree(ntip, 1.0, rng)
    ya, xb = _clades(pa, ca, ntip), _clades(pb, cb, ntip)
    C["td/trees/y"], C["td/trees/x"] = ya[:-3], xb[:-5]
    C["td/trees/ntip"] = np.array([ntip])
    yp, xp = ya[:-1].copy(), xb[:-2].copy()
    pad_bits = np.uint32(0xFFFFFFFF) << np.uint32(ntip % 32)
    yp[::7, -1] |= pad_bits
    xp[::5, -1] |= pad_bits
    C["td/padded/y"], C["td/padded/x"], C["td/padded/ntip"] = yp, xp, np.array([ntip])
    np.savez_compressed(CASES, **C)
    print(f"wrote {CASES} with {len(C)} arrays")


def _cases():
    z = np.load(CASES)
    out = {}
    for k in z.files:
        kind, name, field = k.split("/")
        out.setdefault((kind, name), {})[field] = z[k]
    return out


# ---------------------------------------------------------------------------
# reference runs

def _run(args, cwd, timeout=300):
    r = subprocess.run(args, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{args[0]} exited {r.returncode}: {r.stdout[-400:]!r}")
    return r.stdout.decode(errors="replace")


def run_tools(bindir: str) -> dict:
    """Runs every golden case through the executables in `bindir` (the
    reference build in oracle/_ref, or the drop-ins in casphy_b200/bin) and
    returns their output files as arrays.  Tools missing from `bindir` are
    skipped."""
    _bin = lambda name: os.path.join(bindir, name)  # noqa: E731
    have = lambda name: os.path.exists(_bin(name))  # noqa: E731
    cases = _cases()
    res = {}
    with tempfile.TemporaryDirectory() as d:
        p = lambda n: os.path.join(d, n)  # noqa: E731
        for (kind, name), c in sorted(cases.items()):
            if kind == "ji" and have("joinEdgeIndel"):
                formats.write_mat(p(name + ".tbmat"), c["codes"])
                formats.write_mat(p(name + ".tipSize"), c["tip"].reshape(-1, 1))
                formats.write_f64(p(name + ".w"), c["w"])
                ns, ms = (int(x) for x in c["args"])
                _run([_bin("joinEdgeIndel"), name, name + ".w", str(ns), str(ms), repr(float(c["ratio"][0]))], d)
                res[f"ji/{name}/edge2"] = formats.read_mat(p(name + ".edge2"))
                res[f"ji/{name}/nodeState2"] = np.fromfile(p(name + ".nodeState2"), dtype=np.uint32)
                om = cases.get(("nk", name))
                if om is not None and have("nodeKeepIndel"):
                    formats.write_mat(p(name + ".tboutmat"), om["outmat"])
                    for cut in (1, 3):
                        _run([_bin("nodeKeepIndel"), name, str(cut)], d)
                        res[f"nk/{name}/retain{cut}"] = formats.read_retain(p(name + ".retainNode"))
            elif kind == "jb" and have("joinEdgeBitReverse"):
                formats.write_mat(p(name + ".tbmat"), c["words"])
                formats.write_f64(p(name + ".w"), c["w"])
                for at in (0, 1):
                    _run([_bin("joinEdgeBitReverse"), name, name + ".w", str(at)], d)
                    res[f"jb/{name}/edge2_t{at}"] = formats.read_mat(p(name + ".edge2"))
                    res[f"jb/{name}/nodeState2_t{at}"] = np.fromfile(p(name + ".nodeState2"), dtype=np.uint32)
                    om = cases.get(("nkb", name))
                    if om is not None and at == 1 and have("nodeKeepBit"):
                        formats.write_mat(p(name + ".tboutmat"), om["outmat"])
                        for cut in (1, 2):
                            _run([_bin("nodeKeepBit"), name, str(cut)], d)
                            res[f"nkb/{name}/retain{cut}"] = formats.read_retain(p(name + ".retainNode"))
                # radius search on the same cells (word-plane-major .bmat)
                formats.write_mat(p(name + ".bmat"), c["words"].T)
                for r in (3, 4, 12):
                    _run([_bin("radiusNeighbor"), name, str(r)], d)
                    res[f"rb/{name}/idx{r}"] = formats.read_idx(p(name + ".idx"))
                    res[f"rb/{name}/nNeighbor{r}"] = np.fromfile(p(name + ".nNeighbor"), dtype=np.uint32)
                _run([_bin("tryRadius"), name, "4", "64"], d)
                res[f"trb/{name}/nNeighbor4"] = np.fromfile(p(name + ".nNeighbor"), dtype=np.uint32)
            elif kind == "dna":
                formats.write_mat(p(name + ".tbmat"), c["raw"])
                lv = int(c["lvalid"][0])
                for r in (lv - 20, lv - 100, lv // 2):
                    _run([_bin("radiusNeighborDNA"), name, str(r)], d)
                    res[f"rd/{name}/idx{r}"] = formats.read_idx(p(name + ".idx"))
                    res[f"rd/{name}/nNeighbor{r}"] = np.fromfile(p(name + ".nNeighbor"), dtype=np.uint32)
                _run([_bin("tryRadiusDNA"), name, str(lv - 20), "64"], d)
                res[f"trd/{name}/nNeighbor{lv - 20}"] = np.fromfile(p(name + ".nNeighbor"), dtype=np.uint32)
                # bootstrap column resampler on the fasta2bin matrix
                formats.write_mat(p(name + ".bin"), c["raw"])
                if have("Felsenstein"):
                    _run([_bin("Felsenstein"), name, "7"], d)
                    res[f"fs/{name}/B7bin"] = np.fromfile(p(name + "B7.bin"), dtype=np.uint32)
                    res[f"fs/{name}/B7idx"] = np.fromfile(p(name + "B7.idx"), dtype=np.uint32)
            elif kind == "td":
                formats.write_mat(p(name + "_y"), c["y"])
                formats.write_mat(p(name + "_x"), c["x"])
                _run([_bin("TransferDisStream"), name + "_y", name + "_x", name, str(int(c["ntip"][0]))], d)
                res[f"td/{name}/ymin"] = np.fromfile(p(name + "_ymin.bin"), dtype=np.uint32)
                res[f"td/{name}/xmin"] = np.fromfile(p(name + "_xmin.bin"), dtype=np.uint32)
            print("ran", kind, name, flush=True)
    return res


def run_ref(outdir: str):
    os.makedirs(outdir, exist_ok=True)
    res = run_tools(REF_BIN)
    path = os.path.join(outdir, "reference_outputs.npz")
    np.savez_compressed(path, **res)
    print(f"wrote {path} with {len(res)} arrays")


def collect(outdir: str):
    from golden_check import check_all  # noqa: E402
    src = os.path.join(outdir, "reference_outputs.npz")
    ok, report = check_all(_cases(), dict(np.load(src)))
    print("\n".join(report))
    if not ok:
        raise SystemExit("oracle does not match the reference outputs; fixtures not installed")
    import shutil
    shutil.copyfile(src, OUTPUTS)
    print(f"installed {OUTPUTS}")


if __name__ == "__main__":
    cmd = sys.argv[1] if len(sys.argv) > 1 else ""
    if cmd == "prepare":
        ref = os.environ.get("REF", os.path.join(ROOT, os.pardir, "reference"))
        if not os.path.isdir(os.path.join(ref, "cu")):
            raise SystemExit(f"no CasPhy source tree at {ref}: set REF to the reference checkout")
        prepare(ref)
    elif cmd == "run-ref":
        run_ref(sys.argv[2])
    elif cmd == "collect":
        sys.path.insert(0, HERE)
        collect(sys.argv[2])
    else:
        print(__doc__)
        sys.exit(2)
