"""Golden fixtures for fasta2bin: synthetic FASTA texts run through the
reference's own fasta2bin (oracle/_ref/fasta2bin, built from cu/fasta2bin.cu;
it is host code and runs without a GPU).

    python tests/golden/make_fasta_golden.py   # writes fasta_reference.npz

The texts exercise upper/lower case, IUPAC ambiguity codes, gaps and dots,
sequence lines wrapped at several widths, blank lines, names followed by a
description, a header without sequence lines (dropped), and invariant,
all-gap and all-N columns.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))


def fasta_text(nseq, length, seed):
    rng = np.random.default_rng(seed)
    base = rng.choice(list("ACGT"), size=length)
    rows = []
    for i in range(nseq):
        s = base.copy()
        mut = rng.random(length) < 0.08
        s[mut] = rng.choice(list("ACGTRYKMSWBDHVN-.acgtu"), size=int(mut.sum()))
        rows.append("".join(s))
    # a few fixed columns: all gap, all N, invariant lower case
    rows = [r[:3] + "-" + r[4:] for r in rows]
    rows = [r[:5] + "N" + r[6:] for r in rows]
    rows = [r[:7] + "a" + r[8:] for r in rows]
    lines = []
    for i, r in enumerate(rows):
        lines.append(f">seq{i} some description {i}" if i % 3 == 0 else f">\tseq{i}")
        if i == 2:
            lines.append(">empty_record")
        w = [60, 17, 1000][i % 3]
        for k in range(0, len(r), w):
            lines.append(r[k:k + w] + ("  " if k % 2 else ""))
        if i % 4 == 1:
            lines.append("")
    return "\n".join(lines) + "\n"


CASES = [("f20", 20, 97, 1), ("f300", 300, 513, 2), ("f600", 600, 1200, 3)]


def run(tool, text):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "in.fasta")
        with open(src, "w") as f:
            f.write(text)
        subprocess.run([tool, src, os.path.join(d, "out")], check=True, stdout=subprocess.DEVNULL)
        bin_ = np.fromfile(os.path.join(d, "out.bin"), dtype=np.uint32)
        with open(os.path.join(d, "out_names.txt")) as f:
            names = f.read()
        with open(os.path.join(d, "out_positions.txt")) as f:
            pos = f.read()
    return bin_, names, pos


def main():
    tool = os.path.join(ROOT, "oracle", "_ref", "fasta2bin")
    res = {}
    for name, nseq, length, seed in CASES:
        text = fasta_text(nseq, length, seed)
        b, n, p = run(tool, text)
        res[f"fa/{name}/fasta"] = np.frombuffer(text.encode(), dtype=np.uint8)
        res[f"fa/{name}/bin"] = b
        res[f"fa/{name}/names"] = np.frombuffer(n.encode(), dtype=np.uint8)
        res[f"fa/{name}/positions"] = np.frombuffer(p.encode(), dtype=np.uint8)
        print(name, b[:2], flush=True)
    path = os.path.join(HERE, "fasta_reference.npz")
    np.savez_compressed(path, **res)
    print("wrote", path)


if __name__ == "__main__":
    main()
