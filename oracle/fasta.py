"""fasta2bin restated in Python -- TEST INFRASTRUCTURE.

Follows cu/fasta2bin.cu: read_fasta (:120-183: '>' header lines, the name is
the first token, whitespace removed from sequence lines, blank lines skipped,
a header without sequence lines dropped), count_valid_bases (:35-44: not '-',
'.', 'N'), find_variable_positions (:47-96: a column is variable when some
base count, ambiguity codes counting for each of their bases, is strictly
between 0 and the number of sequences seen), encode_char / encode_sequence
(:11-31, :186-206) and the output files (:208-243, :320-337).
"""
from __future__ import annotations

import numpy as np

_CODE = {"A": 1, "T": 2, "U": 2, "C": 4, "G": 8, "W": 3, "M": 5, "R": 9, "Y": 6, "K": 10, "S": 12, "H": 7,
         "D": 11, "V": 13, "B": 14, "N": 15}


def parse(text: str):
    names, seqs = [], []
    name, seq = "", ""
    for line in text.split("\n"):
        if line == "":
            continue
        if line[0] == ">":
            if seq:
                names.append(name)
                seqs.append(seq)
                seq = ""
            name = line[1:]
            stripped = name.lstrip(" \t")
            if stripped:
                fns = len(name) - len(stripped)
                fs = min([i for i in (name.find(" "), name.find("\t")) if i >= 0], default=-1)
                name = name[fns:fs] if fs >= fns else name[fns:]
        else:
            seq += "".join(ch for ch in line if not ch.isspace())
    if seq:
        names.append(name)
        seqs.append(seq)
    return names, seqs


def convert(text: str):
    """Returns (bin words incl. the {nseq, enc_len} header, names text, positions text)."""
    names, seqs = parse(text)
    n, L = len(seqs), len(seqs[0])
    codes = np.array([[_CODE.get(c.upper(), 0x10) for c in s] for s in seqs], dtype=np.uint32)
    cnt = np.zeros((4, L), dtype=np.int64)
    for b in range(4):
        cnt[b] = ((codes >> b) & 1).astype(bool)[:, :].__and__(codes != 0x10).sum(axis=0)
    var = ((cnt > 0) & (cnt < n)).any(axis=0)
    kept = codes[:, var]
    nw = (kept.shape[1] + 3) // 4
    pad = np.zeros((n, nw * 4), dtype=np.uint32)
    pad[:, :kept.shape[1]] = kept
    words = (pad[:, 0::4] | (pad[:, 1::4] << 8) | (pad[:, 2::4] << 16) | (pad[:, 3::4] << 24)).astype(np.uint32)
    valid = [sum(1 for c in s if c.upper() not in "-.N") for s in seqs]
    names_txt = "SequenceName,ValidBaseCount\n" + "".join(f"{a},{v}\n" for a, v in zip(names, valid))
    pos_txt = "Position,IsVariable\n" + "".join(f"{i},{'Yes' if x else 'No'}\n" for i, x in enumerate(var))
    return np.concatenate([np.array([n, nw], np.uint32), words.reshape(-1)]), names_txt, pos_txt
