"""FP64 CPU oracle for Felsenstein pruning -- TEST INFRASTRUCTURE.

CasPhy has no likelihood code (its cu/Felsenstein.cu is a bootstrap column
resampler), so this oracle restates the published algorithm: Felsenstein
(1981) pruning for the site likelihoods, with the outside ("upward")
recursion for the derivative of log L with respect to every branch length.
It uses dense state spaces in float64 and is therefore independent of the
compact representations the GPU kernels use.  Parity with the GPU is checked
to a relative tolerance on log L, and the gradient is also checked against
central finite differences of this oracle.

Models
  HKY85 (Hasegawa, Kishino & Yano 1985) on the 4-bit IUPAC nibble used by
  fasta2bin: bit 0 = A, bit 1 = T, bit 2 = C, bit 3 = G; a nibble with
  several bits is ambiguous, an empty nibble (gap) is missing data.
  Irreversible edits: per site, state 0 = unedited, states 1..K = alleles;
  P(0->0) = exp(-r t), P(0->a) = q_a (1 - exp(-r t)), P(a->b) = [a == b];
  the root is unedited.  Tip codes follow the .tbmat coding: 0 missing (all
  states allowed), 1 unedited, c >= 2 allele c-1.

Tree: edges (parent[i] -> child[i], length t[i]); tips 0..ntip-1; every
internal node has two children; the root is the node that is no child.
"""
from __future__ import annotations

import numpy as np


def _tree(ntip, parent, child):
    parent = np.asarray(parent, dtype=np.int64)
    child = np.asarray(child, dtype=np.int64)
    nn = len(child) + 1
    kids = [[] for _ in range(nn)]
    edge_of = np.full(nn, -1, dtype=np.int64)
    for e, (p, c) in enumerate(zip(parent, child)):
        kids[p].append(c)
        edge_of[c] = e
    roots = [v for v in range(nn) if edge_of[v] < 0]
    assert len(roots) == 1
    root = roots[0]
    order = []
    stack = [root]
    while stack:
        v = stack.pop()
        order.append(v)
        stack.extend(kids[v])
    return kids, edge_of, root, order  # order: parents before children


def hky85_Q(kappa, pi):
    """Rate matrix in nibble order (A, T, C, G); transitions A<->G, T<->C."""
    pi = np.asarray(pi, dtype=np.float64)
    Q = np.tile(pi, (4, 1))
    for i, j in ((0, 3), (3, 0), (1, 2), (2, 1)):
        Q[i, j] *= kappa
    np.fill_diagonal(Q, 0.0)
    np.fill_diagonal(Q, -Q.sum(axis=1))
    return Q / -np.dot(pi, np.diag(Q))


def _expm_parts(Q, pi):
    # Q is reversible: symmetrise with diag(sqrt(pi)) for a stable eigensystem
    s = np.sqrt(pi)
    S = (s[:, None] * Q) / s[None, :]
    lam, W = np.linalg.eigh((S + S.T) / 2)
    V = W / s[:, None]
    Vi = (W * s[:, None]).T
    return lam, V, Vi


def _P_dP(parts, t):
    lam, V, Vi = parts
    e = np.exp(lam * t)
    return (V * e) @ Vi, (V * (lam * e)) @ Vi


def _dense_tip_partials(model, codes, nsite):
    if model["name"] == "hky85":
        nib = np.asarray(codes, dtype=np.uint32) & 0xF
        L = ((nib[:, :, None] >> np.arange(4)) & 1).astype(np.float64)
        L[nib == 0] = 1.0
        return L
    raise ValueError


def loglik_hky85(ntip, parent, child, t, codes, weights, kappa, pi, grad=False):
    """log L and (optionally) d log L / d t for HKY85.  codes: (ntip, nsite)
    nibbles."""
    kids, edge_of, root, order = _tree(ntip, parent, child)
    pi = np.asarray(pi, dtype=np.float64)
    Q = hky85_Q(kappa, pi)
    parts = _expm_parts(Q, pi)
    nsite = codes.shape[1]
    w = np.ones(nsite) if weights is None else np.asarray(weights, dtype=np.float64)
    tipL = _dense_tip_partials({"name": "hky85"}, codes, nsite)
    nn = len(kids)
    L = np.zeros((nn, nsite, 4))
    lsc = np.zeros((nn, nsite))  # log scale factors
    PP = {}
    for v in reversed(order):
        if v < ntip:
            L[v] = tipL[v]
            continue
        acc = np.ones((nsite, 4))
        sc = np.zeros(nsite)
        for c in kids[v]:
            P, dP = _P_dP(parts, t[edge_of[c]])
            PP[c] = (P, dP)
            acc *= L[c] @ P.T
            sc += lsc[c]
        m = acc.max(axis=1)
        m[m == 0] = 1.0
        L[v] = acc / m[:, None]
        lsc[v] = sc + np.log(m)
    site = np.log(L[root] @ pi) + lsc[root]
    ll = float(np.dot(w, site))
    if not grad:
        return ll
    g = np.zeros(len(t))
    U = {root: np.tile(pi, (nsite, 1))}
    for v in order:
        if v < ntip:
            continue
        a, b = kids[v]
        for c, sib in ((a, b), (b, a)):
            R = U[v] * (L[sib] @ PP[sib][0].T)
            P, dP = PP[c]
            num = np.einsum("ks,ks->k", R, L[c] @ dP.T)
            den = np.einsum("ks,ks->k", R, L[c] @ P.T)
            g[edge_of[c]] = float(np.dot(w, num / den))
            Uc = R @ P
            Uc /= Uc.max(axis=1, keepdims=True)
            U[c] = Uc
    return ll, g


def allele_freqs(codes):
    """Per-site allele frequencies q (sites x (K+1)), index a = code-1 >= 1,
    from the tips' observed alleles (uniform over seen alleles if none)."""
    codes = np.asarray(codes, dtype=np.int64)
    K = max(int(codes.max()) - 1, 1)
    nsite = codes.shape[1]
    q = np.zeros((nsite, K + 1))
    for s in range(nsite):
        col = codes[:, s]
        al = col[col >= 2] - 1
        if al.size:
            cnt = np.bincount(al, minlength=K + 1).astype(np.float64)
            q[s] = cnt / cnt.sum()
        else:
            q[s, 1:] = 1.0 / K
    return q


def loglik_irreversible(ntip, parent, child, t, codes, weights, rate, q, grad=False):
    """Dense FP64 version of the irreversible edit model.  q: per-site allele
    frequencies, shape (nsite, K+1), column 0 unused."""
    kids, edge_of, root, order = _tree(ntip, parent, child)
    codes = np.asarray(codes, dtype=np.int64)
    nsite = codes.shape[1]
    K = q.shape[1] - 1
    S = K + 1
    w = np.ones(nsite) if weights is None else np.asarray(weights, dtype=np.float64)
    nn = len(kids)

    def PdP(tt):
        p = np.exp(-rate * tt)
        P = np.zeros((nsite, S, S))
        dP = np.zeros((nsite, S, S))
        P[:, 0, 0] = p
        P[:, 0, 1:] = q[:, 1:] * (1 - p)
        dP[:, 0, 0] = -rate * p
        dP[:, 0, 1:] = q[:, 1:] * rate * p
        idx = np.arange(1, S)
        P[:, idx, idx] = 1.0
        return P, dP

    L = np.zeros((nn, nsite, S))
    lsc = np.zeros((nn, nsite))
    for v in range(ntip):
        c = codes[v]
        Lv = np.zeros((nsite, S))
        Lv[c == 0] = 1.0
        Lv[c == 1, 0] = 1.0
        al = c >= 2
        Lv[np.nonzero(al)[0], c[al] - 1] = 1.0
        L[v] = Lv
    PP = {}
    for v in reversed(order):
        if v < ntip:
            continue
        acc = np.ones((nsite, S))
        sc = np.zeros(nsite)
        for c in kids[v]:
            P, dP = PdP(t[edge_of[c]])
            PP[c] = (P, dP)
            acc *= np.einsum("kij,kj->ki", P, L[c])
            sc += lsc[c]
        m = acc.max(axis=1)
        m[m == 0] = 1.0
        L[v] = acc / m[:, None]
        lsc[v] = sc + np.log(m)
    site = np.log(L[root][:, 0]) + lsc[root]
    ll = float(np.dot(w, site))
    if not grad:
        return ll
    g = np.zeros(len(t))
    U0 = np.zeros((nsite, S))
    U0[:, 0] = 1.0
    U = {root: U0}
    for v in order:
        if v < ntip:
            continue
        a, b = kids[v]
        for c, sib in ((a, b), (b, a)):
            R = U[v] * np.einsum("kij,kj->ki", PP[sib][0], L[sib])
            P, dP = PP[c]
            num = np.einsum("ki,ki->k", R, np.einsum("kij,kj->ki", dP, L[c]))
            den = np.einsum("ki,ki->k", R, np.einsum("kij,kj->ki", P, L[c]))
            g[edge_of[c]] = float(np.dot(w, num / den))
            Uc = np.einsum("ki,kij->kj", R, P)
            Uc /= Uc.max(axis=1, keepdims=True)
            U[c] = Uc
    return ll, g


def central_differences(f, t, h_rel=1e-5):
    g = np.zeros(len(t))
    for e in range(len(t)):
        h = h_rel * max(t[e], 1e-3)
        tp, tm = t.copy(), t.copy()
        tp[e] += h
        tm[e] -= h
        g[e] = (f(tp) - f(tm)) / (2 * h)
    return g
