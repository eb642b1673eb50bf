"""The FP64 pruning oracle against closed forms, brute-force enumeration and
central differences (no GPU)."""
import itertools

import numpy as np
import pytest

import felsenstein as F
from casphy_b200 import synth


def _jc_same(t):
    return 0.25 + 0.75 * np.exp(-4.0 * t / 3.0)


def _jc_diff(t):
    return 0.25 - 0.25 * np.exp(-4.0 * t / 3.0)


@pytest.mark.parametrize("x1,x2", [(1, 1), (1, 2), (8, 1), (4, 4)])
def test_two_taxa_jc69_closed_form(x1, x2):
    # HKY85 with kappa = 1 and uniform frequencies is JC69
    t1, t2 = 0.13, 0.41
    codes = np.array([[x1], [x2]], dtype=np.uint32)
    ll = F.loglik_hky85(2, [2, 2], [0, 1], np.array([t1, t2]), codes, None, 1.0, [0.25] * 4)
    p = _jc_same(t1 + t2) if x1 == x2 else _jc_diff(t1 + t2)
    assert ll == pytest.approx(np.log(0.25 * p), rel=1e-12)


def test_two_taxa_missing_and_ambiguous():
    t = np.array([0.2, 0.3])
    # a missing tip contributes nothing: L = pi_x
    pi = [0.3, 0.2, 0.2, 0.3]
    ll = F.loglik_hky85(2, [2, 2], [0, 1], t, np.array([[2], [0]], np.uint32), None, 4.0, pi)
    assert ll == pytest.approx(np.log(0.2), rel=1e-12)
    # an ambiguous nibble sums over its bases
    lA = F.loglik_hky85(2, [2, 2], [0, 1], t, np.array([[1], [2]], np.uint32), None, 4.0, pi)
    lC = F.loglik_hky85(2, [2, 2], [0, 1], t, np.array([[4], [2]], np.uint32), None, 4.0, pi)
    lAC = F.loglik_hky85(2, [2, 2], [0, 1], t, np.array([[5], [2]], np.uint32), None, 4.0, pi)
    assert np.exp(lAC) == pytest.approx(np.exp(lA) + np.exp(lC), rel=1e-12)


def test_irreversible_two_taxa_closed_form():
    r, t1, t2 = 1.7, 0.2, 0.5
    p1, p2 = np.exp(-r * t1), np.exp(-r * t2)
    q = np.array([[0.0, 0.7, 0.3]] * 4)
    codes = np.array([[2, 2, 1, 0], [2, 3, 3, 3]], dtype=np.uint32)
    site = [F.loglik_irreversible(2, [2, 2], [0, 1], np.array([t1, t2]), codes[:, [s]], None, r, q[[s]])
            for s in range(4)]
    exp = [q[0, 1] ** 2 * (1 - p1) * (1 - p2), 0.0, p1 * q[0, 2] * (1 - p2), q[0, 2] * (1 - p2)]
    assert site[0] == pytest.approx(np.log(exp[0]), rel=1e-12)
    assert site[1] == -np.inf or np.exp(site[1]) == pytest.approx(q[0, 1] * q[0, 2] * (1 - p1) * (1 - p2))
    assert site[2] == pytest.approx(np.log(exp[2]), rel=1e-12)
    assert site[3] == pytest.approx(np.log(exp[3]), rel=1e-12)


def _brute_hky(ntip, par, ch, t, codes, kappa, pi):
    Q = F.hky85_Q(kappa, np.asarray(pi))
    parts = F._expm_parts(Q, np.asarray(pi))
    nn = 2 * ntip - 1
    internal = list(range(ntip, nn))
    total = 0.0
    for s in range(codes.shape[1]):
        site = 0.0
        for assign in itertools.product(range(4), repeat=len(internal)):
            st = dict(zip(internal, assign))
            pr = pi[st[ntip]]
            for e in range(len(ch)):
                P, _ = F._P_dP(parts, t[e])
                a = st[par[e]]
                if ch[e] >= ntip:
                    pr *= P[a, st[ch[e]]]
                else:
                    nib = int(codes[ch[e], s]) & 0xF
                    allowed = [b for b in range(4) if nib == 0 or (nib >> b) & 1]
                    pr *= sum(P[a, b] for b in allowed)
            site += pr
        total += np.log(site)
    return total


def test_four_taxa_brute_force():
    par, ch, t = synth.yule_tree(4, 0.2, np.random.default_rng(3))
    rng = np.random.default_rng(4)
    codes = rng.choice([0, 1, 2, 4, 8, 5, 15], size=(4, 3)).astype(np.uint32)
    pi = [0.3, 0.2, 0.2, 0.3]
    ll = F.loglik_hky85(4, par, ch, t, codes, None, 4.0, pi)
    assert ll == pytest.approx(_brute_hky(4, par, ch, t, codes, 4.0, pi), rel=1e-12)


def test_gradients_match_central_differences():
    states, (par, ch, t) = synth.hky85_alignment(12, 60, 4.0, [0.3, 0.2, 0.2, 0.3], 0.1, 0.05, seed=2)
    codes = synth.dna_nibbles(states)
    pi = [0.3, 0.2, 0.2, 0.3]
    ll, g = F.loglik_hky85(12, par, ch, t, codes, None, 4.0, pi, grad=True)
    fd = F.central_differences(lambda tt: F.loglik_hky85(12, par, ch, tt, codes, None, 4.0, pi), t)
    assert np.allclose(g, fd, rtol=1e-5, atol=1e-5 * np.abs(g).max())
    ecodes, (par, ch, t) = synth.edit_alignment(12, 40, 1.0, 6, 1.5, 0.3, 0.1, seed=3)
    q = F.allele_freqs(ecodes)
    ll, g = F.loglik_irreversible(12, par, ch, t, ecodes, None, 1.0, q, grad=True)
    fd = F.central_differences(lambda tt: F.loglik_irreversible(12, par, ch, tt, ecodes, None, 1.0, q), t)
    assert np.isfinite(ll)
    assert np.allclose(g, fd, rtol=1e-5, atol=1e-5 * np.abs(g).max())


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_c_loglik_matches_dense_numpy(seed):
    """The site-blocked C log-likelihoods used at full size (HKY85, and the
    compact irreversible-edit form) equal the dense numpy oracle."""
    import oracle as O
    rng = np.random.default_rng(seed)
    pi = [0.3, 0.2, 0.2, 0.3]
    states, (par, ch, t) = synth.hky85_alignment(40, 37, 4.0, pi, 0.05, 0.05, seed=seed)
    nib = synth.dna_nibbles(states)
    w = rng.uniform(0.5, 2.0, 37)
    e = np.stack([par, ch], 1)
    want = F.loglik_hky85(40, par, ch, t, nib, w, 4.0, pi)
    assert abs(O.loglik_hky85(e, t, nib, 4.0, pi, w) - want) <= 1e-11 * abs(want)
    # irreversible edits on a lineage matrix with missing entries, on a random tree
    raw = synth.lineage_states(30, 41, 8, 0.08, 6, 1.3, 0.2, seed=seed)
    codes, ns = synth.regularize(raw)
    _, (p2, c2, t2) = synth.hky85_alignment(30, 2, 4.0, pi, 0.3, 0.0, seed=seed + 10)
    q = O.tip_allele_freqs(codes, ns)
    want = F.loglik_irreversible(30, p2, c2, t2, codes, None, 0.8, q)
    got = O.loglik_irreversible(np.stack([p2, c2], 1), t2, codes, ns, q, 0.8)
    assert abs(got - want) <= 1e-11 * abs(want)
