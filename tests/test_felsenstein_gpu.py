"""Felsenstein pruning on the GPU (FP32 partials, FP64 sums) against the FP64
oracle: log L to 1e-6 relative, the adjoint gradient against the oracle's
gradient and central differences, reproducibility, site chunking, and the
branch-length optimiser (adjoint against per-edge central differences)."""
import numpy as np
import pytest

import felsenstein as F
from casphy_b200 import synth

pytestmark = pytest.mark.gpu

PI = [0.3, 0.2, 0.2, 0.3]
LL_RTOL = 1e-6  # |log L - log L_fp64| / |log L_fp64|


def _edge(par, ch):
    return np.stack([par, ch], axis=1).astype(np.uint32)


def _hky_case(ntip, nsite, seed, mean_bl=0.05, p_gap=0.02):
    states, (par, ch, t) = synth.hky85_alignment(ntip, nsite, 4.0, PI, mean_bl, p_gap, seed=seed)
    return synth.dna_nibbles(states), par, ch, t


def _edit_case(ntip, nsite, seed):
    codes, (par, ch, t) = synth.edit_alignment(ntip, nsite, 1.0, 30, 1.5, 0.15, 0.1, seed=seed)
    return codes, par, ch, t


@pytest.mark.parametrize("ntip,nsite,seed", [(2, 5, 1), (17, 130, 2), (200, 300, 3), (1000, 257, 4)])
def test_hky85_loglik_and_gradient(gpu_lib, ntip, nsite, seed):
    codes, par, ch, t = _hky_case(ntip, nsite, seed)
    w = np.random.default_rng(seed).integers(0, 4, nsite).astype(np.float64)
    ll, g = gpu_lib.felsenstein_loglik(_edge(par, ch), t, codes, kappa=4.0, pi=PI, weights=w, grad=True)
    ll0, g0 = F.loglik_hky85(ntip, par, ch, t, codes, w, 4.0, PI, grad=True)
    assert abs(ll - ll0) <= LL_RTOL * abs(ll0)
    scale = np.abs(g0).max()
    assert np.allclose(g, g0, rtol=2e-4, atol=2e-5 * scale)


@pytest.mark.parametrize("ntip,nsite,seed", [(2, 4, 1), (33, 150, 5), (400, 260, 6)])
def test_irreversible_loglik_and_gradient(gpu_lib, ntip, nsite, seed):
    codes, par, ch, t = _edit_case(ntip, nsite, seed)
    q = F.allele_freqs(codes)
    nallele = q.shape[1] - 1
    ll, g = gpu_lib.felsenstein_loglik(_edge(par, ch), t, codes, model="irreversible", rate=1.0,
                                       nallele=nallele, grad=True)
    ll0, g0 = F.loglik_irreversible(ntip, par, ch, t, codes, None, 1.0, q, grad=True)
    assert abs(ll - ll0) <= LL_RTOL * abs(ll0)
    scale = np.abs(g0).max()
    assert np.allclose(g, g0, rtol=2e-4, atol=2e-5 * scale)


def test_gradient_against_central_differences(gpu_lib):
    codes, par, ch, t = _hky_case(24, 200, 9, mean_bl=0.1)
    _, g = gpu_lib.felsenstein_loglik(_edge(par, ch), t, codes, kappa=4.0, pi=PI, grad=True)
    fd = F.central_differences(lambda tt: F.loglik_hky85(24, par, ch, tt, codes, None, 4.0, PI), t)
    assert np.allclose(g, fd, rtol=1e-3, atol=1e-4 * np.abs(fd).max())


def test_site_chunks_and_repeat_are_bitwise_identical(gpu_lib):
    codes, par, ch, t = _hky_case(300, 1000, 11)
    e = _edge(par, ch)
    a = gpu_lib.felsenstein_loglik(e, t, codes, kappa=4.0, pi=PI, grad=True)
    b = gpu_lib.felsenstein_loglik(e, t, codes, kappa=4.0, pi=PI, grad=True)
    # 299 internal nodes x 36 B per site: a 3 MB budget gives 256-site chunks
    c = gpu_lib.felsenstein_loglik(e, t, codes, kappa=4.0, pi=PI, grad=True, mem_budget=3_000_000)
    assert a[0] == b[0] == c[0]
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[1], c[1])
    codes, par, ch, t = _edit_case(300, 700, 12)
    q = F.allele_freqs(codes)
    kw = dict(model="irreversible", rate=1.0, nallele=q.shape[1] - 1, grad=True)
    a = gpu_lib.felsenstein_loglik(_edge(par, ch), t, codes, **kw)
    c = gpu_lib.felsenstein_loglik(_edge(par, ch), t, codes, mem_budget=1_500_000, **kw)
    assert a[0] == c[0] and np.array_equal(a[1], c[1])


def test_given_allele_frequencies(gpu_lib):
    codes, par, ch, t = _edit_case(50, 90, 13)
    nallele = int(codes.max()) - 1
    q = np.random.default_rng(1).random((90, nallele + 1)) + 0.05
    q[:, 0] = 0
    q /= q.sum(axis=1, keepdims=True)
    ll = gpu_lib.felsenstein_loglik(_edge(par, ch), t, codes, model="irreversible", rate=0.7,
                                    nallele=nallele, allele_freq=q)
    ll0 = F.loglik_irreversible(50, par, ch, t, codes, None, 0.7, q)
    assert abs(ll - ll0) <= LL_RTOL * abs(ll0)


def _fp64_optimum(f_and_g, t0):
    from scipy.optimize import minimize

    def fun(x):
        ll, g = f_and_g(np.exp(x))
        return -ll, -g * np.exp(x)

    r = minimize(fun, np.log(t0), jac=True, method="L-BFGS-B",
                 bounds=[(np.log(1e-8), np.log(10.0))] * len(t0),
                 options=dict(maxiter=5000, ftol=1e-15, gtol=1e-10))
    return -r.fun


def test_optimizer_reaches_fp64_optimum_and_beats_central_differences(gpu_lib):
    codes, par, ch, t_true = _hky_case(20, 400, 21, mean_bl=0.08)
    e = _edge(par, ch)
    t0 = np.full(len(t_true), 0.05)
    kw = dict(kappa=4.0, pi=PI, rel_tol=1e-10, max_iter=300)
    ta, sa = gpu_lib.felsenstein_optimize(e, t0, codes, gradient="adjoint", **kw)
    tf, sf = gpu_lib.felsenstein_optimize(e, t0, codes, gradient="central_diff", **kw)
    la = F.loglik_hky85(20, par, ch, ta, codes, None, 4.0, PI)
    lf = F.loglik_hky85(20, par, ch, tf, codes, None, 4.0, PI)
    l0 = F.loglik_hky85(20, par, ch, t0, codes, None, 4.0, PI)
    best = _fp64_optimum(lambda t: F.loglik_hky85(20, par, ch, t, codes, None, 4.0, PI, grad=True), t0)
    # the adjoint optimiser lands within 1e-6 (relative) of the FP64 optimum
    assert abs(la - best) <= 1e-6 * abs(best)
    assert lf > l0 + 1.0 and la >= lf - 1e-6 * abs(la)
    # the reported final log L is the GPU value at the returned lengths
    assert abs(sa["loglik_end"] - la) <= LL_RTOL * abs(la)
    assert sa["evaluations"] * 10 < sf["evaluations"]


def test_optimizer_irreversible(gpu_lib):
    codes, par, ch, _ = _edit_case(60, 200, 22)
    q = F.allele_freqs(codes)
    t0 = np.full(2 * 60 - 2, 0.1)
    t, st = gpu_lib.felsenstein_optimize(_edge(par, ch), t0, codes, model="irreversible", rate=1.0,
                                         nallele=q.shape[1] - 1, rel_tol=1e-10, max_iter=500)
    l1 = F.loglik_irreversible(60, par, ch, t, codes, None, 1.0, q)
    assert l1 >= F.loglik_irreversible(60, par, ch, t0, codes, None, 1.0, q)
    assert abs(st["loglik_end"] - l1) <= LL_RTOL * abs(l1)
    best = _fp64_optimum(lambda tt: F.loglik_irreversible(60, par, ch, tt, codes, None, 1.0, q, grad=True), t0)
    assert abs(l1 - best) <= 1e-6 * abs(best)


def test_bad_trees_raise(gpu_lib):
    codes, par, ch, t = _hky_case(8, 10, 1)
    e = _edge(par, ch)
    bad = e.copy()
    bad[3, 0] = bad[0, 0]  # a node with three children
    with pytest.raises(gpu_lib.CasphyError):
        gpu_lib.felsenstein_loglik(bad, t, codes, kappa=4.0, pi=PI)
    with pytest.raises(gpu_lib.CasphyError):
        gpu_lib.felsenstein_loglik(e[:-1], t[:-1], codes, kappa=4.0, pi=PI)
    with pytest.raises(gpu_lib.CasphyError):
        gpu_lib.felsenstein_loglik(e, -t, codes, kappa=4.0, pi=PI)


def test_resample_columns_matches_gather(gpu_lib):
    rng = np.random.default_rng(3)
    raw = rng.integers(0, 2**32, size=(37, 11), dtype=np.uint64).astype(np.uint32)
    idx = np.sort(rng.integers(0, 44, size=41)).astype(np.uint32)
    out = gpu_lib.resample_columns(raw, idx)
    b = raw.view(np.uint8).reshape(37, 44)
    exp = np.zeros((37, 44), np.uint8)
    exp[:, :41] = b[:, idx]
    assert np.array_equal(out.view(np.uint8).reshape(37, -1)[:, :41], exp[:, :41])
    assert np.all(out.view(np.uint8).reshape(37, -1)[:, 41:] == 0)


def _fp64_optimum_from(f_and_g, t_start):
    from scipy.optimize import minimize

    def fun(x):
        ll, g = f_and_g(np.exp(x))
        return -ll, -g * np.exp(x)

    r = minimize(fun, np.log(np.maximum(t_start, 1e-8)), jac=True, method="L-BFGS-B",
                 bounds=[(np.log(1e-8), np.log(10.0))] * len(t_start),
                 options=dict(maxiter=2000, ftol=1e-15, gtol=1e-10))
    return -r.fun


def test_benchmark_small_case_reaches_fp64_optimum(gpu_lib):
    """The 128-tip x 2,000-site HKY85 case the adjoint is timed against central
    differences on: the adjoint result, evaluated in FP64, is within 1e-6
    (relative) of the FP64 optimum; the central-difference result is not
    better.  The FP64 optimum is refined by L-BFGS-B from the better of the
    two results."""
    codes, par, ch, _ = _hky_case(128, 2000, 14, mean_bl=0.01)
    e = _edge(par, ch)
    t0 = np.full(2 * 128 - 2, 0.01)
    kw = dict(kappa=4.0, pi=PI, rel_tol=1e-9, max_iter=1000)
    ta, sa = gpu_lib.felsenstein_optimize(e, t0, codes, **kw)
    tf, sf = gpu_lib.felsenstein_optimize(e, t0, codes, gradient="central_diff", **kw)
    f = lambda t, grad=False: F.loglik_hky85(128, par, ch, t, codes, None, 4.0, PI, grad=grad)  # noqa: E731
    la, lf = f(ta), f(tf)
    best = _fp64_optimum_from(lambda t: f(t, True), ta if la >= lf else tf)
    best = max(best, la, lf)
    assert abs(la - best) <= 1e-6 * abs(best)
    assert lf <= la + 1e-7 * abs(la)
    assert abs(sa["loglik_end"] - la) <= LL_RTOL * abs(la)


def test_parsimony_warm_start_edit_model(gpu_lib):
    """The bench's edit-model leg on a small join tree: charAncestralEC on the
    GPU equals the oracle, and L-BFGS started from the parsimony times
    (casphy_b200.branch_lengths.parsimony_start) starts higher than the flat
    start and ends at the same optimum."""
    import bench
    raw = synth.lineage_states(1500, 256, 11, 0.04, 32, 1.5, 0.1, 21)
    codes, nstate = synth.regularize(raw)
    edge, _, _ = gpu_lib.join_indel(codes, nstate, np.ones((nstate, 256)))
    res = bench.blopt_c5(gpu_lib, codes, nstate, edge)
    par = res["charAncestralEC"]
    ws = par["warm_start"]
    assert par["identical"]
    assert ws["loglik_start"] > res["loglik_start"]
    assert abs(ws["loglik_end_rel_diff_to_flat_start"]) <= 1e-6
