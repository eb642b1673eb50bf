"""Clade matching approximateCompare2_AVX2 and the cal.abs transfer support:
the oracle against the outputs of the reference's own function
(tests/golden/transfer_support_reference.npz), and the GPU against both."""
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _cases():
    z = np.load(os.path.join(HERE, "golden", "transfer_support_reference.npz"))
    out = {}
    for k in z.files:
        name, rest = k.split("/", 1)
        out.setdefault(name, {})[rest] = z[k]
    return sorted(out.items())


def _queries(c):
    n = sum(1 for k in c if k.endswith("/edge") and k.startswith("q"))
    return [c[f"q{q}/edge"] for q in range(n)]


@pytest.mark.parametrize("name,c", _cases(), ids=lambda x: x if isinstance(x, str) else "")
def test_oracle_matches_reference(name, c):
    ntip, cache = (int(v) for v in c["ntip"])
    for q, e in enumerate(_queries(c)):
        for k, thr in enumerate(c["thr"]):
            if f"q{q}/t{k}/out_of_cache" in c:
                with pytest.raises(RuntimeError):
                    O.approx_compare(c["rows"], ntip, c["ref"], e, cache_size=cache, threshold=float(thr))
                continue
            r2q, q2r = O.approx_compare(c["rows"], ntip, c["ref"], e, cache_size=cache, threshold=float(thr))
            assert np.array_equal(r2q, c[f"q{q}/t{k}/ref2qry"]) and np.array_equal(q2r, c[f"q{q}/t{k}/qry2ref"])


def _support(ref2qry_list, sizes, ntip, thr):
    """cal.abs's support column from the function's outputs, as R computes it."""
    node_size = np.concatenate([[ntip], sizes[::-1]]).astype(np.float64)
    dis = np.stack([r[:, 1] for r in ref2qry_list], axis=1).astype(np.float64)
    return ((dis / node_size[:, None]) <= thr).sum(axis=1) / dis.shape[1], node_size.astype(np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("name,c", _cases(), ids=lambda x: x if isinstance(x, str) else "")
def test_gpu_matches_reference(gpu_lib, name, c):
    ntip, cache = (int(v) for v in c["ntip"])
    qs = _queries(c)
    for k, thr in enumerate(c["thr"]):
        r2q, q2r, status = gpu_lib.approx_compare(c["rows"], ntip, c["ref"], qs, cache_size=cache,
                                                  threshold=float(thr))
        for q in range(len(qs)):
            if f"q{q}/t{k}/out_of_cache" in c:
                assert status[q] != 0
                continue
            assert status[q] == 0
            assert np.array_equal(r2q[q], c[f"q{q}/t{k}/ref2qry"]), (name, q, k)
            assert np.array_equal(q2r[q], c[f"q{q}/t{k}/qry2ref"]), (name, q, k)


@pytest.mark.gpu
def test_gpu_cal_abs_matches_reference():
    """cal.abs at thresholds 0.05 and 0.3 (compared at 0.1 and 0.35) over the
    five bootstrap trees of the 600-tip case."""
    import casphy_b200.lib as L
    c = dict(_cases())["join600"]
    ntip = int(c["ntip"][0])
    qs = _queries(c)
    for k, thr in enumerate((0.05, 0.3)):
        sup, size = L.cal_abs(c["ref"], ntip, qs, threshold=thr)
        want, wsize = _support([c[f"q{q}/t{k}/ref2qry"] for q in range(len(qs))], c["sizes"], ntip, thr)
        assert np.array_equal(size, wsize)
        assert np.array_equal(sup, want)
    # a query tree beyond the cache is an error, as the reference stops
    # a caterpillar over 9,000 tips listed internal child first keeps every
    # internal node open at once in the reverse edge order
    n = 9000
    down = [(n + i, n + i + 1) for i in range(n - 2)]
    tips = [(2 * n - 2, n - 2), (2 * n - 2, n - 1)] + [(n + i, i) for i in range(n - 3, -1, -1)]
    big = np.array(down + tips, np.uint32)
    with pytest.raises(L.CasphyError) as e:
        L.cal_abs(big, n, [big], threshold=0.05)
    assert e.value.status == 2


@pytest.mark.gpu
def test_gpu_matches_oracle_larger(gpu_lib):
    """2,000-tip join tree against 12 join trees of column-resampled data, one
    launch sequence for all of them, at two thresholds."""
    from casphy_b200 import synth
    words = synth.binary_workload(2000, 512, 16, 0.03, 0.05, seed=41)
    ref, _, _ = gpu_lib.join_bit(words, None, 1)
    rng = np.random.default_rng(5)
    bits = np.unpackbits(words.view(np.uint8), axis=1, bitorder="little")[:, :512]
    qs = []
    for _ in range(12):
        wb = np.ascontiguousarray(np.packbits(bits[:, rng.integers(0, 512, 512)], axis=1, bitorder="little"))
        e, _, _ = gpu_lib.join_bit(wb.view(np.uint32), None, 1)
        qs.append(e)
    rows, _ = gpu_lib.node_des(ref, 2000)
    for thr in (0.1, 0.3):
        r2q, q2r, status = gpu_lib.approx_compare(rows, 2000, ref, qs, threshold=thr)
        assert not status.any()
        for q, e in enumerate(qs):
            a, b = O.approx_compare(rows, 2000, ref, e, threshold=thr)
            assert np.array_equal(r2q[q], a) and np.array_equal(q2r[q], b)


@pytest.mark.gpu
def test_gpu_rejects_malformed_trees(gpu_lib):
    c = dict(_cases())["yule300"]
    ref, rows = c["ref"], c["rows"]
    q = _queries(c)[0]
    # a query tree whose rows list a node's own edge before its parent edge
    moved = q.copy()
    i = int(np.nonzero(moved[:, 1] >= 301)[0][0])
    j = int(np.nonzero(moved[:, 0] == moved[i, 1])[0][0])
    moved[[i, j]] = moved[[j, i]]
    with pytest.raises(gpu_lib.CasphyError) as err:
        gpu_lib.approx_compare(rows, 300, ref, [moved])
    assert err.value.status == 1
    # a reference tree whose parent links form a cycle u -> v -> u
    loop = ref.copy()
    for k in np.nonzero(loop[:, 1] >= 301)[0]:
        u = loop[k, 1]
        m = np.nonzero((loop[:, 0] == u) & (loop[:, 1] >= 301))[0]
        if len(m):
            loop[k, 0] = loop[m[0], 1]
            break
    with pytest.raises(gpu_lib.CasphyError) as err:
        gpu_lib.approx_compare(rows, 300, loop, [q])
    assert err.value.status == 1
