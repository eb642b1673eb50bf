"""Byte-for-byte comparison of an implementation against the reference outputs.

``check_all(cases, ref, impl)`` runs every golden case through ``impl`` (an
object exposing the same functions as oracle/oracle.py: join_indel,
join_bit, node_keep, radius_bit, radius_dna, try_radius_bit, try_radius_dna,
transfer_dis) and compares with the reference tools' files.  With impl=None
the CPU oracle is checked.
"""
from __future__ import annotations

import numpy as np


def _hdr(a):
    return np.asarray(a, dtype=np.uint32).reshape(-1)


def edge2_bytes(edge):
    e = np.asarray(edge, dtype=np.uint32).reshape(-1, 2)
    return np.concatenate([_hdr([e.shape[0], 2]), e.reshape(-1)])


def node_state2_bytes(state, ntip, ncol):
    s = np.asarray(state, dtype=np.uint32).reshape(-1)
    return np.concatenate([_hdr([ntip - 1, ncol]), s])


def _cmp(report, name, got, want):
    got = np.asarray(got, dtype=np.uint32).reshape(-1)
    want = np.asarray(want, dtype=np.uint32).reshape(-1)
    ok = got.shape == want.shape and bool(np.array_equal(got, want))
    if not ok:
        extra = ""
        if got.shape == want.shape:
            bad = np.nonzero(got != want)[0]
            extra = f" first mismatch at {bad[0]} ({got[bad[0]]} vs {want[bad[0]]}), {bad.size} differ"
        report.append(f"MISMATCH {name}: got {got.shape} want {want.shape}{extra}")
    else:
        report.append(f"ok {name}")
    return ok


def iter_checks(cases, ref, impl=None, kinds=None):
    """Yield (name, ok_bool, message) for every comparable golden output."""
    if impl is None:
        import oracle as impl  # noqa: F811
    for (kind, name), c in sorted(cases.items()):
        if kinds and kind not in kinds:
            continue
        rep = []
        if kind == "ji":
            codes = c["codes"]
            ns, ms = (int(x) for x in c["args"])
            edge, state, _ = impl.join_indel(codes, ns, c["w"], c["tip"], ms, float(c["ratio"][0]))
            ntip, ncol = codes.shape
            want = ref[f"ji/{name}/edge2"]
            ok = _cmp(rep, f"ji/{name}/edge2", edge2_bytes(edge),
                      np.concatenate([_hdr(want.shape), want.reshape(-1)]))
            ok &= _cmp(rep, f"ji/{name}/nodeState2", node_state2_bytes(state, ntip, ncol), ref[f"ji/{name}/nodeState2"])
            yield f"ji/{name}", ok, "; ".join(rep)
            om = cases.get(("nk", name))
            if om is not None:
                for cut in (1, 3):
                    key = f"nk/{name}/retain{cut}"
                    if key in ref:
                        rep = []
                        got = impl.node_keep(state, edge, om["outmat"], cut, bit=False)
                        yield key, _cmp(rep, key, got, ref[key]), "; ".join(rep)
        elif kind == "jb":
            words = c["words"]
            ntip, nbin = words.shape
            for at in (0, 1):
                key = f"jb/{name}/edge2_t{at}"
                if key not in ref:
                    continue
                rep = []
                edge, state, _ = impl.join_bit(words, c["w"], at)
                ok = _cmp(rep, key, edge2_bytes(edge),
                          np.concatenate([_hdr(ref[key].shape), ref[key].reshape(-1)]))
                ok &= _cmp(rep, f"jb/{name}/nodeState2_t{at}", node_state2_bytes(state, ntip, nbin),
                           ref[f"jb/{name}/nodeState2_t{at}"])
                yield f"jb/{name}/t{at}", ok, "; ".join(rep)
                om = cases.get(("nkb", name))
                if om is not None and at == 1:
                    for cut in (1, 2):
                        key = f"nkb/{name}/retain{cut}"
                        if key in ref:
                            rep = []
                            got = impl.node_keep(state, edge, om["outmat"], cut, bit=True)
                            yield key, _cmp(rep, key, got, ref[key]), "; ".join(rep)
            bmat = np.ascontiguousarray(words.T)
            for r in (3, 4, 12):
                key = f"rb/{name}/idx{r}"
                if key not in ref:
                    continue
                rep = []
                counts, idx = impl.radius_bit(bmat, c["w"], r)
                ok = _cmp(rep, key, idx, ref[key])
                ok &= _cmp(rep, f"rb/{name}/nNeighbor{r}", np.concatenate([_hdr([1, ntip]), counts]),
                           ref[f"rb/{name}/nNeighbor{r}"])
                yield f"rb/{name}/r{r}", ok, "; ".join(rep)
            key = f"trb/{name}/nNeighbor4"
            if key in ref:
                nn = ref[key]
                nrep = int(nn[1])
                q = nn[2:2 + nrep]
                rep = []
                got = impl.try_radius_bit(bmat, c["w"], 4, q)
                yield key, _cmp(rep, key, got, nn[2 + nrep:]), "; ".join(rep)
        elif kind == "dna":
            raw = c["raw"]
            lv = int(c["lvalid"][0])
            for r in (lv - 20, lv - 100, lv // 2):
                key = f"rd/{name}/idx{r}"
                if key not in ref:
                    continue
                rep = []
                counts, idx = impl.radius_dna(raw, r)
                ok = _cmp(rep, key, idx, ref[key])
                ok &= _cmp(rep, f"rd/{name}/nNeighbor{r}", np.concatenate([_hdr([1, raw.shape[0]]), counts]),
                           ref[f"rd/{name}/nNeighbor{r}"])
                yield f"rd/{name}/r{r}", ok, "; ".join(rep)
            key = f"trd/{name}/nNeighbor{lv - 20}"
            if key in ref:
                nn = ref[key]
                nrep = int(nn[1])
                rep = []
                got = impl.try_radius_dna(raw, lv - 20, nn[2:2 + nrep])
                yield key, _cmp(rep, key, got, nn[2 + nrep:]), "; ".join(rep)
        elif kind == "td":
            ntip = int(c["ntip"][0])
            ymin, ysize, xmin, xsize = impl.transfer_dis(c["y"], c["x"], ntip)
            rep = []
            ny, nx = c["y"].shape[0], c["x"].shape[0]
            ok = _cmp(rep, f"td/{name}/ymin", np.concatenate([_hdr([2, ny]), ymin, ysize]), ref[f"td/{name}/ymin"])
            ok &= _cmp(rep, f"td/{name}/xmin", np.concatenate([_hdr([2, nx]), xmin, xsize]), ref[f"td/{name}/xmin"])
            yield f"td/{name}", ok, "; ".join(rep)


def check_all(cases, ref, impl=None, kinds=None):
    report, ok = [], True
    for name, good, msg in iter_checks(cases, ref, impl, kinds):
        ok &= good
        report.append(msg)
    return ok, report
