#!/usr/bin/env python
"""Headline benchmark: greedy indel join (joinEdgeIndel) of the 200,000-cell
x 1,024-site CRISPR indel workload on B200.

One step = one complete tree: initial all-pairs local maxima, the greedy join
loop, pre-order relabelling and the gathered node-state rows, from codes
already resident in HBM.  The metric is pair-scores per second over the whole
job (tree seconds are reported beside it).  `e2e` times the same step through
the host-buffer C ABI call (casphy_join_indel), with the host->device copy of
the codes and the device->host copy of the tree and node states inside the
timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun every rank builds its own replica of the tree (the greedy join
has a sequential argmax dependence and does not shard); value = pair-scores of
all ranks / max-over-ranks time.  --impl reference times the reference's
own CPU join (greedyJoinEdge2 of src/functions.cpp, compiled from its source
behind an Rcpp stand-in header into oracle/_ref/; the oracle port when that
library was not built) on a bounded sample on the host cores; under torchrun
only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "pair-scores/s & tree s @200k cells; BL-opt & bootstrap speedup vs plain at 1e-6"
UNIT = "pair-scores/s"
WORKLOAD = dict(ncell=200_000, nsite=1024, depth=20, p_edit=0.02, nallele=256, zipf_s=1.3,
                p_missing=0.15, seed=5)
CPU_SAMPLE_CELLS = 5000      # oracle port (multi-threaded restatement of cu/joinEdgeIndel.cu)
TWIN_SAMPLE_CELLS = 1024     # the reference's own CPU join (greedyJoinEdge2), a few seconds a tree
RADIUS_SPARSE = 150          # C2 radius with sparse lists (3.3 neighbours per row); shared >= 4 lists every pair
DTYPE = "fp16-exact integer counts"  # integer sums that equal the reference's binary16 sums (unit weights)


def workload_name():
    w = WORKLOAD
    return (f"joinEdgeIndel CRISPR indel {w['ncell']} cells x {w['nsite']} sites, {w['nallele']} alleles "
            f"Zipf({w['zipf_s']}), Yule depth {w['depth']}, p_edit {w['p_edit']}, {int(w['p_missing']*100)}% missing, "
            f"unit weights, minSize 0 minRatio 2")


def gen_workload(ncell=None):
    from casphy_b200 import synth
    w = dict(WORKLOAD)
    raw = synth.lineage_states(w["ncell"], w["nsite"], w["depth"], w["p_edit"], w["nallele"], w["zipf_s"],
                               w["p_missing"], w["seed"])
    if ncell is not None:
        raw = raw[:ncell]
    codes, nstate = synth.regularize(raw)
    weight = np.ones((nstate, w["nsite"]), dtype=np.float64)
    return codes, nstate, weight


# ---------------------------------------------------------------------------
# clocks sampled during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------

def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profile(kernel):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        v = d.get(kernel)
        return float(v) if v is not None else None
    except Exception:
        return None


def cpu_port_run(codes, nstate, weight, nthreads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    t0 = time.perf_counter()
    _, _, st = O.join_indel(codes, nstate, weight, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return float(st[1]), dt


def cpu_twin_run(codes, nstate, weight):
    """The reference's CPU path for this job: greedyJoinEdge2 (src/functions
    .cpp:1880-2017, what phy.join runs when no CUDA path is given), compiled
    from the reference's source into oracle/_ref/libcputwin_ref.so.  It is
    single-threaded.  Its pair-scores: N(N-1)/2 at the start plus, after each
    join, one per remaining live node, (N-1)^2 in all."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cputwin as T
    n = codes.shape[0]
    t0 = time.perf_counter()
    T.greedy_join_edge2(codes, nstate, weight, want_edge=False)
    dt = time.perf_counter() - t0
    return float((n - 1) ** 2), dt


def cpu_twin_available():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libcputwin_ref.so"))


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, world, rank):
    """The reference's CPU path on a bounded sample of the workload per step:
    greedyJoinEdge2 compiled from the reference's source when it was built
    here, else the oracle port."""
    if rank != 0:
        return 0
    twin = cpu_twin_available()
    if twin:
        ncell, cores, kind = TWIN_SAMPLE_CELLS, 1, "reference"
        run = cpu_twin_run
        what = ("greedyJoinEdge2 (src/functions.cpp:1880-2017) compiled from the reference's source behind an "
                "Rcpp stand-in header, single-threaded as in R; pair-scores counted as its own (N-1)^2")
    else:
        ncell, cores, kind = CPU_SAMPLE_CELLS, os.cpu_count() or 1, "port"
        run = lambda c, n, w: cpu_port_run(c, n, w, cores)  # noqa: E731
        what = "greedy join restated from cu/joinEdgeIndel.cu (oracle port)"
    codes, nstate, weight = gen_workload(ncell)
    times, pairs = [], 0.0
    if args.warmup > 0:
        wc, wn, ww = gen_workload(256)
        run(wc, wn, ww)
    for _ in range(args.steps):
        p, dt = run(codes, nstate, weight)
        times.append(dt)
        pairs = p
    tot = sum(times)
    value = pairs * args.steps / tot
    sample = (f"first {ncell} cells of the {WORKLOAD['ncell']}-cell workload per step "
              f"({pairs:.0f} pair-scores, {tot / args.steps:.2f} s a tree; {what}; {cores} thread(s))")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE, "data": "synthetic",
            "config": {"workload": workload_name(), "cells_per_step": ncell},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def bootstrap_suite(L, plain=True):
    """Batched bootstrap (200 replicates of the 10,000-cell x 512-site binary
    matrix, 2,000-10,000 cells each) against 200 plain runs one replicate at
    a time (join -> clades -> TransferDisStream), both through the host API."""
    from casphy_b200 import bootstrap as B
    from casphy_b200 import synth
    ncell, nsite, nrep = 10_000, 512, 200
    words = synth.binary_workload(ncell, nsite, 16, 0.03, 0.05, seed=11)
    full_edge, _, _ = L.join_bit(words, None, 1)
    off, cells, w = B.make_replicates(ncell, nsite, nrep, 2000, 10_000, seed=12)
    L.bootstrap_bit(words, full_edge, off, cells, w, threshold=0.05)  # warm-up
    t0 = time.perf_counter()
    got = L.bootstrap_bit(words, full_edge, off, cells, w, threshold=0.05)
    batched_s = time.perf_counter() - t0
    groups = {k: got["stats"][k] for k in ("max_ctas_per_rep", "tuned", "join_longest_ms", "join_busy_ms",
                                           "cost_alpha_us", "cost_beta_us", "cost_gamma_us", "graph")}
    if not plain:
        return {"batched_s": batched_s, "batched_device_ms": got["stats"]["total_ms"], "join_groups": groups}
    full_bits = B.clade_bits(full_edge, ncell, (ncell + 31) // 32)
    ymin = np.zeros_like(got["ymin"])
    ysize = np.zeros_like(got["ysize"])
    t0 = time.perf_counter()
    for r in range(nrep):
        c = cells[off[r]:off[r + 1]]
        ymin[r], ysize[r] = B.plain_replicate(L, words, full_bits, c, w[r])
    plain_s = time.perf_counter() - t0
    same = bool(np.array_equal(ymin, got["ymin"]) and np.array_equal(ysize, got["ysize"]))
    sup_same = bool(np.array_equal(B.support_counts(ymin, ysize, 0.05), got["support"]))
    return {"workload": f"{nrep} replicates of the {ncell} x {nsite} binary matrix (Yule depth 16, p_edit 0.03, "
                        "5% missing), columns resampled with replacement, 2000-10000 cells each; transfer support "
                        "of the full-data tree's clades at threshold 0.05",
            "batched_s": batched_s, "batched_device_ms": got["stats"]["total_ms"],
            "batched_phases": {k: got["stats"][k] for k in ("prep_ms", "join_ms", "transfer_ms")},
            "join_groups": groups,
            "plain_s": plain_s, "plain": "casphy_join_bit + clade bitsets + casphy_transfer_dis per replicate",
            "speedup": plain_s / batched_s, "transfer_values_identical": same, "support_identical": sup_same}


def blopt_suite(L):
    """Adjoint L-BFGS branch lengths on the 20,000 x 2,000 HKY85 alignment,
    and adjoint against per-edge central differences on a 128-tip subproblem
    with the same sites (the central-difference run needs 2 evaluations per
    edge per gradient and is not run at full size)."""
    from casphy_b200 import synth
    pi = [0.3, 0.2, 0.2, 0.3]
    states, (par, ch, t_true) = synth.hky85_alignment(20_000, 2000, 4.0, pi, 0.01, 0.02, seed=13)
    codes = synth.dna_nibbles(states)
    edge = np.stack([par, ch], 1).astype(np.uint32)
    t0 = np.full(len(t_true), 0.01)
    L.felsenstein_optimize(edge, t0, codes, kappa=4.0, pi=pi, rel_tol=1e-9, max_iter=3)  # warm-up
    t_end, full = L.felsenstein_optimize(edge, t0, codes, kappa=4.0, pi=pi, rel_tol=1e-9, max_iter=1000)
    # the GPU's log L at its final branch lengths against FP64 pruning of the same tree
    import oracle as O
    ll64 = O.loglik_hky85(edge, t_end, codes, 4.0, pi)
    s_states, (sp, sc, st) = synth.hky85_alignment(128, 2000, 4.0, pi, 0.01, 0.02, seed=14)
    s_codes = synth.dna_nibbles(s_states)
    s_edge = np.stack([sp, sc], 1).astype(np.uint32)
    s_t0 = np.full(len(st), 0.01)
    _, adj = L.felsenstein_optimize(s_edge, s_t0, s_codes, kappa=4.0, pi=pi, rel_tol=1e-9, max_iter=1000)
    _, fd = L.felsenstein_optimize(s_edge, s_t0, s_codes, kappa=4.0, pi=pi, rel_tol=1e-9, max_iter=1000,
                                   gradient="central_diff")
    rel = abs(fd["loglik_end"] - adj["loglik_end"]) / abs(adj["loglik_end"])
    # algorithmic bytes of one evaluation with gradient, per site: inside
    # writes a 20 B partial per internal node and reads each child once (20 B
    # internal, 4 B tip code); outside reads U (16 B), the two children again
    # and writes U (16 B) for each internal child
    ntip = codes.shape[0]
    nint, nsite = ntip - 1, codes.shape[1]
    per_site = 20 * nint + 2 * (20 * (nint - 1) + 4 * ntip) + 16 * (nint - 1) + 16 * (nint - 1)
    alg = float(per_site) * nsite
    hbm, how = peaks()
    achieved = alg * full["evaluations"] / full["eval_seconds"] / 1e9 if full["eval_seconds"] else 0.0
    return {"workload": "HKY85 (kappa 4, pi .3/.2/.2/.3) 20000 tips x 2000 sites, Yule tree, Exp(mean 0.01) "
                        "branches, 2% gaps; start at t = 0.01; FP32 partials, FP64 sums and L-BFGS step",
            "adjoint_s": full["seconds"], "iterations": full["iterations"], "evaluations": full["evaluations"],
            "eval_graph_s": full["eval_seconds"],
            "ms_per_evaluation": full["seconds"] * 1e3 / max(full["evaluations"], 1),
            "loglik_start": full["loglik_start"], "loglik_end": full["loglik_end"],
            "loglik_fp64_at_end": ll64, "loglik_rel_err_vs_fp64": abs(full["loglik_end"] - ll64) / abs(ll64),
            "fp64_oracle": "oracle_loglik_hky85 (Felsenstein pruning in double precision) at the final lengths",
            "fd_evaluations_per_gradient": 2 * len(t0),
            "roofline": {"kernels": "k_inside_hky + k_outside_hky (evaluation graph)", "bound": "hbm",
                         "alg_bytes_per_evaluation": alg, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_source": f"{how} hbm_gbs"},
            "small_case": {"workload": "same model, 128 tips x 2000 sites", "adjoint_s": adj["seconds"],
                           "adjoint_evaluations": adj["evaluations"], "adjoint_loglik": adj["loglik_end"],
                           "central_diff_s": fd["seconds"], "central_diff_evaluations": fd["evaluations"],
                           "central_diff_loglik": fd["loglik_end"], "speedup": fd["seconds"] / adj["seconds"],
                           "target": "log L within 1e-6 (relative) of the FP64 optimum; the adjoint result is "
                                     "checked against it in FP64 by tests/test_felsenstein_gpu.py",
                           "central_diff_gap_to_adjoint": (adj["loglik_end"] - fd["loglik_end"]) / abs(adj["loglik_end"]),
                           "central_diff_reached_target": rel <= 1e-6,
                           "speedup_kind": ("time to the target" if rel <= 1e-6 else
                                            "lower bound: the central-difference run stops short of the target "
                                            "(binary32 differences), so its whole run time is counted")}}


def _timed(fn, reps=1):
    fn()
    t0 = time.perf_counter()
    for _ in range(reps):
        out = fn()
    return out, (time.perf_counter() - t0) / reps


def rows_suite(L, nthreads):
    """The other rows of the hot path on their own configs, each timed through
    the host API (inputs and outputs through host memory) next to the CPU
    restatement (oracle/) on the host cores."""
    import oracle as O
    from casphy_b200 import bootstrap as B
    from casphy_b200 import synth
    twin = cpu_twin_available()
    if twin:
        import cputwin as T

    def same_clades(e_a, e_b, ntip):
        nw = (ntip + 31) // 32
        return (set(map(bytes, B.clade_bits(e_a, ntip, nw))) == set(map(bytes, B.clade_bits(e_b, ntip, nw))))

    res = {}
    # C1: indel 1,024 x 256, joinEdgeIndel + nodeKeepIndel
    raw = synth.lineage_states(1024, 256, 12, 0.04, 64, 1.5, 0.10, seed=21)
    codes, ns = synth.regularize(raw)
    w = np.ones((ns, 256))
    (edge, state, st), t_gpu = _timed(lambda: L.join_indel(codes, ns, w), reps=3)
    out_raw = synth.lineage_states(256, 256, 12, 0.04, 64, 1.5, 0.10, seed=22)
    outm, _ = synth.regularize(out_raw)
    keep, t_keep = _timed(lambda: L.node_keep(state, edge, outm, 2), reps=3)
    t0 = time.perf_counter()
    e0, s0, _ = O.join_indel(codes, ns, w, None, 0, 2.0, nthreads)
    k0 = O.node_keep(s0, e0, outm, 2)
    t_cpu = time.perf_counter() - t0
    res["C1_joinEdgeIndel_nodeKeepIndel"] = {
        "workload": "indel 1024 cells x 256 sites, 64 alleles Zipf(1.5), depth 12, p_edit 0.04, 10% missing; "
                    "nodeKeepIndel against 256 out-group cells, cutoff 2",
        "gpu_s": t_gpu + t_keep, "join_device_ms": st["total_ms"], "cpu_s": t_cpu, "cpu_cores": nthreads,
        "identical": bool(np.array_equal(edge, e0) and np.array_equal(state, s0) and np.array_equal(keep, k0))}
    if twin:
        t0 = time.perf_counter()
        te = T.greedy_join_edge2(codes, ns, w)
        res["C1_joinEdgeIndel_nodeKeepIndel"]["reference_cpu"] = {
            "function": "greedyJoinEdge2 (src/functions.cpp:1880-2017), 1 thread", "join_s": time.perf_counter() - t0,
            "same_tree": bool(same_clades(np.stack([te[0, :-1], te[1, :-1]], 1), edge, 1024))}
    # C2: binary 10,000 x 512: joinEdgeBitReverse, radiusNeighbor r=4, TransferDisStream vs the true tree
    words = synth.binary_workload(10_000, 512, 16, 0.03, 0.05, seed=23)
    (bedge, bstate, bst), t_join = _timed(lambda: L.join_bit(words, None, 1))
    bmat = np.ascontiguousarray(words.T)
    wr = np.ones(512)
    (cnt, idx), t_rad = _timed(lambda: L.radius_bit(bmat, wr, 4))
    (cnt_s, idx_s), t_rad_s = _timed(lambda: L.radius_bit(bmat, wr, RADIUS_SPARSE), reps=3)
    t0 = time.perf_counter()
    oc_full, oi_full = O.radius_bit(bmat, wr, 4, nthreads)
    t_cr_full = time.perf_counter() - t0
    rad_full_same = bool(np.array_equal(cnt, oc_full) and np.array_equal(idx, oi_full))
    del oc_full, oi_full
    t0 = time.perf_counter()
    oc_s, oi_s = O.radius_bit(bmat, wr, RADIUS_SPARSE, nthreads)
    t_cr_s = time.perf_counter() - t0
    rad_sparse_same = bool(np.array_equal(cnt_s, oc_s) and np.array_equal(idx_s, oi_s))
    truth = synth.lineage_clades(10_000, 16, seed=23)
    est = B.clade_bits(bedge, 10_000, (10_000 + 31) // 32)
    (ymin, ysize, xmin, xsize), t_td = _timed(lambda: L.transfer_dis(truth, est, 10_000))
    sub = 3000
    t0 = time.perf_counter()
    O.join_bit(words[:sub], None, 1, nthreads)
    t_cj = time.perf_counter() - t0
    t0 = time.perf_counter()
    c0, i0 = O.radius_bit(np.ascontiguousarray(words[:sub].T), wr, 4, nthreads)
    t_cr = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.transfer_dis(truth[:sub], est[:sub], 10_000, nthreads)
    t_ct = time.perf_counter() - t0
    res["C2_binary"] = {
        "workload": "base-editor 10000 cells x 512 sites, depth 16, p_edit 0.03, 5% missing",
        "joinEdgeBitReverse": {"gpu_s": t_join, "device_ms": bst["total_ms"], "pairs": bst["pair_scores"],
                               "cpu_sample": f"first {sub} cells", "cpu_s_sample": t_cj},
        "radiusNeighbor_r4": {"gpu_s": t_rad, "pairs": 10_000 * 10_000, "neighbours": int(cnt.sum()),
                              "note": "shared >= 4 lists every pair: a 400 MB list expansion and copy",
                              "cpu_sample": f"first {sub} cells", "cpu_s_sample": t_cr,
                              "sample_identical": None, "identical": rad_full_same,
                              "cpu_full_s": t_cr_full},
        f"radiusNeighbor_r{RADIUS_SPARSE}": {"gpu_s": t_rad_s, "pairs": 10_000 * 10_000,
                                             "neighbours": int(cnt_s.sum()), "cpu_full_s": t_cr_s,
                                             "identical": rad_sparse_same},
        "TransferDisStream_vs_true_tree": {"gpu_s": t_td, "rows_y": int(truth.shape[0]), "rows_x": int(est.shape[0]),
                                           "words": int(truth.shape[1]),
                                           "mean_normalised_distance": float(np.mean(ymin / np.maximum(ysize, 1))),
                                           "cpu_sample": f"first {sub} rows of each", "cpu_s_sample": t_ct},
        "cpu_cores": nthreads}
    # cal.abs: transfer support of the C2 join tree's clades over join trees of
    # column-resampled copies of the matrix (approximateCompare2_AVX2 per tree)
    nq = 100
    rng = np.random.default_rng(29)
    bits = np.unpackbits(words.view(np.uint8), axis=1, bitorder="little")[:, :512]
    qtrees = []
    for _ in range(nq):
        wb = np.ascontiguousarray(np.packbits(bits[:, rng.integers(0, 512, 512)], axis=1, bitorder="little"))
        qe, _, _ = L.join_bit(wb.view(np.uint32), None, 1)
        qtrees.append(qe)
    (sup, nsz), t_ca = _timed(lambda: L.cal_abs(bedge, 10_000, qtrees, threshold=0.05), reps=3)
    res["C2_binary"]["cal_abs"] = {"query_trees": nq, "gpu_s": t_ca, "mean_support": float(sup[1:].mean())}
    if twin:
        rows1, _ = O.node_des(bedge, 10_000)
        t0 = time.perf_counter()
        tdis, bad = T.approx_compare_many(rows1, 10_000, bedge, qtrees, nthreads, threshold=float(np.float32(0.1)))
        t_tc = time.perf_counter() - t0
        want = ((tdis.T / nsz[:, None].astype(np.float64)) <= 0.05).sum(axis=1) / nq
        res["C2_binary"]["cal_abs"]["reference_cpu"] = {
            "function": f"approximateCompare2_AVX2 (src/functions.cpp:5450-5600) per tree, {nthreads} threads",
            "s": t_tc, "same_support_as_gpu": bool(bad == 0 and np.array_equal(want, sup))}
    # a20: parsimony change counts per edge (ancestralBitReverse) on the C2 join tree
    (pstate, plen), t_par = _timed(lambda: L.ancestral_bit(words, bedge), reps=3)
    t0 = time.perf_counter()
    ostate, olen = O.ancestral_bit(words, bedge)
    t_cpar = time.perf_counter() - t0
    res["C2_binary"]["ancestralBitReverse"] = {"gpu_s": t_par, "cpu_s": t_cpar, "edges": int(len(plen)),
                                               "total_changes": int(plen.sum()),
                                               "identical": bool(np.array_equal(pstate, ostate) and
                                                                 np.array_equal(plen, olen))}
    # the GPU radius lists of the sample rows are those of the full run restricted to j < sub
    g_c, g_i = L.radius_bit(np.ascontiguousarray(words[:sub].T), wr, 4)
    res["C2_binary"]["radiusNeighbor_r4"]["sample_identical"] = bool(np.array_equal(g_c, c0) and
                                                                     np.array_equal(g_i, i0))
    if twin:
        tsub = 2000
        t0 = time.perf_counter()
        tj = T.greedy_join_edge_bit(words[:tsub], ancestral_type=1)
        t_tj = time.perf_counter() - t0
        gj, _, _ = L.join_bit(words[:tsub], None, 1)
        t0 = time.perf_counter()
        tc, _ = T.radius_weighted_rows(words[:sub], 4, 0, sub, nthreads)
        t_tr = time.perf_counter() - t0
        res["C2_binary"]["reference_cpu"] = {
            "joinEdgeBitReverse": {"function": "greedyJoinEdgeBitReverse (src/functions.cpp:3316-3461), 1 thread",
                                   "sample": f"first {tsub} cells", "s_sample": t_tj,
                                   "same_tree_as_gpu": bool(same_clades(tj.T, gj, tsub))},
            "radiusNeighbor_r4": {"function": f"radiusWeightedParallel (src/functions.cpp:1825-1857) per row, "
                                              f"{nthreads} threads", "sample": f"first {sub} cells",
                                  "s_sample": t_tr, "same_counts_as_gpu": bool(np.array_equal(tc, g_c))}}
    # C3: DNA 20,000 x 2,000 HKY85 through fasta2bin coding, radiusNeighborDNA at Hamming 20
    states, _ = synth.hky85_alignment(20_000, 2000, 4.0, [0.3, 0.2, 0.2, 0.3], 0.01, 0.02, seed=13)
    raw, var = synth.dna_to_fasta2bin(states)
    lvalid = int(var.sum())
    (dc, di), t_dna = _timed(lambda: L.radius_dna(raw, lvalid - 20))
    sub = 4000
    t0 = time.perf_counter()
    oc, oi = O.radius_dna(raw[:sub], lvalid - 20, nthreads)
    t_cd = time.perf_counter() - t0
    gc, gi = L.radius_dna(raw[:sub], lvalid - 20)
    t0 = time.perf_counter()
    ocf, oif = O.radius_dna(raw, lvalid - 20, nthreads)
    t_cdf = time.perf_counter() - t0
    dna_full_same = bool(np.array_equal(dc, ocf) and np.array_equal(di, oif))
    res["C3_radiusNeighborDNA"] = {
        "workload": f"HKY85 20000 x 2000 (kappa 4, pi .3/.2/.2/.3, Exp(0.01) Yule), 2% gaps, fasta2bin coding, "
                    f"{lvalid} variable columns; shared >= L_valid - 20",
        "gpu_s": t_dna, "pairs": 20_000 * 20_000, "neighbours": int(dc.sum()),
        "cpu_sample": f"first {sub} sequences", "cpu_s_sample": t_cd, "cpu_cores": nthreads,
        "sample_identical": bool(np.array_equal(gc, oc) and np.array_equal(gi, oi)),
        "identical": dna_full_same, "cpu_full_s": t_cdf}
    if twin:
        t0 = time.perf_counter()
        tc, _ = T.radius_weighted_dna_rows(raw[:sub], lvalid - 20, 0, sub, nthreads)
        res["C3_radiusNeighborDNA"]["reference_cpu"] = {
            "function": f"radiusWeightedDNAParallel (src/functions.cpp:4021-4036) per row, {nthreads} threads",
            "sample": f"first {sub} sequences", "s_sample": time.perf_counter() - t0,
            "same_counts_as_gpu": bool(np.array_equal(tc, gc))}
    # fasta2bin on the C3 alignment written as FASTA, beside the reference's
    # own fasta2bin (host code, built from cu/fasta2bin.cu into oracle/_ref)
    import subprocess
    import tempfile
    letters = np.frombuffer(b"ACGT-", dtype=np.uint8)
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "c3.fasta")
        with open(src, "wb") as f:
            for i in range(states.shape[0]):
                f.write(b">s%d\n" % i)
                f.write(letters[states[i]].tobytes())
                f.write(b"\n")
        ours = os.path.join(ROOT, "casphy_b200", "bin", "fasta2bin")
        ref = os.path.join(ROOT, "oracle", "_ref", "fasta2bin")
        t0 = time.perf_counter()
        subprocess.run([ours, src, os.path.join(d, "a")], check=True, stdout=subprocess.DEVNULL)
        t_f = time.perf_counter() - t0
        f2b = {"workload": "the C3 alignment (20000 x 2000, 2% gaps) as a FASTA file", "casphy_s": t_f}
        if os.path.exists(ref):
            t0 = time.perf_counter()
            subprocess.run([ref, src, os.path.join(d, "b")], check=True, stdout=subprocess.DEVNULL)
            f2b["reference_s"] = time.perf_counter() - t0
            same = all(open(os.path.join(d, "a" + x), "rb").read() == open(os.path.join(d, "b" + x), "rb").read()
                       for x in (".bin", "_names.txt", "_positions.txt"))
            f2b["identical_files"] = bool(same)
        res["C3_fasta2bin"] = f2b
    # tipMerge on 140,000 tips' clustered neighbour lists (avg 18 per row)
    counts, nidx = synth.neighbour_lists(140_000, 4)
    mem, t_tm = _timed(lambda: L.tip_merge(counts, nidx, 0.4))
    t0 = time.perf_counter()
    omem = O.tip_merge(counts, nidx, 0.4)
    t_ctm = time.perf_counter() - t0
    res["tipMerge"] = {"workload": "140000 tips, clustered symmetric neighbour lists (synth.neighbour_lists, "
                                   "seed 4, mean 18 per row), pShared 0.4",
                       "gpu_s": t_tm, "cpu_s": t_ctm, "categories": int(mem.max()) + 1,
                       "identical": bool(np.array_equal(mem, omem))}
    return res


def reference_gpu_rows(budget_s=240.0):
    """The reference's own GPU tools (built from cu/*.cu for sm_100a into
    oracle/_ref/ by oracle/Makefile) against the drop-in executables on the
    same input files: process wall clock of each, one run each after one
    untimed run of both (CUDA start-up is inside both), output files compared
    byte for byte.  A reference run that exceeds its time limit is reported as
    such; the rows stop when the whole budget is spent."""
    import tempfile
    from casphy_b200 import bootstrap as B
    from casphy_b200 import formats, synth
    ref_bin = os.path.join(ROOT, "oracle", "_ref")
    our_bin = os.path.join(ROOT, "casphy_b200", "bin")
    if not os.path.isdir(ref_bin):
        return {"unavailable": "oracle/_ref was not built (needs the CasPhy source tree at build time)"}
    t_start = time.perf_counter()
    rows = {}

    def run(exe, args, cwd, timeout):
        t0 = time.perf_counter()
        try:
            r = subprocess.run([exe] + args, cwd=cwd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                               timeout=timeout)
            return time.perf_counter() - t0, r.returncode
        except subprocess.TimeoutExpired:
            return None, "timeout"

    def row(name, ref_exe, our_exe, args, outputs, setup, timeout=120.0, reps=1):
        left = budget_s - (time.perf_counter() - t_start)
        if left < 10:
            rows[name] = {"skipped": "bench budget for these rows spent"}
            return
        with tempfile.TemporaryDirectory() as d:
            desc = setup(d)
            res = {"workload": desc}
            got = {}
            for who, exe in (("reference", os.path.join(ref_bin, ref_exe)), ("casphy", os.path.join(our_bin, our_exe))):
                if not os.path.exists(exe):
                    res[who + "_s"] = None
                    continue
                run(exe, args, d, min(timeout, left))  # untimed first run
                times = []
                for _ in range(reps):
                    dt, rc = run(exe, args, d, min(timeout, left))
                    if dt is None or rc != 0:
                        times = None
                        res[who + "_error"] = rc
                        break
                    times.append(dt)
                res[who + "_s"] = min(times) if times else None
                got[who] = {o: open(os.path.join(d, o), "rb").read() for o in outputs
                            if os.path.exists(os.path.join(d, o))}
                for o in outputs:
                    if os.path.exists(os.path.join(d, o)):
                        os.remove(os.path.join(d, o))
            if res.get("reference_s") and res.get("casphy_s"):
                res["speedup"] = res["reference_s"] / res["casphy_s"]
            if "reference" in got and "casphy" in got:
                res["identical_files"] = bool(got["reference"] == got["casphy"] and
                                              len(got["casphy"]) == len(outputs))
            rows[name] = res

    # C1: joinEdgeIndel, 1,024 cells x 256 sites (the reference binary with MAXCOL 1000)
    def c1(d):
        raw = synth.lineage_states(1024, 256, 12, 0.04, 64, 1.5, 0.10, seed=21)
        codes, ns = synth.regularize(raw)
        formats.write_mat(os.path.join(d, "c1.tbmat"), codes)
        formats.write_mat(os.path.join(d, "c1.tipSize"), np.ones((1024, 1), np.uint32))
        formats.write_f64(os.path.join(d, "c1.w"), np.ones((ns, 256)))
        c1.ns = ns
        return "joinEdgeIndel, indel 1024 cells x 256 sites (C1), unit weights"
    raw1 = synth.lineage_states(1024, 256, 12, 0.04, 64, 1.5, 0.10, seed=21)
    ns1 = synth.regularize(raw1)[1]
    row("C1_joinEdgeIndel", "joinEdgeIndel", "joinEdgeIndel", ["c1", "c1.w", str(ns1), "0", "2"],
        ["c1.edge2", "c1.nodeState2"], c1)

    # C5 prefix: joinEdgeIndel at 1,024 sites (the reference built with MAXCOL 1024)
    codes5, ns5, _ = gen_workload(5000)

    def c5(d):
        formats.write_mat(os.path.join(d, "c5.tbmat"), codes5)
        formats.write_mat(os.path.join(d, "c5.tipSize"), np.ones((codes5.shape[0], 1), np.uint32))
        formats.write_f64(os.path.join(d, "c5.w"), np.ones((ns5, codes5.shape[1])))
        return "joinEdgeIndel, first 5000 cells of the 200000 x 1024 indel workload (C5 prefix), unit weights"
    row("C5_prefix5k_joinEdgeIndel", "joinEdgeIndel_MAXCOL1024", "joinEdgeIndel",
        ["c5", "c5.w", str(ns5), "0", "2"], ["c5.edge2", "c5.nodeState2"], c5, timeout=180.0)

    # C2: joinEdgeBitReverse, radiusNeighbor (shared >= 4 and a sparse radius), TransferDisStream
    words = synth.binary_workload(10_000, 512, 16, 0.03, 0.05, seed=23)

    def c2(d):
        formats.write_mat(os.path.join(d, "c2.tbmat"), words)
        formats.write_f64(os.path.join(d, "c2.w"), np.ones(512))
        formats.write_mat(os.path.join(d, "c2.bmat"), words.T)
        return "base-editor 10000 cells x 512 sites (C2)"
    row("C2_joinEdgeBitReverse_type1", "joinEdgeBitReverse", "joinEdgeBitReverse", ["c2", "c2.w", "1"],
        ["c2.edge2", "c2.nodeState2"], c2, timeout=180.0)
    for r in (4, RADIUS_SPARSE):
        row(f"C2_radiusNeighbor_r{r}", "radiusNeighbor", "radiusNeighbor", ["c2", str(r)],
            ["c2.idx", "c2.nNeighbor"], c2, timeout=180.0)
    edge, _, _ = __import__("casphy_b200.lib", fromlist=["x"]).join_bit(words, None, 1)
    truth = synth.lineage_clades(10_000, 16, seed=23)
    est = B.clade_bits(edge, 10_000, (10_000 + 31) // 32)

    def td(d):
        formats.write_mat(os.path.join(d, "td_y"), truth)
        formats.write_mat(os.path.join(d, "td_x"), est)
        return "TransferDisStream, true tree's 9998 clades against the C2 join tree's (313 words), 1 GPU"
    row("C2_TransferDisStream", "TransferDisStream", "TransferDisStream", ["td_y", "td_x", "td", "10000"],
        ["td_ymin.bin", "td_xmin.bin"], td, timeout=180.0)

    # C3: radiusNeighborDNA at Hamming 20 on the fasta2bin matrix
    states, _ = synth.hky85_alignment(20_000, 2000, 4.0, [0.3, 0.2, 0.2, 0.3], 0.01, 0.02, seed=13)
    raw3, var = synth.dna_to_fasta2bin(states)
    lv = int(var.sum())

    def c3(d):
        formats.write_mat(os.path.join(d, "c3.tbmat"), raw3)
        return f"radiusNeighborDNA, HKY85 20000 x 2000 via fasta2bin coding, shared >= {lv} - 20 (C3)"
    row("C3_radiusNeighborDNA", "radiusNeighborDNA", "radiusNeighborDNA", ["c3", str(lv - 20)],
        ["c3.idx", "c3.nNeighbor"], c3, timeout=180.0)
    rows["timing"] = ("process wall clock (CUDA start-up, file reads and writes included for both), best of one "
                      "run after one untimed run of each")
    return rows


def sharded_suite(L, world, rank, local):
    """The parts of the path that shard, over all ranks (one GPU each, NCCL
    on the ranks' GPUs): radius search by query-row blocks, TransferDisStream
    by y-row blocks, bootstrap replicates k::world.  Each part is timed on the
    device around the whole sharded call (compute and exchange), max over
    ranks; rank 0 also checks the gathered result against one-GPU calls."""
    import torch
    from casphy_b200 import bootstrap as B
    from casphy_b200 import shard, synth
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    res = {"ranks": world, "exchange": "NCCL all-gather / all-reduce of int32 views of u32 data on the GPUs"}

    def timed(fn):
        barrier(world)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return out, max_over_ranks(a.elapsed_time(b) / 1e3, world)

    words = synth.binary_workload(10_000, 512, 16, 0.03, 0.05, seed=23)
    bmat = np.ascontiguousarray(words.T)
    wr = np.ones(512)
    rows = lambda lo, hi: L.radius_bit_rows(bmat, wr, RADIUS_SPARSE, lo, hi)  # noqa: E731
    timed(lambda: shard.radius_sharded(rows, 10_000, device=dev))  # warm-up
    (c, i), t = timed(lambda: shard.radius_sharded(rows, 10_000, device=dev))
    res[f"C2_radiusNeighbor_r{RADIUS_SPARSE}"] = {"s": t}
    if rank == 0:
        c1, i1 = L.radius_bit(bmat, wr, RADIUS_SPARSE)
        res[f"C2_radiusNeighbor_r{RADIUS_SPARSE}"]["identical_to_one_gpu"] = bool(
            np.array_equal(c, c1) and np.array_equal(i, i1))
    states, _ = synth.hky85_alignment(20_000, 2000, 4.0, [0.3, 0.2, 0.2, 0.3], 0.01, 0.02, seed=13)
    raw, var = synth.dna_to_fasta2bin(states)
    lv = int(var.sum())
    drows = lambda lo, hi: L.radius_dna_rows(raw, lv - 20, lo, hi)  # noqa: E731
    timed(lambda: shard.radius_sharded(drows, 20_000, device=dev))
    (dc, di), t = timed(lambda: shard.radius_sharded(drows, 20_000, device=dev))
    res["C3_radiusNeighborDNA"] = {"s": t}
    if rank == 0:
        c1, i1 = L.radius_dna(raw, lv - 20)
        res["C3_radiusNeighborDNA"]["identical_to_one_gpu"] = bool(np.array_equal(dc, c1) and np.array_equal(di, i1))
    edge, _, _ = L.join_bit(words, None, 1)
    truth = synth.lineage_clades(10_000, 16, seed=23)
    est = B.clade_bits(edge, 10_000, (10_000 + 31) // 32)
    timed(lambda: shard.transfer_dis_sharded(L.transfer_dis, truth, est, 10_000, device=dev))
    td, t = timed(lambda: shard.transfer_dis_sharded(L.transfer_dis, truth, est, 10_000, device=dev))
    res["C2_TransferDisStream"] = {"s": t}
    if rank == 0:
        one = L.transfer_dis(truth, est, 10_000)
        res["C2_TransferDisStream"]["identical_to_one_gpu"] = bool(all(np.array_equal(a, b) for a, b in zip(td, one)))
    bwords = synth.binary_workload(10_000, 512, 16, 0.03, 0.05, seed=11)
    full_edge, _, _ = L.join_bit(bwords, None, 1)
    off, cells, w = B.make_replicates(10_000, 512, 200, 2000, 10_000, seed=12)
    bs = lambda: shard.bootstrap_sharded(L.bootstrap_bit, bwords, full_edge, off, cells, w, device=dev)  # noqa: E731
    bs()
    (sup, ymin, ysize), t = timed(bs)
    res["C4_bootstrap_200"] = {"s": t}
    if rank == 0:
        one = L.bootstrap_bit(bwords, full_edge, off, cells, w, threshold=0.05)
        res["C4_bootstrap_200"]["identical_to_one_gpu"] = bool(
            np.array_equal(sup, one["support"]) and np.array_equal(ymin, one["ymin"]))
    return res


def blopt_c5(L, codes, nstate, edge):
    """Irreversible edit-model branch lengths on the 200,000-cell join tree, and
    the reference's parsimony change counts (charAncestralEC) on the same tree."""
    e = np.asarray(edge, dtype=np.uint32).reshape(-1, 2)
    raw = codes.astype(np.int32) - 1  # .tbmat coding back to -1 missing, 0 unedited, alleles
    (pstate, plen), t_par = _timed(lambda: L.ancestral_char(raw, e))
    import oracle as O
    t0 = time.perf_counter()
    _, olen = O.ancestral_char(raw, e)
    t_cpar = time.perf_counter() - t0
    par = {"gpu_s": t_par, "cpu_s": t_cpar, "edges": int(len(plen)), "total_changes": int(plen.sum()),
           "identical": bool(np.array_equal(plen, olen))}
    t0 = np.full(len(e), 0.05)
    t_end, st = L.felsenstein_optimize(e, t0, codes, model="irreversible", rate=1.0, nallele=int(nstate),
                                       rel_tol=1e-9, max_iter=1000)
    # FP64 pruning of the same tree at the final lengths (compact form of the
    # edit model), allele frequencies as the library takes them by default
    q = O.tip_allele_freqs(codes, int(nstate))
    ll64 = O.loglik_irreversible(e, t_end, codes, int(nstate), q, 1.0)
    # the same optimisation started from the parsimony counts
    from casphy_b200.branch_lengths import parsimony_start
    tw = parsimony_start(e, pstate, plen, raw.shape[0], rate=1.0)
    del pstate
    tw_end, sw = L.felsenstein_optimize(e, tw, codes, model="irreversible", rate=1.0, nallele=int(nstate),
                                        rel_tol=1e-9, max_iter=1000)
    llw64 = O.loglik_irreversible(e, tw_end, codes, int(nstate), q, 1.0)
    par["warm_start"] = {
        "start": "t = -log(1 - k/n0) per edge from the change counts k and the parent's unedited sites n0",
        "adjoint_s": sw["seconds"], "iterations": sw["iterations"], "evaluations": sw["evaluations"],
        "loglik_start": sw["loglik_start"], "loglik_end": sw["loglik_end"],
        "loglik_fp64_at_end": llw64, "loglik_rel_err_vs_fp64": abs(sw["loglik_end"] - llw64) / abs(llw64),
        "loglik_end_rel_diff_to_flat_start": (sw["loglik_end"] - st["loglik_end"]) / abs(st["loglik_end"])}
    return {"workload": "irreversible edit model (rate 1, allele frequencies from the tips) on the 200000-cell "
                        "join tree of the headline workload, 1024 sites; start at t = 0.05",
            "adjoint_s": st["seconds"], "iterations": st["iterations"], "evaluations": st["evaluations"],
            "eval_graph_s": st["eval_seconds"],
            "ms_per_evaluation": st["seconds"] * 1e3 / max(st["evaluations"], 1),
            "loglik_start": st["loglik_start"], "loglik_end": st["loglik_end"],
            "loglik_fp64_at_end": ll64, "loglik_rel_err_vs_fp64": abs(st["loglik_end"] - ll64) / abs(ll64),
            "fp64_oracle": "oracle_loglik_irreversible (compact FP64 pruning) at the final lengths, allele "
                           "frequencies from the tips' counts",
            "levels_inside": st["levels_inside"], "levels_outside": st["levels_outside"],
            "charAncestralEC": par}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="casphy", choices=["casphy", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-extras", action="store_true", help="skip the bootstrap and branch-length measurements")
    ap.add_argument("--only", choices=["bootstrap", "blopt", "rows"], default=None,
                    help="run one of the extra measurements alone (profiling)")
    ap.add_argument("--no-plain", action="store_true", help="with --only bootstrap: skip the plain runs")
    ap.add_argument("--cells", type=int, default=None,
                    help="profiling only: use the first N cells of the workload")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc

    import ctypes as C
    import torch
    import casphy_b200.lib as L

    lib = L.lib()
    torch.cuda.set_device(local)
    if args.only:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        res = (bootstrap_suite(L, plain=not args.no_plain) if args.only == "bootstrap" else
               blopt_suite(L) if args.only == "blopt" else rows_suite(L, os.cpu_count() or 1))
        if rank == 0:
            print(json.dumps({args.only: res}), flush=True)
        return 0
    codes, nstate, weight = gen_workload(args.cells)
    ntip, ncol = codes.shape
    d_codes = torch.from_numpy(codes.view(np.int32)).cuda()
    d_state = torch.empty((ntip - 1, ncol), dtype=torch.int32, device="cuda")
    edge = np.zeros(2 * (2 * ntip - 2), dtype=np.uint32)
    wflat = np.ascontiguousarray(weight.reshape(-1))
    tip = np.ones(ntip, dtype=np.uint32)
    stream = torch.cuda.current_stream()
    st = L.JoinStats()

    def step():
        rc = lib.casphy_join_indel_dev(ntip, ncol, C.c_void_p(d_codes.data_ptr()), nstate, wflat, tip, 0, 2.0,
                                       edge, C.c_void_p(d_state.data_ptr()), C.byref(st),
                                       C.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise L.CasphyError(rc, "casphy_join_indel_dev")

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()
    stats = st.as_dict()
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        join_ms, launches = [], 0
        for _ in range(args.steps):
            step()
            join_ms.append(st.join_loop_ms)
            launches += st.kernel_launches
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    elapsed = ev0.elapsed_time(ev1) / 1e3
    elapsed = max_over_ranks(elapsed, world)
    # pair-scores of a tree counted as (N-1)^2, the count of the reference's
    # CPU join (greedyJoinEdge2) that the reference arm reports, so that the
    # two arms' values compare as tree times; the lazy loop's own count (the
    # reference GPU loop's schedule, from the oracle) is reported beside it
    pairs = float(ntip - 1) ** 2
    value = pairs * args.steps * world / elapsed
    # the tree against the oracle's digest of the same workload
    identical, digest_case = None, {None: "c5_200k", 50_000: "c5_50k", 20_000: "c5_20k"}.get(args.cells)
    hashes = {}
    try:
        with open(os.path.join(ROOT, "tests", "golden", "scale_hashes.json")) as f:
            hashes = json.load(f)
    except OSError:
        pass
    if digest_case in hashes:
        import hashlib
        ref = hashes[digest_case]
        sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()  # noqa: E731
        identical = bool(sha(edge[: 2 * (2 * ntip - 2)]) == ref["edge_sha256"] and
                         sha(d_state.cpu().numpy().view(np.uint32)) == ref["state_sha256"])

    # end to end through the host-buffer entry point
    h_codes = torch.from_numpy(codes.view(np.int32)).pin_memory()
    h_state = torch.empty((ntip - 1, ncol), dtype=torch.int32).pin_memory()
    hcodes_np = h_codes.numpy().view(np.uint32)
    hstate_np = h_state.numpy().view(np.uint32)
    e2e_steps = max(1, args.e2e_steps)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        rc = lib.casphy_join_indel(ntip, ncol, hcodes_np, nstate, wflat, tip, 0, 2.0, edge,
                                   hstate_np, C.byref(st))
        if rc != 0:
            raise L.CasphyError(rc, "casphy_join_indel")
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
    e2e_val = pairs * e2e_steps * world / e2e_s

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        # samples are re-regularised exactly as R would for those cells
        sub_codes, sub_ns, sub_w = gen_workload(CPU_SAMPLE_CELLS)
        p, dt = cpu_port_run(sub_codes, sub_ns, sub_w, nthreads)
        port = {"value": p / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
                "sample": (f"first {CPU_SAMPLE_CELLS} cells of this workload ({p:.0f} pair-scores in {dt:.1f} s), "
                           "greedy join restated from cu/joinEdgeIndel.cu")}
        if cpu_twin_available():
            tc, tn, tw = gen_workload(TWIN_SAMPLE_CELLS)
            p2, dt2 = cpu_twin_run(tc, tn, tw)
            cpu = {"value": p2 / dt2, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": (f"first {TWIN_SAMPLE_CELLS} cells of this workload ({p2:.0f} pair-scores in "
                              f"{dt2:.1f} s): greedyJoinEdge2 (src/functions.cpp:1880-2017), the reference's CPU "
                              "join, compiled from its source; single-threaded as in R"),
                   "port": port}
        else:
            cpu = port

    hbm, how = peaks()
    jl = float(np.mean(join_ms))
    achieved = stats["alg_bytes_join"] / (jl / 1e3) / 1e9 if jl > 0 else 0.0
    roof = {"kernel": "k_join (persistent join loop)", "bound": "hbm", "achieved": achieved, "peak": hbm,
            "unit": "GB/s", "frac": achieved / hbm, "peak_source": f"{how} hbm_gbs",
            "traffic": traffic_from_profile("k_join"),
            "alg_bytes_per_launch": stats["alg_bytes_join"], "launch_ms": jl,
            "alg_bytes_rule": "1/8 byte per (candidate, query site): one bitset bit",
            "two_byte_rule": {"note": "2 bytes per (candidate, query site), the u16-code rule of the scope table",
                              "achieved": achieved * 16, "frac": achieved * 16 / hbm},
            "init_scan": {"alg_bytes": stats["alg_bytes_init"], "ms": stats["init_scan_ms"],
                          "achieved_gbs": stats["alg_bytes_init"] / (stats["init_scan_ms"] / 1e3) / 1e9
                          if stats["init_scan_ms"] else None}}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE, "data": "synthetic",
            "config": {"workload": workload_name() if args.cells is None else
                       f"first {ntip} cells of: " + workload_name(), "cells": ntip, "sites": ncol, "nState": int(nstate),
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs (800 MB codes) larger than the 126 MB L2; no flush between steps"},
            "tree_s": elapsed / args.steps,
            "pair_scores_counted": "(N-1)^2 per tree, as the reference's CPU join computes",
            "identical": identical,
            "identical_to": (f"sha256 of the oracle's edge list and node states for this workload "
                             f"(tests/golden/scale_hashes.json {digest_case})" if identical is not None else None),
            "tree_stats": dict({k: stats[k] for k in ("joins", "stale_recomputes", "pair_scores", "compactions",
                                                      "phases", "refreshes", "int_path")},
                               reference_loop_pair_scores=hashes.get(digest_case, {}).get("pair_scores"),
                               reference_loop_stale_rescans=hashes.get(digest_case, {}).get("stale_recomputes")),
            "e2e": {"value": e2e_val, "unit": UNIT,
                    "h2d_bytes_per_step": int(codes.nbytes + wflat.nbytes + tip.nbytes),
                    "d2h_bytes_per_step": int(edge.nbytes + hstate_np.nbytes), "tree_s": e2e_s / e2e_steps},
            "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary()}
    if cpu is not None and cpu.get("kind") == "reference":
        # the headline as tree times: the reference CPU join's rate extrapolated
        # to (N-1)^2 pair-scores (its N x N float cache needs 160 GB at 200k)
        cpu_tree_s = pairs / cpu["value"]
        line["vs_reference_tree_time"] = {"reference_cpu_tree_s_extrapolated": cpu_tree_s,
                                          "casphy_e2e_tree_s": e2e_s / e2e_steps,
                                          "ratio": cpu_tree_s / (e2e_s / e2e_steps)}
    if world > 1 and args.cells is None and not args.no_extras:
        line["sharded"] = sharded_suite(L, world, rank, local)  # every rank: collectives inside
    if rank == 0 and world == 1 and args.cells is None and not args.no_extras:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        line["reference_gpu"] = reference_gpu_rows()
        line["blopt_c5"] = blopt_c5(L, codes, nstate, edge)
        line["bootstrap"] = bootstrap_suite(L)
        line["blopt"] = blopt_suite(L)
        line["rows"] = rows_suite(L, os.cpu_count() or 1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
