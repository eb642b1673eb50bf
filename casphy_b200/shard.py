"""Multi-GPU partitioning of the parts of the path that shard (one process
per GPU, torch.distributed for the exchange).

* Bootstrap replicates are independent units: rank k runs replicates
  k, k + world, ...; the per-clade support counts are summed (all-reduce SUM)
  and the per-replicate TransferDisStream rows are gathered.
* Radius search splits the query rows into contiguous blocks (each row's
  list depends only on that row); counts and lists are all-gathered.
* TransferDisStream splits its y rows (cu/TransferDisStream.cu runs y chunks
  on several GPUs the same way, :130-344): every rank takes a block of whole
  8-row groups, so the groups the x-side minimum is formed over stay aligned
  as in a one-GPU run; x minima are combined with all-reduce MIN.
* The greedy joins do not shard (every join depends on the previous argmax):
  several GPUs run independent trees (replicas).

Every exchanged array is u32 data viewed as int32 (bit for bit; the values
that are reduced, counts and distances, are below 2^31), placed on `device`
when one is given (the rank's GPU, for NCCL) and on the host otherwise (gloo).

`compute` is the single-device function (casphy_b200.lib on a GPU); tests
pass the CPU oracle instead to check the partitioning on gloo ranks.
"""
from __future__ import annotations

import numpy as np


def block(n: int, world: int, rank: int, align: int = 1):
    """[lo, hi) of rank's contiguous share of n items, cut at multiples of align."""
    groups = (n + align - 1) // align
    per = (groups + world - 1) // world
    lo = min(rank * per * align, n)
    hi = min((rank + 1) * per * align, n)
    return lo, hi


def _dev(a, device):
    """u32 array -> int32 tensor (same bits) on device (host when None)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32))
    return t.to(device) if device is not None else t


def _host(t):
    """int32 tensor -> u32 array (same bits)."""
    return t.cpu().numpy().view(np.uint32)


def transfer_dis_sharded(compute, y, x, ntip, group=None, device=None):
    """TransferDisStream over world ranks; every rank returns the full
    (ymin, ysize, xmin, xsize)."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    y = np.ascontiguousarray(y, dtype=np.uint32)
    x = np.ascontiguousarray(x, dtype=np.uint32)
    ny, ncol = y.shape
    lo, hi = block(ny, world, rank, align=8)
    ymin_l, ysize_l, xmin_l, xsize = compute(y[lo:hi], x, ntip) if hi > lo else (
        np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.full(len(x), 32 * ncol, np.uint32), None)
    if xsize is None:
        _, _, _, xsize = compute(y[:0], x, ntip)
    xm = _dev(xmin_l, device)
    dist.all_reduce(xm, op=dist.ReduceOp.MIN, group=group)
    # gather the y slices (fixed-size buffers: the largest share)
    share = block(ny, world, 0, align=8)[1]
    buf = np.zeros((2, share), dtype=np.uint32)
    buf[0, :hi - lo] = ymin_l
    buf[1, :hi - lo] = ysize_l
    t = _dev(buf, device)
    parts = [t.new_zeros(t.shape) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    ymin = np.zeros(ny, np.uint32)
    ysize = np.zeros(ny, np.uint32)
    for k, p in enumerate(parts):
        a, b = block(ny, world, k, align=8)
        p = _host(p)
        ymin[a:b] = p[0, :b - a]
        ysize[a:b] = p[1, :b - a]
    return ymin, ysize, _host(xm).copy(), xsize


def bootstrap_sharded(compute, words, full_edge, offsets, cells, weights, threshold=0.05, group=None,
                      device=None):
    """Replicates k::world on rank k; returns (support over all replicates,
    ymin, ysize in replicate order) on every rank.  `compute` has the
    signature of casphy_b200.lib.bootstrap_bit."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    offsets = np.asarray(offsets, dtype=np.int64)
    nrep = len(offsets) - 1
    mine = list(range(rank, nrep, world))
    nX = np.asarray(words).shape[0] - 2
    per = (nrep + world - 1) // world
    buf = np.zeros((2, per, nX), np.uint32)
    sup = np.zeros(nX, np.uint32)
    if mine:
        sub_cells = np.concatenate([cells[offsets[r]:offsets[r + 1]] for r in mine])
        sub_off = np.concatenate([[0], np.cumsum([offsets[r + 1] - offsets[r] for r in mine])]).astype(np.uint32)
        got = compute(words, full_edge, sub_off, sub_cells, np.asarray(weights)[mine], threshold=threshold)
        sup[:] = got["support"]
        buf[0, :len(mine)] = got["ymin"]
        buf[1, :len(mine)] = got["ysize"]
    s = _dev(sup, device)
    dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    t = _dev(buf, device)
    parts = [t.new_zeros(t.shape) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    ymin = np.zeros((nrep, nX), np.uint32)
    ysize = np.zeros((nrep, nX), np.uint32)
    for k, p in enumerate(parts):
        p = _host(p)
        for i, r in enumerate(range(k, nrep, world)):
            ymin[r] = p[0, i]
            ysize[r] = p[1, i]
    return _host(s).copy(), ymin, ysize


def radius_sharded(compute_rows, nrows, group=None, device=None):
    """Radius lists over world ranks.  compute_rows(lo, hi) returns (counts,
    idx) of query rows [lo, hi) (casphy_b200.lib.radius_bit_rows or
    radius_dna_rows with the matrix bound); every rank returns the full
    (counts, idx)."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    lo, hi = block(nrows, world, rank)
    counts, idx = compute_rows(lo, hi) if hi > lo else (np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    n = _dev(np.array([len(idx)], np.uint32), device)
    sizes = [n.new_zeros(n.shape) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(_host(x)[0]) for x in sizes]
    share = block(nrows, world, 0)[1]
    c = np.zeros(share, np.uint32)
    c[:hi - lo] = counts
    i = np.zeros(max(max(sizes), 1), np.uint32)
    i[:len(idx)] = idx
    tc, ti = _dev(c, device), _dev(i, device)
    pc = [tc.new_zeros(tc.shape) for _ in range(world)]
    pi = [ti.new_zeros(ti.shape) for _ in range(world)]
    dist.all_gather(pc, tc, group=group)
    dist.all_gather(pi, ti, group=group)
    out_c, out_i = [], []
    for k in range(world):
        a, b = block(nrows, world, k)
        out_c.append(_host(pc[k])[:b - a])
        out_i.append(_host(pi[k])[:sizes[k]])
    return np.concatenate(out_c).astype(np.uint32), np.concatenate(out_i).astype(np.uint32)
