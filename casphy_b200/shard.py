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


def _torch_u32(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32).astype(np.int64))


def transfer_dis_sharded(compute, y, x, ntip, group=None, device=None):
    """TransferDisStream over world ranks; every rank returns the full
    (ymin, ysize, xmin, xsize)."""
    import torch
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
    xm = _torch_u32(xmin_l)
    if device is not None:
        xm = xm.to(device)
    dist.all_reduce(xm, op=dist.ReduceOp.MIN, group=group)
    # gather the y slices (fixed-size buffers: the largest share)
    share = block(ny, world, 0, align=8)[1]
    buf = np.zeros((2, share), dtype=np.int64)
    buf[0, :hi - lo] = ymin_l
    buf[1, :hi - lo] = ysize_l
    t = torch.from_numpy(buf)
    if device is not None:
        t = t.to(device)
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    ymin = np.zeros(ny, np.uint32)
    ysize = np.zeros(ny, np.uint32)
    for k, p in enumerate(parts):
        a, b = block(ny, world, k, align=8)
        p = p.cpu().numpy()
        ymin[a:b] = p[0, :b - a]
        ysize[a:b] = p[1, :b - a]
    return ymin, ysize, xm.cpu().numpy().astype(np.uint32), xsize


def bootstrap_sharded(compute, words, full_edge, offsets, cells, weights, threshold=0.05, group=None,
                      device=None):
    """Replicates k::world on rank k; returns (support over all replicates,
    ymin, ysize in replicate order) on every rank.  `compute` has the
    signature of casphy_b200.lib.bootstrap_bit."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    offsets = np.asarray(offsets, dtype=np.int64)
    nrep = len(offsets) - 1
    mine = list(range(rank, nrep, world))
    nX = np.asarray(words).shape[0] - 2
    ymin_l = np.zeros((len(mine), nX), np.int64)
    ysize_l = np.zeros((len(mine), nX), np.int64)
    sup = np.zeros(nX, np.int64)
    if mine:
        sub_cells = np.concatenate([cells[offsets[r]:offsets[r + 1]] for r in mine])
        sub_off = np.concatenate([[0], np.cumsum([offsets[r + 1] - offsets[r] for r in mine])]).astype(np.uint32)
        got = compute(words, full_edge, sub_off, sub_cells, np.asarray(weights)[mine], threshold=threshold)
        sup[:] = got["support"]
        ymin_l[:] = got["ymin"]
        ysize_l[:] = got["ysize"]
    s = torch.from_numpy(sup)
    if device is not None:
        s = s.to(device)
    dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    per = (nrep + world - 1) // world
    buf = np.zeros((2, per, nX), np.int64)
    buf[0, :len(mine)] = ymin_l
    buf[1, :len(mine)] = ysize_l
    t = torch.from_numpy(buf)
    if device is not None:
        t = t.to(device)
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    ymin = np.zeros((nrep, nX), np.uint32)
    ysize = np.zeros((nrep, nX), np.uint32)
    for k, p in enumerate(parts):
        p = p.cpu().numpy()
        for i, r in enumerate(range(k, nrep, world)):
            ymin[r] = p[0, i]
            ysize[r] = p[1, i]
    return s.cpu().numpy().astype(np.uint32), ymin, ysize


def radius_sharded(compute_rows, nrows, group=None, device=None):
    """Radius lists over world ranks.  compute_rows(lo, hi) returns (counts,
    idx) of query rows [lo, hi) (casphy_b200.lib.radius_bit_rows or
    radius_dna_rows with the matrix bound); every rank returns the full
    (counts, idx)."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    lo, hi = block(nrows, world, rank)
    counts, idx = compute_rows(lo, hi) if hi > lo else (np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    n = torch.tensor([len(idx)], dtype=torch.int64)
    if device is not None:
        n = n.to(device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(x.item()) for x in sizes]
    share = block(nrows, world, 0)[1]
    c = np.zeros(share, np.int64)
    c[:hi - lo] = counts
    i = np.zeros(max(sizes) if sizes else 0, np.int64)
    i[:len(idx)] = idx
    tc, ti = torch.from_numpy(c), torch.from_numpy(i)
    if device is not None:
        tc, ti = tc.to(device), ti.to(device)
    pc = [torch.zeros_like(tc) for _ in range(world)]
    pi = [torch.zeros_like(ti) for _ in range(world)]
    dist.all_gather(pc, tc, group=group)
    dist.all_gather(pi, ti, group=group)
    out_c, out_i = [], []
    for k in range(world):
        a, b = block(nrows, world, k)
        out_c.append(pc[k].cpu().numpy()[:b - a])
        out_i.append(pi[k].cpu().numpy()[:sizes[k]])
    return np.concatenate(out_c).astype(np.uint32), np.concatenate(out_i).astype(np.uint32)
