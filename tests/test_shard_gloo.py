"""Sharded TransferDisStream, radius lists and bootstrap on two and three gloo
ranks (CPU, oracle as the per-rank compute) equal the one-process results;
three ranks split 61 rows, 37 columns and 5 replicates unevenly."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_bootstrap(words, full_edge, off, cells, w, threshold=0.05):
    import oracle as O
    from casphy_b200 import bootstrap as B
    N = words.shape[0]
    fb = B.clade_bits(full_edge, N, (N + 31) // 32)
    nrep = len(off) - 1
    ymin = np.zeros((nrep, N - 2), np.uint32)
    ysize = np.zeros((nrep, N - 2), np.uint32)
    for r in range(nrep):
        ymin[r], ysize[r] = B.plain_replicate(O, words, fb, cells[off[r]:off[r + 1]], w[r])
    return {"support": B.support_counts(ymin, ysize, threshold), "ymin": ymin, "ysize": ysize}


def _worker(rank, world, port, q):
    import sys
    for p in (ROOT, os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import oracle as O
    from casphy_b200 import bootstrap as B
    from casphy_b200 import shard, synth
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        y = rng.integers(0, 2**32, size=(61, 5), dtype=np.uint64).astype(np.uint32)
        x = rng.integers(0, 2**32, size=(37, 5), dtype=np.uint64).astype(np.uint32)
        td = shard.transfer_dis_sharded(O.transfer_dis, y, x, 150)
        words = synth.binary_workload(160, 64, 8, 0.05, 0.05, seed=6)
        full_edge, _, _ = O.join_bit(words, None, 1)
        off, cells, w = B.make_replicates(160, 64, 5, 40, 160, seed=7)
        bs = shard.bootstrap_sharded(_oracle_bootstrap, words, full_edge, off, cells, w)
        bmat = np.ascontiguousarray(words.T)
        fc, fi = O.radius_bit(bmat, np.ones(64), 3)
        starts = np.concatenate([[0], np.cumsum(fc.astype(np.int64))])

        def rows(lo, hi):  # one rank's share, cut from the oracle's full lists
            return fc[lo:hi], fi[starts[lo]:starts[hi]]

        rd = shard.radius_sharded(rows, len(fc))
        q.put((rank, td, bs, rd, (fc, fi)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharding_matches_one_process(world):
    import oracle as O
    from casphy_b200 import bootstrap as B
    from casphy_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(5)
    y = rng.integers(0, 2**32, size=(61, 5), dtype=np.uint64).astype(np.uint32)
    x = rng.integers(0, 2**32, size=(37, 5), dtype=np.uint64).astype(np.uint32)
    want_td = O.transfer_dis(y, x, 150)
    words = synth.binary_workload(160, 64, 8, 0.05, 0.05, seed=6)
    full_edge, _, _ = O.join_bit(words, None, 1)
    off, cells, w = B.make_replicates(160, 64, 5, 40, 160, seed=7)
    want_bs = _oracle_bootstrap(words, full_edge, off, cells, w)
    for _, td, bs, rd, full in res:
        assert np.array_equal(rd[0], full[0]) and np.array_equal(rd[1], full[1])
        for a, b in zip(td, want_td):
            assert np.array_equal(a, b)
        assert np.array_equal(bs[0], want_bs["support"])
        assert np.array_equal(bs[1], want_bs["ymin"]) and np.array_equal(bs[2], want_bs["ysize"])


def test_block_alignment():
    from casphy_b200.shard import block
    for n in (0, 1, 7, 8, 61, 1000):
        for world in (1, 2, 3, 8):
            cover = []
            for r in range(world):
                lo, hi = block(n, world, r, align=8)
                assert hi == lo or lo % 8 == 0
                cover.extend(range(lo, hi))
            assert cover == list(range(n))
