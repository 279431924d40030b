"""The N > 1 paths on CPU with gloo, world size 2: max-over-ranks timing and
the column-sharded top-k gather/merge (equal to the unsharded top-k, with
fp16-rounded and with scaled scores)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as orc


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _scales(nb, N):
    rng = np.random.default_rng(3)
    return rng.uniform(0.5, 2.0, nb).astype(np.float32), rng.uniform(0.5, 2.0, N).astype(np.float32)


def _worker(rank, world, port, q):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root / "qpg-rotormap_b200"))
    sys.path.insert(0, str(root))
    from oracle import oracle as orc
    from rotormap import dist as rdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t = rdist.max_over_ranks([1.0 + rank, 5.0 - rank])
        rng = np.random.default_rng(0)
        E = np.array([0xC4, 0xC0, 0xB8, 0x00, 0x38, 0x40, 0x44], np.uint8)
        A = E[rng.integers(0, 7, (50, 64))]
        B = E[rng.integers(0, 7, (3001, 64))]
        lo, hi = rdist.shard_bounds(B.shape[0], world, rank)
        v, l = orc.topk_e4m3(A, B[lo:hi], 20, 0)
        gv, gl = rdist.gather_shard_topk(torch.from_numpy(v), torch.from_numpy(l), lo, 20)
        # scaled scores: shards rank with a unit row scale, the row scale comes after the merge
        sa, sb = _scales(A.shape[0], B.shape[0])
        v, l = orc.topk_e4m3(A, B[lo:hi], 20, 2, np.ones(A.shape[0], np.float32), sb[lo:hi])
        sv, sl = rdist.gather_shard_topk(torch.from_numpy(v), torch.from_numpy(l), lo, 20)
        sv = rdist.scale_rows(sv, torch.from_numpy(sa))
        q.put((rank, t, gv.numpy(), gl.numpy(), sv.numpy(), sl.numpy()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_gloo_timing_and_sharded_topk():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    rng = np.random.default_rng(0)
    E = np.array([0xC4, 0xC0, 0xB8, 0x00, 0x38, 0x40, 0x44], np.uint8)
    A = E[rng.integers(0, 7, (50, 64))]
    B = E[rng.integers(0, 7, (3001, 64))]
    rv, rl = orc.topk_e4m3(A, B, 20, 0)
    sa, sb = _scales(A.shape[0], B.shape[0])
    qv, ql = orc.topk_e4m3(A, B, 20, 2, sa, sb)
    for rank, t, gv, gl, sv, sl in res:
        assert t == [2.0, 5.0]
        assert np.array_equal(gv, rv) and np.array_equal(gl, rl)
        assert np.array_equal(sv, qv) and np.array_equal(sl, ql)


def test_shard_bounds_cover_every_column():
    from rotormap import dist as rdist
    for N, G in ((10, 3), (16777216, 8), (5, 8)):
        b = [rdist.shard_bounds(N, G, r) for r in range(G)]
        assert b[0][0] == 0 and b[-1][1] == N
        assert all(b[i][1] == b[i + 1][0] for i in range(G - 1))
