"""Column-sharded search (one index shard per rank) merged with the
library's list-merge kernel: equal to the single-engine result, bit for bit.
The all-gather of a multi-GPU run is emulated on one GPU by laying the
shards' lists side by side (the layout torch.distributed.all_gather + cat
produces)."""
import numpy as np
import pytest
import torch

import rotormap as rm
from rotormap import dist as rdist

from test_gpu_search import int_e4m3

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("G,k", [(1, 20), (2, 20), (3, 8), (8, 32), (32, 5)])
def test_merge_kernel_matches_torch_merge(G, k):
    rng = np.random.default_rng(G * 100 + k)
    nb = 777
    vals = np.round(rng.standard_normal((nb, G, k)) * 4) / 4  # many equal values
    vals = -np.sort(-vals, axis=2).astype(np.float32)
    locs = rng.permutation(nb * G * k * 3)[: nb * G * k].reshape(nb, G, k).astype(np.int32) + 1
    # sort each list by (value desc, column asc) and blank some tails
    for r in range(nb):
        for g in range(G):
            o = np.lexsort((locs[r, g], -vals[r, g]))
            vals[r, g], locs[r, g] = vals[r, g][o], locs[r, g][o]
            e = int(rng.integers(0, 3))
            if e:
                vals[r, g, k - e:], locs[r, g, k - e:] = -np.inf, 0
    v = torch.from_numpy(vals.reshape(nb, G * k)).cuda()
    l = torch.from_numpy(locs.reshape(nb, G * k)).cuda()
    a = rdist.merge_topk_lists(v, l, G, k)
    b = rdist.merge_topk(v.cpu(), l.cpu(), k)
    assert torch.equal(a[0].cpu(), b[0]) and torch.equal(a[1].cpu(), b[1].to(torch.int32))


@pytest.mark.parametrize("G", [2, 3, 5])
@pytest.mark.parametrize("score", ["f16", "scaled"])
def test_column_sharded_search_equals_single_engine(G, score):
    rng = np.random.default_rng(G)
    nb, N, rdim, k = 300, 40_001, 256, 20
    A8, _ = int_e4m3(rng, (nb, rdim), -1, 1)
    B8, _ = int_e4m3(rng, (N, rdim), -1, 1)
    sa = torch.from_numpy(rng.uniform(0.5, 2.0, nb).astype(np.float32)).cuda() if score == "scaled" else None
    sb = torch.from_numpy(rng.uniform(0.5, 2.0, N).astype(np.float32)).cuda() if score == "scaled" else None
    A = torch.from_numpy(A8).cuda()
    B = torch.from_numpy(B8).cuda()
    full = rm.TopKEngine(B, k=k, rows_cap=nb, score=score, scaleB=sb)
    v0, l0 = full.search(A, nb, sa)
    unit = torch.ones(nb, dtype=torch.float32, device="cuda") if sa is not None else None
    vs, ls = [], []
    for r in range(G):
        lo, hi = rdist.shard_bounds(N, G, r)
        # each rank owns a copy of its shard (and of its column scales)
        Bs = B[lo:hi].clone()
        sbs = sb[lo:hi].clone() if sb is not None else None
        eng = rm.TopKEngine(Bs, k=k, rows_cap=nb, score=score, scaleB=sbs)
        v, l = eng.search(A, nb, unit)
        vs.append(v)
        ls.append(torch.where(l > 0, l + lo, l))
        eng.close()
    mv, ml = rdist.merge_topk_lists(torch.cat(vs, 1), torch.cat(ls, 1), G, k)
    if sa is not None:
        mv = rdist.scale_rows(mv, sa)
    assert torch.equal(mv, v0) and torch.equal(ml, l0)
    full.close()
