"""Batching form: ragged request sets in one persistent launch, graph replay
and the autotuner.  A read's top-k must not depend on which ragged set (or
graph replay) it was mapped in."""
import numpy as np
import pytest
import torch

import rotormap as rm
from rotormap import synth

pytestmark = pytest.mark.gpu

K = 100


@pytest.fixture(scope="module")
def setup():
    heads = [">b1", ">b2", ">b3"]
    recs = synth.random_genome([200_000, 150_000, 50_000], seed=8, gc=0.41)
    re = rm.RopeEncoder(k=K, s=8, m=4, c=4)
    idx = rm.build_index(re, synth.genome_fasta(heads, recs), kstep=10)
    rng = np.random.default_rng(9)
    sizes = np.exp(rng.uniform(0, np.log(3000), 40)).astype(int)
    reqs = []
    for i, n in enumerate(sizes):
        reads, _, _, _ = synth.sample_reads_even(heads, recs, int(n), K, float(rng.uniform(0, 0.15)), seed=200 + i)
        reqs.append(synth.pack_reads(reads, K))
    return re, idx, reqs


def _per_request(eng, re, reqs):
    out = []
    for w in reqs:
        d = torch.from_numpy(w.reshape(-1).view(np.int32)).cuda()
        a8, nrm = rm.encode_frag_real_batch_alloc(torch.uint8, re, d)
        v, l = eng.search(a8)
        out.append((v.cpu().numpy(), l.cpu().numpy()))
    return out


def test_ragged_launch_and_graph_replay_match_per_request(setup):
    re, idx, reqs = setup
    total = sum(w.shape[0] for w in reqs)
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=rm.bucket_rows(total))
    ref = _per_request(eng, re, reqs)
    b = rm.RaggedBatcher(eng, re, total, use_graphs=True)
    got = b.run(reqs)
    for (v, l), (rv, rl) in zip(got, ref):
        assert np.array_equal(v, rv) and np.array_equal(l, rl)
    # replay the same bucket with another ragged split of other data
    perm = [reqs[i] for i in np.random.default_rng(1).permutation(len(reqs))]
    got2 = b.run(perm)
    ref2 = _per_request(eng, re, perm)
    assert len(b.graphs) == 1
    for (v, l), (rv, rl) in zip(got2, ref2):
        assert np.array_equal(v, rv) and np.array_equal(l, rl)
    eng.close()


def test_autotuner_keeps_results(setup, tmp_path):
    re, idx, reqs = setup
    sub = reqs[:12]
    total = sum(w.shape[0] for w in sub)
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=rm.bucket_rows(total))
    tuner = rm.Autotuner(str(tmp_path / "tune.json"))
    b = rm.RaggedBatcher(eng, re, total, tuner=tuner, use_graphs=True)
    got = b.run(sub)
    assert len(tuner.log) >= 3 and (tmp_path / "tune.json").exists()
    eng.set_tuning(0, 0)
    ref = _per_request(eng, re, sub)
    for (v, l), (rv, rl) in zip(got, ref):
        assert np.array_equal(v, rv) and np.array_equal(l, rl)
    eng.close()
