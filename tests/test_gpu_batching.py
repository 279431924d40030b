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
    # a generous budget: candidates run on the real engine, every knob is tried
    tuner = rm.Autotuner(str(tmp_path / "tune.json"), budget=1e3)
    b = rm.RaggedBatcher(eng, re, total, tuner=tuner, use_graphs=True)
    got = b.run(sub)
    assert len(tuner.log) >= 6 and (tmp_path / "tune.json").exists()
    assert all(e["cols"] == idx.N for e in tuner.log)
    assert {"kernel", "epilogue", "pace", "kt"} <= set(tuner.log[0])
    eng.set_tuning(0, 0, kernel="auto", epilogue="auto", pace=0, kt=0)
    ref = _per_request(eng, re, sub)
    for (v, l), (rv, rl) in zip(got, ref):
        assert np.array_equal(v, rv) and np.array_equal(l, rl)
    # a second tuner reads the persisted choice instead of timing again
    t2 = rm.Autotuner(str(tmp_path / "tune.json"), budget=1e3)
    b2 = rm.RaggedBatcher(eng, re, total, tuner=t2, use_graphs=True)
    got2 = b2.run(sub)
    assert t2.log == [] and t2.last.get("cached")
    for (v, l), (rv, rl) in zip(got2, ref):
        assert np.array_equal(v, rv) and np.array_equal(l, rl)
    eng.close()


@pytest.mark.parametrize("cfg", [dict(kernel="1sm"), dict(kernel="2sm"), dict(epilogue="4"), dict(epilogue="8"),
                                 dict(pace=32), dict(pace=-1), dict(kt=32), dict(kt=64), dict(splits=3),
                                 dict(ctas=100)])
def test_every_schedule_gives_identical_results(setup, cfg):
    """The autotuner may pick any of these: none may change a result."""
    re, idx, reqs = setup
    w = np.concatenate(reqs[:6])
    d = torch.from_numpy(w.reshape(-1).view(np.int32)).cuda()
    a8, _ = rm.encode_frag_real_batch_alloc(torch.uint8, re, d)
    eng = rm.TopKEngine(idx.embeds8, k=20, rows_cap=a8.shape[0])
    v0, l0 = (t.cpu().numpy() for t in eng.search(a8))
    eng.set_tuning(cfg.get("splits", 0), cfg.get("ctas", 0), kernel=cfg.get("kernel"),
                   epilogue=cfg.get("epilogue"), pace=cfg.get("pace"), kt=cfg.get("kt"))
    v1, l1 = (t.cpu().numpy() for t in eng.search(a8))
    assert np.array_equal(v0, v1) and np.array_equal(l0, l1)
    eng.close()
