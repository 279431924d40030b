"""Precision form: per-row-scaled fp8 bulk search, FP32 exact rescoring of
the candidates (re-encoding their reference windows on the fly), and the FP64
sampled-row check that states score error and top-k recall.

The index meta the rescoring needs (packed genome, per-column genome position
and strand) is uploaded once per index (`DeviceMeta`).
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import check, lib, ptr, stream_handle
from .encoder import RopeEncoder, encode_frag_real_batch


class DeviceMeta:
    """Packed genome + column positions / strands of an index, on the device."""

    def __init__(self, idx, device=None, genome: torch.Tensor | None = None):
        dev = device or (idx.embeds8.device if isinstance(idx.embeds8, torch.Tensor) else "cuda")
        if genome is None and idx.genome is None:
            from .index import attach_genome
            attach_genome(idx)  # an index read from a reference .bin: pack its source FASTA
        if genome is None:
            genome = torch.from_numpy(np.ascontiguousarray(idx.genome).view(np.int32)).to(dev)
        self.genome = genome
        self.col_pos = torch.from_numpy(np.ascontiguousarray(idx.col_pos, dtype=np.int64)).to(dev)
        self.strand = torch.from_numpy(np.ascontiguousarray(idx.strand, dtype=np.uint8)).to(dev)
        self.N = int(idx.N)


def rescore_fp32(re: RopeEncoder, meta: DeviceMeta, words: torch.Tensor, cand: torch.Tensor, topk: int = 20,
                 normalize: int = 0, want_scores: bool = False, stream=None):
    """r2m_rescore_fp32: words (nb, W) int32 device, cand (nb, kc) 1-based ids
    -> (vals (nb, topk), locs (nb, topk)[, scores (nb, kc)])."""
    nb, kc = cand.shape
    dev = cand.device
    vals = torch.empty((nb, topk), dtype=torch.float32, device=dev)
    locs = torch.empty((nb, topk), dtype=torch.int32, device=dev)
    scores = torch.empty((nb, kc), dtype=torch.float32, device=dev) if want_scores else None
    check(lib().r2m_rescore_fp32(ptr(words), nb, ptr(cand), kc, ptr(meta.genome), ptr(meta.col_pos),
                                 ptr(meta.strand), meta.N, re.k, re.s, re.m, re.c, normalize, ptr(scores),
                                 ptr(vals), ptr(locs), topk, stream_handle(stream)))
    return (vals, locs, scores) if want_scores else (vals, locs)


def check_fp64(re: RopeEncoder, meta: DeviceMeta, words: torch.Tensor, cand: torch.Tensor | None = None,
               stream=None):
    """r2m_check_fp64 on S sampled reads -> (vals64 (S, 20), locs (S, 20)[, cand
    scores64 (S, kc)]).  Synchronizes."""
    S = words.shape[0]
    dev = words.device
    vals = torch.empty((S, 20), dtype=torch.float64, device=dev)
    locs = torch.empty((S, 20), dtype=torch.int32, device=dev)
    cs = None
    kc = 0
    if cand is not None:
        kc = cand.shape[1]
        cs = torch.empty((S, kc), dtype=torch.float64, device=dev)
    check(lib().r2m_check_fp64(ptr(words), S, ptr(meta.genome), ptr(meta.col_pos), ptr(meta.strand), meta.N,
                               re.k, re.s, re.m, re.c, ptr(cand), kc, ptr(cs), ptr(vals), ptr(locs),
                               stream_handle(stream)))
    return (vals, locs, cs) if cand is not None else (vals, locs)


def map_precise(eng, re: RopeEncoder, meta: DeviceMeta, words: torch.Tensor, topk: int = 20,
                normalize: int = 0, stream=None):
    """The precision flow on device-resident read words: per-row-scaled fp8
    top-kc (kc = engine k) -> FP32 rescoring -> top-k.  Returns
    (fp8 vals, fp8 locs, fp32 vals, fp32 locs)."""
    nb = words.shape[0]
    dev = words.device
    a8 = eng.a8[:nb]
    sa = eng.scaleA[:nb]
    norms = torch.empty((nb, re.m), dtype=torch.float32, device=dev)
    encode_frag_real_batch(a8, norms, re, words.reshape(-1), normalize, sa, stream)
    v8, l8 = eng.search(a8, nb, sa, stream=stream)
    v32, l32 = rescore_fp32(re, meta, words, l8, topk, normalize, stream=stream)
    return v8, l8, v32, l32
