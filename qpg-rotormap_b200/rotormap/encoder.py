"""Rope encoder host API (mirror of RotorMap/encode/: ropeencoder.jl, kernel.jl).

All device work runs in librotormap_b200.so; tensors are torch CUDA tensors
used as plain device buffers.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _lib
from ._lib import check, lib, ptr, stream_handle


@dataclass(frozen=True)
class RopeEncoder:
    """RopeEncoder(k, s, m, c) (RotorMap/encode/ropeencoder.jl:16-30).

    k: phase denominator and fragment length; s: s-mer length; m: copies
    (multiplicity); c: compact c-mer length (bins = m * 4^c).
    """
    k: int
    s: int = 5
    m: int = 1
    c: int = 0

    def dim(self) -> int:
        """Complex bins (ropeencoder.jl:30); the real row is 2 * dim."""
        return self.m * 4 ** self.c if self.c else self.m * 4 ** self.s

    @property
    def rdim(self) -> int:
        return 2 * self.dim()

    @property
    def words(self) -> int:
        return (self.k + 15) // 16


def dim(re: RopeEncoder) -> int:
    return re.dim()


_KIND = {torch.float32: _lib.OUT_F32, torch.float16: _lib.OUT_F16}


def out_kind_of(dest: torch.Tensor, scaled: bool) -> int:
    if dest.dtype == torch.uint8:
        return _lib.OUT_E4M3_SCALED if scaled else _lib.OUT_E4M3
    if dest.dtype in _KIND:
        return _KIND[dest.dtype]
    raise TypeError(f"unsupported encoder output dtype {dest.dtype}")


def encode_frag_real_batch(dest: torch.Tensor, dest_norms: torch.Tensor, re: RopeEncoder,
                           dnas: torch.Tensor, normalize: int = 0,
                           dest_scales: torch.Tensor | None = None, stream=None):
    """encode_frag_real_batch! (RotorMap/encode/kernel.jl:298-325).

    dest: (n, 2*m*4^c) float32 / float16 / uint8 (e4m3) CUDA tensor -- uint8
    without `dest_scales` is the reference quantisation e4m3(fp32(fp16(x)));
    with `dest_scales` (n,) float32 it is the per-row scaled e4m3 form.
    dest_norms: (n, m) float32.  dnas: flat or (n, W) uint32/int32 words.
    """
    if re.c < 1:
        raise ValueError("the fragment kernel needs c >= 1 (compact bins)")
    n = dest.shape[0]
    if dest.shape != (n, re.rdim):
        raise ValueError(f"dest must be (n, {re.rdim}) -- the [Re; Im] concatenation")
    if tuple(dest_norms.shape) != (n, re.m) or dest_norms.dtype != torch.float32:
        raise ValueError(f"dest_norms must be float32 (n, {re.m})")
    if dnas.numel() != n * re.words:
        raise ValueError("dnas must hold n * cld(k, 16) words")
    for t in (dest, dest_norms, dnas):
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("encoder buffers must be contiguous CUDA tensors")
    kind = out_kind_of(dest, dest_scales is not None)
    check(lib().r2m_encode_frag_real_batch(ptr(dest), kind, ptr(dest_norms), ptr(dest_scales),
                                           ptr(dnas), n, re.k, re.s, re.m, re.c, normalize,
                                           stream_handle(stream)))
    return dest, dest_norms


def encode_frag_real_batch_alloc(dtype, re: RopeEncoder, dnas: torch.Tensor, normalize: int = 0,
                                 scaled: bool = False, stream=None):
    """Allocating variant (kernel.jl:328-335): returns (embeds, norms[, scales])."""
    n = dnas.numel() // re.words
    dev = dnas.device
    dest = torch.empty((n, re.rdim), dtype=dtype, device=dev)
    norms = torch.empty((n, re.m), dtype=torch.float32, device=dev)
    scales = torch.empty((n,), dtype=torch.float32, device=dev) if scaled else None
    encode_frag_real_batch(dest, norms, re, dnas, normalize, scales, stream)
    return (dest, norms, scales) if scaled else (dest, norms)


def revcomp_frag_words(drc: torch.Tensor, dnas: torch.Tensor, k: int, n: int, stream=None):
    """revcomp_frag_words! (RotorMap/index/build.jl:464-476)."""
    W = (k + 15) // 16
    if dnas.numel() != n * W or drc.numel() != n * W:
        raise ValueError("drc and dnas must hold n * cld(k, 16) words")
    check(lib().r2m_revcomp_frag_words(ptr(drc), ptr(dnas), k, n, stream_handle(stream)))
    return drc


def f32_to_f8(dst: torch.Tensor, src: torch.Tensor, stream=None):
    """f32_to_f8! (RotorMap/gemm/fp8_convert.jl:100): e4m3 RNE satfinite."""
    if dst.numel() != src.numel() or src.dtype != torch.float32 or dst.dtype != torch.uint8:
        raise ValueError("f32_to_f8 needs float32 src and uint8 dst of equal size")
    check(lib().r2m_f32_to_e4m3(ptr(dst), ptr(src), src.numel(), stream_handle(stream)))
    return dst


def f16_to_f8(dst: torch.Tensor, src: torch.Tensor, stream=None):
    """The fp16 -> fp32 -> e4m3 step of upload_fp16_as_f8! (engine_fp8.jl:355-371)."""
    if dst.numel() != src.numel() or src.dtype != torch.float16 or dst.dtype != torch.uint8:
        raise ValueError("f16_to_f8 needs float16 src and uint8 dst of equal size")
    check(lib().r2m_f16_to_e4m3(ptr(dst), ptr(src), src.numel(), stream_handle(stream)))
    return dst
