// encode.cu -- the fused rope encoder (reads and index windows), the
// reverse-complement word kernel and the e4m3 quantisers.
//
// Encoder semantics follow the reference kernel kernel_rope_frag_real
// (RotorMap/encode/kernel.jl:86-290) and its fp64 twin _ref_rope_frag
// (RotorMap/encode/reference.jl:37-93):
//   * window p (0-based, p < nw = k-s+1) reads the little-endian 2s-bit field
//     of bases [p, p+s): smer = (stream >> 2p) & (4^s-1);
//   * lower = smer & (4^c-1), upper = smer >> 2c,
//     csmer = lower ^ ((upper * 0x9E3779B1) & (4^c-1));
//   * bin = csmer*m + idm gets the phasor exp(+i*theta_idm*p) with
//     theta_idm = f32(factor) * f32(2*pi/k), factor = 1 (m = 1) else
//     2*idm/(m-1)+1 (idm 0-based);
//   * the bins of csmer 2*sum_{i<c} 4^i ("GG..G") are zeroed;
//   * normalize modes 0..3 as the reference; the real row is the split
//     [Re(bin 0..D-1); Im(bin 0..D-1)], D = m*4^c.
//
// B200 design: one warp per fragment (the reference spends one 512-thread
// block per 150-base read with 143 active threads).  The phasor of every
// (idm, p) is computed once per block into shared memory with the exact fp32
// recipe of the reference thread that owns window p (direct cos/sin at the
// thread's first window, then the fp32 complex recurrence), so the values
// are the reference's.  Histogram sums are deterministic: windows are added
// to their bins in increasing p (warp match_any groups equal bins inside a
// 32-window batch; the group's leader adds them in lane order).  The output
// conversion (fp32 / fp16 / e4m3 / scaled e4m3) is fused into the final pass.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "common.cuh"

namespace r2m {

struct EncParams {
  int k, s, m, c, normalize;
  int W;      // words per fragment = cld(k,16)
  int nw;     // windows = k-s+1
  int nbin;   // complex bins D = m*4^c
  int rdim;   // 2*nbin
  int Wc;     // the reference thread chunk: cld(nw,512), made odd
  uint32_t bmask, cbmask, csmerG;
  float theta[8];  // per idm, fp32
  int table_in_smem;
  int hist_floats;  // per-warp histogram floats (2*nbin, rounded to whole 16-bin chunks)
  int cs_u16;       // per-warp csmer slots (nw rounded up to 8)
  int words_u32;    // per-warp staged words (W + 2, rounded up to 4)
  int sp_nslot;     // sparse path: most distinct c-mers a fragment can have, min(nw, 4^c)
};

static int make_params(EncParams &P, int k, int s, int m, int c, int normalize) {
  R2M_REQUIRE(s >= 1 && s <= 16, "s must be in 1..16 (the s-mer lives in a 32-bit funnel window)");
  R2M_REQUIRE(c >= 1 && c <= s, "c must be in 1..s");
  R2M_REQUIRE(m >= 1 && m <= 8, "m must be in 1..8");
  R2M_REQUIRE(k >= s, "k must be >= s (no s-mer windows otherwise)");
  R2M_REQUIRE(k <= (1 << 22), "k too large");
  R2M_REQUIRE(normalize >= 0 && normalize <= 3, "normalize must be 0..3");
  R2M_REQUIRE((long long)m << (2 * c) <= 16384, "m*4^c too large for the shared-memory histogram");
  P.k = k; P.s = s; P.m = m; P.c = c; P.normalize = normalize;
  P.W = (k + 15) / 16;
  P.nw = k - s + 1;
  P.nbin = m << (2 * c);
  P.rdim = 2 * P.nbin;
  int wc = (P.nw + 511) / 512;
  if ((wc & 1) == 0) wc += 1;
  P.Wc = wc;
  P.bmask = (s == 16) ? 0xFFFFFFFFu : ((1u << (2 * s)) - 1u);
  P.cbmask = (c == 16) ? 0xFFFFFFFFu : ((1u << (2 * c)) - 1u);
  uint32_t allones = 0;
  for (int i = 0; i < c; ++i) allones += 1u << (2 * i);
  P.csmerG = 2u * allones;  // 0-based index of the reference's 2*allones+1
  float base = (float)(2.0 * M_PI / (double)k);
  for (int i = 0; i < 8; ++i) {
    float f = (m == 1) ? 1.0f : (float)(2.0 * (double)i / (double)(m - 1) + 1.0);
    P.theta[i] = f * base;
  }
  P.hist_floats = (P.rdim + 31) & ~31;
  P.cs_u16 = (P.nw + 7) & ~7;
  P.words_u32 = (P.W + 2 + 3) & ~3;
  {
    const long long ncm = 1LL << (2 * c);
    P.sp_nslot = (int)(ncm < P.nw ? ncm : P.nw);
  }
  return R2M_OK;
}

// Exact reference phasor of window p for copy idm (see file header).
__device__ __forceinline__ float2 ref_phasor(const EncParams &P, int idm, int p) {
  float th = P.theta[idm];
  int p0 = (p / P.Wc) * P.Wc;
  float a = th * (float)p0;
  float re = cosf(a), im = sinf(a);
  if (p != p0) {
    float xr = cosf(th), xi = sinf(th);
    for (int q = p0; q < p; ++q) {
      float nr = __fsub_rn(__fmul_rn(re, xr), __fmul_rn(im, xi));
      float ni = __fadd_rn(__fmul_rn(re, xi), __fmul_rn(im, xr));
      re = nr;
      im = ni;
    }
  }
  return make_float2(re, im);
}

// Global table (used when the per-block shared copy does not fit):
// one thread per (idm, reference chunk) walks the chunk's recurrence.
__global__ void k_phasor_table(EncParams P, float2 *table) {
  int nchunk = (P.nw + P.Wc - 1) / P.Wc;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nchunk * P.m) return;
  int idm = t / nchunk, ch = t % nchunk;
  int p0 = ch * P.Wc, p1 = min(p0 + P.Wc, P.nw);
  float th = P.theta[idm];
  float a = th * (float)p0;
  float re = cosf(a), im = sinf(a);
  float xr = cosf(th), xi = sinf(th);
  for (int p = p0; p < p1; ++p) {
    table[(size_t)idm * P.nw + p] = make_float2(re, im);
    float nr = __fsub_rn(__fmul_rn(re, xr), __fmul_rn(im, xi));
    float ni = __fadd_rn(__fmul_rn(re, xi), __fmul_rn(im, xr));
    re = nr;
    im = ni;
  }
}

template <int OUT>
struct OutT;
template <>
struct OutT<R2M_OUT_F32> { static constexpr int bytes = 4; };
template <>
struct OutT<R2M_OUT_F16> { static constexpr int bytes = 2; };
template <>
struct OutT<R2M_OUT_E4M3> { static constexpr int bytes = 1; };
template <>
struct OutT<R2M_OUT_E4M3_SCALED> { static constexpr int bytes = 1; };

template <int OUT>
__device__ __forceinline__ void store16(void *row, int i0, const float (&v)[16]) {
  if constexpr (OUT == R2M_OUT_F32) {
    float4 *d = reinterpret_cast<float4 *>(reinterpret_cast<float *>(row) + i0);
#pragma unroll
    for (int q = 0; q < 4; ++q) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  } else if constexpr (OUT == R2M_OUT_F16) {
    uint32_t h[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      __half2 t = __floats2half2_rn(v[2 * q], v[2 * q + 1]);
      h[q] = *reinterpret_cast<uint32_t *>(&t);
    }
    uint4 *d = reinterpret_cast<uint4 *>(reinterpret_cast<__half *>(row) + i0);
    d[0] = make_uint4(h[0], h[1], h[2], h[3]);
    d[1] = make_uint4(h[4], h[5], h[6], h[7]);
  } else {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t lo = f32x2_to_e4m3x2(v[4 * q], v[4 * q + 1]);
      uint32_t hi = f32x2_to_e4m3x2(v[4 * q + 2], v[4 * q + 3]);
      w[q] = lo | (hi << 16);
    }
    *reinterpret_cast<uint4 *>(reinterpret_cast<uint8_t *>(row) + i0) =
        make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// 16 values -> e4m3(fp16(x)) (the reference's fp16 stream quantised by
// f32_to_f8 of the widened value) with one cvt per pair, 16-byte store.
__device__ __forceinline__ void store16_f16e4m3(void *row, int i0, const float (&v)[16]) {
  uint32_t w[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    __half2 h01 = __floats2half2_rn(v[4 * q], v[4 * q + 1]);
    __half2 h23 = __floats2half2_rn(v[4 * q + 2], v[4 * q + 3]);
    uint16_t lo, hi;
    asm("cvt.rn.satfinite.e4m3x2.f16x2 %0, %1;" : "=h"(lo) : "r"(*reinterpret_cast<uint32_t *>(&h01)));
    asm("cvt.rn.satfinite.e4m3x2.f16x2 %0, %1;" : "=h"(hi) : "r"(*reinterpret_cast<uint32_t *>(&h23)));
    w[q] = (uint32_t)lo | ((uint32_t)hi << 16);
  }
  *reinterpret_cast<uint4 *>(reinterpret_cast<uint8_t *>(row) + i0) = make_uint4(w[0], w[1], w[2], w[3]);
}

template <int OUT>
__device__ __forceinline__ void store1(void *row, int i, float v) {
  if constexpr (OUT == R2M_OUT_F32) {
    reinterpret_cast<float *>(row)[i] = v;
  } else if constexpr (OUT == R2M_OUT_F16) {
    reinterpret_cast<__half *>(row)[i] = __float2half_rn(v);
  } else {
    reinterpret_cast<uint8_t *>(row)[i] = f32_to_e4m3(v);
  }
}

// Shared-memory histogram layout.  Complex bin cb (Re, Im adjacent) lives in
// chunk j = cb / 16 (32 floats = 8 float4 slots), complex slot w = cb % 16,
// float4 slot w / 2 -- stored at slot (w / 2) ^ (j % 8).  The output passes
// give each lane one chunk and walk its 8 slots in order; without the XOR
// every lane of a step would hit the same four banks (chunks are 128 bytes
// apart), with it the 32 lanes of a step cover all 32 banks.
__device__ __forceinline__ int hoff(int cb) {
  const int j = cb >> 4, w = cb & 15;
  return ((((j << 3) | ((w >> 1) ^ (j & 7))) << 2) | ((w & 1) << 1));
}

// Value of output element i (split layout) before the storage conversion.
// E4M3 parity mode rounds through fp16 first, like the reference's fp16
// stream followed by f32_to_f8 of the widened value.
template <int OUT>
__device__ __forceinline__ float out_value(const EncParams &P, const float *hist,
                                           const float *nrmv, int i, float scale) {
  int bin = (i < P.nbin) ? i : i - P.nbin;
  int part = (i < P.nbin) ? 0 : 1;
  float nrm = nrmv[P.normalize == 0 ? 0 : (bin % P.m)];
  float x = hist[hoff(bin) + part] / nrm;
  if constexpr (OUT == R2M_OUT_E4M3) x = __half2float(__float2half_rn(x));
  if constexpr (OUT == R2M_OUT_E4M3_SCALED) x = x * scale;
  return x;
}

// Histogram of the fragment whose words are staged in `words` (W words + a
// zero guard word), built by one warp: phasor sums per bin in window order,
// G-homopolymer bins zeroed, modes 2/3 reshaped; `nrmv` receives the divisor
// of every copy (index 0 for mode 0) and `norms_out` the reference's norms
// row.  The normalised value of split element i is hist[...]/nrmv[...].
__device__ __forceinline__ void fragment_hist(const EncParams &P, const float2 *table, float *hist, uint16_t *cs,
                              const uint32_t *words, float *nrmv, float *norms_out, float *amax_raw = nullptr) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  // zero the histogram
  for (int i = lane * 4; i < P.hist_floats; i += 128)
    *reinterpret_cast<float4 *>(hist + i) = make_float4(0.f, 0.f, 0.f, 0.f);
  // scrambled c-mer of every window
  for (int p = lane; p < P.nw; p += 32) {
    int wo = p >> 4;
    uint32_t sh = (uint32_t)(p & 15) << 1;
    uint32_t w0 = words[wo], w1 = words[wo + 1];
    uint32_t v = sh == 0 ? w0 : ((w0 >> sh) | (w1 << (32u - sh)));
    uint32_t smer = v & P.bmask;
    uint32_t lower = smer & P.cbmask;
    uint32_t upper = (2 * P.c >= 32) ? 0u : (smer >> (2 * P.c));
    uint32_t key = (upper * 0x9E3779B1u) & P.cbmask;
    cs[p] = (uint16_t)(lower ^ key);
  }
  __syncwarp();
  // accumulate phasors in increasing window order (deterministic)
  for (int b0 = 0; b0 < P.nw; b0 += 32) {
    int p = b0 + lane;
    bool act = p < P.nw;
    unsigned amask = __ballot_sync(FULL, act);
    if (act) {
      uint32_t cbin = cs[p];
      unsigned grp = __match_any_sync(amask, cbin);
      if (lane == __ffs(grp) - 1) {
        if (P.m == 4) {
          // the group's bins 4 cbin .. 4 cbin + 3 (float4 slots 2 (cbin % 4)
          // and the next one of chunk cbin / 4, swizzled): one read-modify-
          // write, the members' phasors added in window (lane) order
          float4 *hc = reinterpret_cast<float4 *>(hist + ((cbin >> 2) << 5));
          const int sw = (int)((cbin >> 2) & 7), s0 = (int)(2 * (cbin & 3));
          float4 *h0 = hc + (s0 ^ sw), *h1 = hc + ((s0 + 1) ^ sw);
          float4 h01 = *h0, h23 = *h1;
          unsigned g = grp;
          do {
            const int j = __ffs(g) - 1;
            g &= g - 1;
            const float2 p0 = table[b0 + j], p1 = table[(size_t)P.nw + b0 + j];
            const float2 p2 = table[2 * (size_t)P.nw + b0 + j], p3 = table[3 * (size_t)P.nw + b0 + j];
            h01.x += p0.x; h01.y += p0.y; h01.z += p1.x; h01.w += p1.y;
            h23.x += p2.x; h23.y += p2.y; h23.z += p3.x; h23.w += p3.y;
          } while (g);
          *h0 = h01;
          *h1 = h23;
        } else {
          for (int idm = 0; idm < P.m; ++idm) {
            float *h = hist + hoff((int)(cbin * P.m + idm));
            float re = h[0], im = h[1];
            const float2 *tb = table + (size_t)idm * P.nw + b0;
            unsigned g = grp;
            while (g) {
              int j = __ffs(g) - 1;
              g &= g - 1;
              float2 ph = tb[j];
              re += ph.x;
              im += ph.y;
            }
            h[0] = re;
            h[1] = im;
          }
        }
      }
    }
    __syncwarp();
  }
  // zero the G-homopolymer bins
  if (lane < P.m) {
    float *h = hist + hoff(P.csmerG * P.m + lane);
    h[0] = 0.f;
    h[1] = 0.f;
  }
  __syncwarp();
  // modes 2/3 reshape every bin first (fp64 arithmetic, fp32 storage)
  if (P.normalize >= 2) {
    for (int b = lane; b < P.nbin; b += 32) {
      float *h = hist + hoff(b);
      float re = h[0], im = h[1];
      double a = (double)hypotf(re, im);
      double d = (P.normalize == 2) ? (a + 2.220446049250313e-16) : sqrt(a + 2.220446049250313e-16);
      h[0] = (float)((double)re / d);
      h[1] = (float)((double)im / d);
    }
    __syncwarp();
  }
  // per-copy sums of squares
  float part[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) part[t] = 0.f;
  if (P.m <= 4 && (P.hist_floats & 127) == 0) {
    // walk the histogram linearly in float4 slots (the order of a sum of
    // squares is free): slot s of chunk j holds complex bins 2w', 2w' + 1 of
    // the chunk, w' = s ^ (j % 8), i.e. copies 2(w' & 1) and 2(w' & 1) + 1
    // for m = 4, copies 0 and 1 for m = 2, copy 0 for m = 1
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, mx = 0.f;
    const float4 *h4 = reinterpret_cast<const float4 *>(hist);
    const int nslot = P.hist_floats >> 2;
    for (int i = lane; i < nslot; i += 32) {
      const float4 t = h4[i];
      const float e0 = __fadd_rn(__fmul_rn(t.x, t.x), __fmul_rn(t.y, t.y));
      const float e1 = __fadd_rn(__fmul_rn(t.z, t.z), __fmul_rn(t.w, t.w));
      mx = fmaxf(mx, fmaxf(fmaxf(fabsf(t.x), fabsf(t.y)), fmaxf(fabsf(t.z), fabsf(t.w))));
      const bool hi = (((i & 7) ^ ((i >> 3) & 7)) & 1) != 0;  // w' odd: copies 2, 3
      if (hi) {
        a2 += e0;
        a3 += e1;
      } else {
        a0 += e0;
        a1 += e1;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(FULL, a0, o);
      a1 += __shfl_xor_sync(FULL, a1, o);
      a2 += __shfl_xor_sync(FULL, a2, o);
      a3 += __shfl_xor_sync(FULL, a3, o);
      mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
    }
    if (P.m == 4) {
      part[0] = a0, part[1] = a1, part[2] = a2, part[3] = a3;
    } else if (P.m == 2) {
      part[0] = a0 + a2, part[1] = a1 + a3;
    } else {
      part[0] = (a0 + a2) + (a1 + a3);
    }
    if (amax_raw) *amax_raw = mx;
  } else if ((32 % P.m) == 0) {
    // every bin of this lane (b = lane + 32j) belongs to copy lane % m: one
    // accumulator, then a butterfly over the lanes of the same copy (the
    // lanes of other copies would only add zeros, so the sums are the same)
    float acc = 0.f, mx = 0.f;
    for (int b = lane; b < P.nbin; b += 32) {
      float2 z = *reinterpret_cast<const float2 *>(hist + hoff(b));
      acc += __fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y));
      mx = fmaxf(mx, fmaxf(fabsf(z.x), fabsf(z.y)));
    }
    if (amax_raw) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
      *amax_raw = mx;
    }
    for (int o = 16; o >= P.m; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
#pragma unroll
    for (int q = 0; q < 8; ++q) part[q] = __shfl_sync(FULL, acc, q < P.m ? q : 0);
  } else {
    float mx = 0.f;
    for (int b = lane; b < P.nbin; b += 32) {
      const float *h = hist + hoff(b);
      float re = h[0], im = h[1];
      float e = __fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im));
      mx = fmaxf(mx, fmaxf(fabsf(re), fabsf(im)));
      int t = b % P.m;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q == t) part[q] += e;
    }
    if (amax_raw) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
      *amax_raw = mx;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part[q] += __shfl_xor_sync(FULL, part[q], o);
    }
  }
  if (lane == 0) {
    if (P.normalize == 0) {
      float acc = part[0];
      for (int q = 1; q < P.m; ++q) acc += part[q];
      float nrm = (float)((double)sqrtf(acc) + 1e-16);
      nrmv[0] = nrm;
      norms_out[0] = nrm;
      for (int q = 1; q < P.m; ++q) norms_out[q] = part[q];
    } else {
      for (int q = 0; q < P.m; ++q) {
        float nrm;
        if (P.normalize == 1) nrm = sqrtf(part[q]) + 1e-7f;
        else nrm = (float)((double)sqrtf(part[q]) + 2.220446049250313e-16);
        nrmv[q] = nrm;
        norms_out[q] = nrm;
      }
    }
  }
  __syncwarp();
}

// Encode the fragment whose words are staged in `words` (W words + a zero
// guard word) with one warp; write row `row` (rdim elements of OUT), the m
// norms and (scaled e4m3) the row scale.
template <int OUT>
__device__ void encode_fragment(const EncParams &P, const float2 *table, float *hist,
                                uint16_t *cs, const uint32_t *words, float *nrmv, void *row,
                                float *norms_out, float *scale_out) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  const bool fast = P.normalize == 0 && (P.nbin % 16) == 0 && P.nbin >= 16;
  float amax_raw = 0.f;
  fragment_hist(P, table, hist, cs, words, nrmv, norms_out, fast ? &amax_raw : nullptr);
  if (fast) {
    // one output pass: each lane takes chunks of 16 bins, divides every value
    // by the norm, scales, converts and stores the chunk's Re and Im runs
    const float nrm = nrmv[0];
    // x / nrm for every value with one reciprocal: y = RN(1/nrm), q0 = x*y,
    // r = x - q0*nrm (exact with FMA), q = RN(q0 + r*y) is the correctly
    // rounded quotient (Markstein's theorem) -- the same value as x / nrm
    const float y = __frcp_rn(nrm);
    auto divn = [&](float x) {
      float q0 = x * y;
      float r = fmaf(-q0, nrm, x);
      return fmaf(r, y, q0);
    };
    const int nchunk = P.nbin >> 4;
    float scale = 1.0f;
    if constexpr (OUT == R2M_OUT_E4M3_SCALED) {
      // a correctly rounded division is monotone and odd, so the largest
      // normalised magnitude is the largest raw magnitude divided once
      const float amax = divn(amax_raw);
      scale = amax > 0.f ? 448.0f / amax : 1.0f;
      if (lane == 0) *scale_out = amax > 0.f ? amax / 448.0f : 0.0f;
    }
    for (int j = lane; j < nchunk; j += 32) {
      const float4 *h4 = reinterpret_cast<const float4 *>(hist + 32 * j);
      const int sw = j & 7;
      float re[16], im[16];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        float4 t = h4[q ^ sw];
        re[2 * q] = divn(t.x);
        im[2 * q] = divn(t.y);
        re[2 * q + 1] = divn(t.z);
        im[2 * q + 1] = divn(t.w);
      }
      if constexpr (OUT == R2M_OUT_E4M3_SCALED) {
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          re[e] *= scale;
          im[e] *= scale;
        }
      }
      if constexpr (OUT == R2M_OUT_E4M3) {
        store16_f16e4m3(row, 16 * j, re);
        store16_f16e4m3(row, P.nbin + 16 * j, im);
      } else {
        store16<OUT>(row, 16 * j, re);
        store16<OUT>(row, P.nbin + 16 * j, im);
      }
    }
    __syncwarp();
    return;
  }
  // output pass (amax first for the scaled form)
  float scale = 1.0f;
  if constexpr (OUT == R2M_OUT_E4M3_SCALED) {
    float amax = 0.f;
    for (int i = lane; i < P.rdim; i += 32)
      amax = fmaxf(amax, fabsf(out_value<R2M_OUT_F32>(P, hist, nrmv, i, 1.0f)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(FULL, amax, o));
    scale = amax > 0.f ? 448.0f / amax : 1.0f;
    if (lane == 0) *scale_out = amax > 0.f ? amax / 448.0f : 0.0f;
  }
  const bool vec = (P.rdim % 16) == 0;
  if (vec) {
    for (int i0 = lane * 16; i0 < P.rdim; i0 += 512) {
      float v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = out_value<OUT>(P, hist, nrmv, i0 + j, scale);
      store16<OUT>(row, i0, v);
    }
  } else {
    for (int i = lane; i < P.rdim; i += 32) store1<OUT>(row, i, out_value<OUT>(P, hist, nrmv, i, scale));
  }
  __syncwarp();
}

// Per-warp shared-memory carve-up.
struct WarpSmem {
  float *hist;
  uint16_t *cs;
  uint32_t *words;
  uint32_t *words2;  // second word buffer (reverse complement)
  float *nrmv;
};

__device__ __forceinline__ size_t warp_smem_bytes(const EncParams &P) {
  return (size_t)P.hist_floats * 4 + (size_t)P.cs_u16 * 2 + (size_t)P.words_u32 * 4 * 2 + 32;
}

__device__ __forceinline__ WarpSmem carve(const EncParams &P, unsigned char *base, int warp) {
  size_t per = warp_smem_bytes(P);
  unsigned char *p = base + per * warp;
  WarpSmem w;
  w.hist = reinterpret_cast<float *>(p);
  p += (size_t)P.hist_floats * 4;
  w.words = reinterpret_cast<uint32_t *>(p);
  p += (size_t)P.words_u32 * 4;
  w.words2 = reinterpret_cast<uint32_t *>(p);
  p += (size_t)P.words_u32 * 4;
  w.nrmv = reinterpret_cast<float *>(p);
  p += 32;
  w.cs = reinterpret_cast<uint16_t *>(p);
  return w;
}

// Block prologue: the phasor table in shared memory (or the global copy).
__device__ __forceinline__ const float2 *block_table(const EncParams &P, unsigned char *smem,
                                                     const float2 *gtable) {
  if (!P.table_in_smem) return gtable;
  float2 *t = reinterpret_cast<float2 *>(smem);
  int total = P.m * P.nw;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int idm = i / P.nw, p = i % P.nw;
    t[i] = ref_phasor(P, idm, p);
  }
  __syncthreads();
  return t;
}

__device__ __forceinline__ size_t table_bytes(const EncParams &P) {
  return P.table_in_smem ? (((size_t)P.m * P.nw * 8 + 15) & ~(size_t)15) : 0;
}

template <int OUT>
__global__ void __launch_bounds__(256) k_encode_frags(EncParams P, const uint32_t *__restrict__ dnas,
                                                      int64_t n, void *dest, float *norms,
                                                      float *scales, const float2 *gtable) {
  extern __shared__ __align__(16) unsigned char smem[];
  const float2 *table = block_table(P, smem, gtable);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem ws = carve(P, smem + table_bytes(P), warp);
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const size_t rowbytes = (size_t)P.rdim * OutT<OUT>::bytes;
  for (int64_t f = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; f < n; f += nwarps) {
    const uint32_t *src = dnas + f * P.W;
    for (int i = lane; i < P.W; i += 32) ws.words[i] = __ldg(src + i);
    if (lane == 0) ws.words[P.W] = 0u;
    __syncwarp();
    encode_fragment<OUT>(P, table, ws.hist, ws.cs, ws.words, ws.nrmv,
                         reinterpret_cast<unsigned char *>(dest) + rowbytes * f,
                         norms + f * P.m, scales ? scales + f : nullptr);
  }
}

// Index windows: forward window from the packed genome, then its reverse
// complement, into the reference's per-batch [fwd block | rc block] columns.
template <int OUT>
__global__ void __launch_bounds__(256) k_encode_ref(EncParams P, const uint32_t *__restrict__ genome,
                                                    const int64_t *__restrict__ win_pos,
                                                    int64_t nwin, int64_t batch, void *dest,
                                                    float *norms, float *scales,
                                                    const float2 *gtable) {
  extern __shared__ __align__(16) unsigned char smem[];
  const float2 *table = block_table(P, smem, gtable);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem ws = carve(P, smem + table_bytes(P), warp);
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const size_t rowbytes = (size_t)P.rdim * OutT<OUT>::bytes;
  const int r = P.k & 15;
  const uint32_t tailmask = r == 0 ? 0xFFFFFFFFu : ((1u << (2 * r)) - 1u);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; i < nwin; i += nwarps) {
    const int64_t pos = __ldg(win_pos + i);
    const int64_t q = pos >> 4;
    const uint32_t sh = (uint32_t)(pos & 15) << 1;
    for (int j = lane; j < P.W; j += 32) {
      uint32_t a = __ldg(genome + q + j), b = __ldg(genome + q + j + 1);
      uint32_t v = sh == 0 ? a : ((a >> sh) | (b << (32u - sh)));
      if (j == P.W - 1) v &= tailmask;
      ws.words[j] = v;
    }
    if (lane == 0) ws.words[P.W] = 0u;
    __syncwarp();
    // reverse complement: rc base j = 3 - fwd base (k-1-j)
    for (int j = lane; j < P.W; j += 32) {
      uint32_t w = 0;
      for (int b = 0; b < 16; ++b) {
        int t = 16 * j + b;
        if (t < P.k) {
          int src = P.k - 1 - t;
          uint32_t code = (ws.words[src >> 4] >> (2 * (src & 15))) & 3u;
          w |= (3u - code) << (2 * b);
        }
      }
      ws.words2[j] = w;
    }
    if (lane == 0) ws.words2[P.W] = 0u;
    __syncwarp();
    const int64_t b = i / batch, off = i - b * batch;
    const int64_t nb = min(batch, nwin - b * batch);
    const int64_t colf = 2 * b * batch + off, colr = colf + nb;
    encode_fragment<OUT>(P, table, ws.hist, ws.cs, ws.words, ws.nrmv,
                         reinterpret_cast<unsigned char *>(dest) + rowbytes * colf,
                         norms + colf * P.m, scales ? scales + colf : nullptr);
    encode_fragment<OUT>(P, table, ws.hist, ws.cs, ws.words2, ws.nrmv,
                         reinterpret_cast<unsigned char *>(dest) + rowbytes * colr,
                         norms + colr * P.m, scales ? scales + colr : nullptr);
  }
}

__device__ __forceinline__ uint32_t lanerev32(uint32_t x) {
  x = ((x & 0x33333333u) << 2) | ((x >> 2) & 0x33333333u);
  x = ((x & 0x0F0F0F0Fu) << 4) | ((x >> 4) & 0x0F0F0F0Fu);
  x = ((x & 0x00FF00FFu) << 8) | ((x >> 8) & 0x00FF00FFu);
  return (x << 16) | (x >> 16);
}

// One thread per output word: complement, left-align the k bases to the end
// of the W-word stream, then reverse word order and the sixteen 2-bit lanes.
__global__ void k_revcomp(uint32_t *drc, const uint32_t *dnas, int W, int64_t n, uint32_t shbits) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)W * n) return;
  int64_t f = g / W;
  int p = (int)(g - f * W);
  int i = W - 1 - p;
  const uint32_t *src = dnas + f * W;
  uint32_t x = ~src[i];
  uint32_t v = x;
  if (shbits != 0) v = (x << shbits) | (i > 0 ? ((~src[i - 1]) >> (32u - shbits)) : 0u);
  drc[g] = lanerev32(v);
}

// ------------------------------------------------------------------
// Sparse fragment encoder (normalize = 0).
//
// At read length a fragment has few windows (143 at k = 150) against many
// bins (1024 complex bins at s8 m4 c4), so a dense per-warp histogram is
// mostly zeros that are cleared, summed and scanned again.  This path keeps
// one accumulator of m complex bins per DISTINCT c-mer of the fragment (a
// slot; slots are numbered in order of first appearance and a 4^c-byte map
// gives each c-mer's slot).  Windows are added in increasing window order:
// within a 32-window batch the members of a c-mer group add in rounds, by
// their rank in the group, so every bin is the same sum, formed in the same
// order, as the dense histogram's.  The norm and the row maximum are taken
// over the slots; each slot's values are divided, scaled and converted once;
// the output pass writes the dense row in 16-byte chunks, c-mer-major, with
// each c-mer's converted values taken from its slot, or zero.  The words of
// the fragment live in registers (lane t holds word t) and every window's
// 2s-bit field comes from two shuffles; the reverse complement of an index
// window is formed the same way.

template <int N>
struct Bytes;
template <>
struct Bytes<1> { using T = uint8_t; };
template <>
struct Bytes<2> { using T = uint16_t; };
template <>
struct Bytes<4> { using T = uint32_t; };
template <>
struct Bytes<8> { using T = uint2; };
template <>
struct Bytes<16> { using T = uint4; };

__device__ __forceinline__ unsigned long long f2_bits(float2 a) {
  return *reinterpret_cast<const unsigned long long *>(&a);
}
__device__ __forceinline__ float2 bits_f2(unsigned long long x) { return *reinterpret_cast<const float2 *>(&x); }
// Paired fp32 arithmetic (sm_100 f32x2): each half is the IEEE result of
// the scalar operation.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(d);
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return bits_f2(d);
}

// m values of one part (Re or Im) of a c-mer -> their m * bytes(OUT)
// output bytes, in the row's element order.
template <int OUT, int M>
__device__ __forceinline__ typename Bytes<M * OutT<OUT>::bytes>::T pack_part(const float (&v)[M]) {
  constexpr int CB = M * OutT<OUT>::bytes;
  union {
    typename Bytes<CB>::T t;
    uint32_t w[(CB + 3) / 4];
    uint16_t h[(CB + 1) / 2];
    uint8_t b[CB];
  } u;
  if constexpr (OUT == R2M_OUT_F32) {
#pragma unroll
    for (int q = 0; q < M; ++q) u.w[q] = __float_as_uint(v[q]);
  } else if constexpr (OUT == R2M_OUT_F16) {
    if constexpr (M == 1) {
      u.h[0] = __half_as_ushort(__float2half_rn(v[0]));
    } else {
#pragma unroll
      for (int q = 0; q < M / 2; ++q) {
        __half2 t = __floats2half2_rn(v[2 * q], v[2 * q + 1]);
        u.w[q] = *reinterpret_cast<uint32_t *>(&t);
      }
    }
  } else {
    // e4m3 pairs: low byte = first value
    uint16_t pr[(M + 1) / 2];
#pragma unroll
    for (int q = 0; q < (M + 1) / 2; ++q) {
      const float a = v[2 * q], b = (2 * q + 1 < M) ? v[2 * q + 1] : 0.0f;
      if constexpr (OUT == R2M_OUT_E4M3) {
        __half2 h = __floats2half2_rn(a, b);
        asm("cvt.rn.satfinite.e4m3x2.f16x2 %0, %1;" : "=h"(pr[q]) : "r"(*reinterpret_cast<uint32_t *>(&h)));
      } else {
        pr[q] = f32x2_to_e4m3x2(a, b);
      }
    }
    if constexpr (M == 1) {
      u.b[0] = (uint8_t)(pr[0] & 0xFF);
    } else {
#pragma unroll
      for (int q = 0; q < M / 2; ++q) u.h[q] = pr[q];
    }
  }
  return u.t;
}

// Per-warp shared memory of the sparse path (sizes in SparseLayout).
struct SparseLayout {
  int smap, acc, conv;  // byte sizes: slot map, accumulators, one conversion array
  int warp;             // total per warp
};

__host__ __device__ inline SparseLayout sparse_layout(int c, int m, int nslot, int outb) {
  SparseLayout L;
  const int ncm = 1 << (2 * c);
  L.smap = (ncm + 15) & ~15;
  L.acc = ((nslot * m * 8) + 15) & ~15;
  L.conv = ((nslot * m * outb) + 15) & ~15;
  // the two conversion arrays share their region with the per-c-mer group
  // masks of the accumulation (4 bytes per c-mer), which they follow
  const int masks = (4 * ncm + 15) & ~15;
  L.warp = L.smap + L.acc + (2 * L.conv > masks ? 2 * L.conv : masks);
  return L;
}

// The m complex values of one slot (or of one window's phasors) live in
// planes: plane j holds copies 2j and 2j+1 of every slot as one 16-byte
// entry (m = 1: one plane of 8-byte entries).  Lanes that touch consecutive
// slots then read consecutive 16 bytes, and random slots spread over the
// banks instead of falling on the same few (a slot-major 32-byte record
// puts every slot on one of 4 bank groups).
template <int M>
__device__ __forceinline__ void ld_planes(const float2 *base, int stride, int i, float2 (&v)[M]) {
  if constexpr (M == 1) {
    v[0] = base[i];
  } else {
    const float4 *b4 = reinterpret_cast<const float4 *>(base);
#pragma unroll
    for (int j = 0; j < M / 2; ++j) {
      const float4 t = b4[j * stride + i];
      v[2 * j] = make_float2(t.x, t.y);
      v[2 * j + 1] = make_float2(t.z, t.w);
    }
  }
}
template <int M>
__device__ __forceinline__ void st_planes(float2 *base, int stride, int i, const float2 (&v)[M]) {
  if constexpr (M == 1) {
    base[i] = v[0];
  } else {
    float4 *b4 = reinterpret_cast<float4 *>(base);
#pragma unroll
    for (int j = 0; j < M / 2; ++j)
      b4[j * stride + i] = make_float4(v[2 * j].x, v[2 * j].y, v[2 * j + 1].x, v[2 * j + 1].y);
  }
}

// Encode the fragment whose W words are in `wreg` (lane t: word t, zero for
// t >= W) with one warp into `row`, its m norms and (scaled) its row scale.
template <int OUT, int M>
__device__ __forceinline__ void sparse_fragment(const EncParams &P, const float2 *__restrict__ table,
                                                unsigned char *warea, uint32_t wreg, unsigned char *row,
                                                float *norms_out, float *scale_out) {
  constexpr int OUTB = OutT<OUT>::bytes, CB = M * OUTB, CPC = 16 / CB;
  using T = typename Bytes<CB>::T;
  using TM = typename Bytes<CPC>::T;
  const SparseLayout L = sparse_layout(P.c, M, P.sp_nslot, OUTB);
  const int ns = P.sp_nslot;  // entries per accumulator plane
  uint8_t *smap = warea;
  float2 *acc = reinterpret_cast<float2 *>(warea + L.smap);
  T *conv_re = reinterpret_cast<T *>(warea + L.smap + L.acc);
  T *conv_im = reinterpret_cast<T *>(warea + L.smap + L.acc + L.conv);
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  const unsigned lt = (1u << lane) - 1u;
  const int ncm = 1 << (2 * P.c);
  // group masks of the accumulation: bit l of gmask[cb] = lane l's window
  // has c-mer cb (formed with shared atomic ORs, cleared by each group's
  // leader after its batch, so zero between batches)
  uint32_t *gmask = reinterpret_cast<uint32_t *>(conv_re);
  for (int i = lane * 16; i < ncm; i += 512) *reinterpret_cast<uint4 *>(smap + i) = make_uint4(~0u, ~0u, ~0u, ~0u);
  for (int i = lane * 4; i < ncm; i += 128) *reinterpret_cast<uint4 *>(gmask + i) = make_uint4(0u, 0u, 0u, 0u);
  __syncwarp();
  // ---- accumulate, window order
  int nslots = 0;
  const int nw = P.nw;
  const uint32_t bmask = P.bmask, cbmask = P.cbmask, c2 = 2u * (uint32_t)P.c;
  for (int b0 = 0; b0 < nw; b0 += 32) {
    const int p = b0 + lane;
    const bool valid = p < nw;
    const int wo = p >> 4;
    const uint32_t w0 = __shfl_sync(FULL, wreg, wo & 31), w1 = __shfl_sync(FULL, wreg, (wo + 1) & 31);
    const uint32_t v = __funnelshift_r(w0, w1, (uint32_t)(p & 15) << 1);
    const uint32_t smer = v & bmask;
    const uint32_t upper = c2 >= 32u ? 0u : (smer >> c2);
    const uint32_t cb = (smer & cbmask) ^ ((upper * 0x9E3779B1u) & cbmask);
    // the lanes of this batch whose windows share a c-mer (a group), as a
    // lane mask: every lane ORs its bit into its c-mer's word
    if (valid) atomicOr(gmask + cb, 1u << lane);
    __syncwarp();
    const unsigned grp = valid ? gmask[cb] : (1u << lane);
    const int rank = __popc(grp & lt);
    const bool leader = valid && rank == 0;
    int s_l = 0xFF;
    if (leader) s_l = smap[cb];
    const bool isnew = leader && s_l == 0xFF;
    const unsigned newm = __ballot_sync(FULL, isnew);
    if (isnew) {
      s_l = nslots + __popc(newm & lt);
      smap[cb] = (uint8_t)s_l;
    }
    nslots += __popc(newm);
    const int slot = __shfl_sync(FULL, s_l, __ffs(grp) - 1);
    if (leader) gmask[cb] = 0u;  // read by all members above; the rounds below end with a warp sync
    float2 ph[M];
    if (valid) ld_planes<M>(table, nw, p, ph);
    // round 0: every group's first member (distinct slots: no conflict)
    if (leader) {
      float2 a[M];
      if (isnew) {
#pragma unroll
        for (int q = 0; q < M; ++q) a[q] = make_float2(0.f, 0.f);  // 0 + x, as a cleared bin
      } else {
        ld_planes<M>(acc, ns, slot, a);
      }
#pragma unroll
      for (int q = 0; q < M; ++q) a[q] = add2(a[q], ph[q]);
      st_planes<M>(acc, ns, slot, a);
    }
    __syncwarp();
    // later rounds: the r-th member of every group with more than r members
    const unsigned more = __ballot_sync(FULL, valid && rank > 0);
    if (more) {
      const int rounds = (int)__reduce_max_sync(FULL, valid ? (unsigned)rank : 0u);
      for (int r = 1; r <= rounds; ++r) {
        if (valid && rank == r) {
          float2 a[M];
          ld_planes<M>(acc, ns, slot, a);
#pragma unroll
          for (int q = 0; q < M; ++q) a[q] = add2(a[q], ph[q]);
          st_planes<M>(acc, ns, slot, a);
        }
        __syncwarp();
      }
    }
  }
  // ---- the G-homopolymer c-mer's bins are zero
  if (lane == 0) {
    const int sg = smap[P.csmerG];
    if (sg != 0xFF) {
      float2 z[M];
#pragma unroll
      for (int q = 0; q < M; ++q) z[q] = make_float2(0.f, 0.f);
      st_planes<M>(acc, ns, sg, z);
    }
  }
  __syncwarp();
  // ---- per-copy energies and the largest magnitude
  float part[M], mx = 0.f;
  float2 e2[M];  // per copy: sum of Re^2 and sum of Im^2, paired
#pragma unroll
  for (int q = 0; q < M; ++q) e2[q] = make_float2(0.f, 0.f);
  for (int sl = lane; sl < nslots; sl += 32) {
    float2 zv[M];
    ld_planes<M>(acc, ns, sl, zv);
#pragma unroll
    for (int q = 0; q < M; ++q) {
      const float2 z = zv[q];
      e2[q] = fma2(z, z, e2[q]);
      mx = fmaxf(mx, fmaxf(fabsf(z.x), fabsf(z.y)));
    }
  }
#pragma unroll
  for (int q = 0; q < M; ++q) part[q] = e2[q].x + e2[q].y;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < M; ++q) part[q] += __shfl_xor_sync(FULL, part[q], o);
    mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
  }
  float tot = part[0];
#pragma unroll
  for (int q = 1; q < M; ++q) tot += part[q];
  const float nrm = (float)((double)sqrtf(tot) + 1e-16);
#pragma unroll
  for (int q = 0; q < M; ++q)
    if (lane == q) norms_out[q] = q == 0 ? nrm : part[q];
  // x / nrm for every value with one reciprocal: y = RN(1/nrm), q0 = x*y,
  // r = x - q0*nrm (exact with FMA), RN(q0 + r*y) is the correctly rounded
  // quotient (Markstein) -- the reference's fp32 `hist ./= nrm`
  const float y = __frcp_rn(nrm);
  const float2 y2 = make_float2(y, y), nn2 = make_float2(-nrm, -nrm);
  float scale = 1.0f;
  if constexpr (OUT == R2M_OUT_E4M3_SCALED) {
    const float q0 = mx * y;
    const float amax = fmaf(fmaf(-q0, nrm, mx), y, q0);
    scale = amax > 0.f ? 448.0f / amax : 1.0f;
    if (lane == 0) *scale_out = amax > 0.f ? amax / 448.0f : 0.0f;
  }
  const float2 sc2 = make_float2(scale, scale);
  // ---- convert each slot once
  for (int sl = lane; sl < nslots; sl += 32) {
    float re[M], im[M];
    float2 xv[M];
    ld_planes<M>(acc, ns, sl, xv);
#pragma unroll
    for (int q = 0; q < M; ++q) {
      const float2 x = xv[q];
      const float2 q0 = mul2(x, y2);
      float2 d = fma2(fma2(q0, nn2, x), y2, q0);
      if constexpr (OUT == R2M_OUT_E4M3_SCALED) d = mul2(d, sc2);
      re[q] = d.x;
      im[q] = d.y;
    }
    conv_re[sl] = pack_part<OUT, M>(re);
    conv_im[sl] = pack_part<OUT, M>(im);
  }
  __syncwarp();
  // ---- the dense row, 16-byte chunks, c-mer-major: [Re part | Im part]
  const int nch = (ncm * CB) >> 4;  // chunks per part
  for (int j = lane; j < 2 * nch; j += 32) {
    const bool isim = j >= nch;
    const int jj = isim ? j - nch : j;
    union {
      TM t;
      uint8_t b[CPC];
    } sm;
    sm.t = *reinterpret_cast<const TM *>(smap + jj * CPC);
    const T *cv = isim ? conv_im : conv_re;
    union {
      uint4 v;
      T t[CPC];
    } o;
#pragma unroll
    for (int e = 0; e < CPC; ++e) {
      T val = T();
      const int sl = sm.b[e];
      if (sl != 0xFF) val = cv[sl];
      o.t[e] = val;
    }
    *reinterpret_cast<uint4 *>(row + (isim ? ncm * CB : 0) + ((size_t)jj << 4)) = o.v;
  }
  __syncwarp();
}

// Phasor table of the sparse path, in planes (see ld_planes): copies 2j and
// 2j+1 of window p are entry p of plane j; the reference thread's exact
// fp32 values.
__device__ __forceinline__ void sparse_table(const EncParams &P, float2 *t) {
  const int total = P.m * P.nw;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int idm = i / P.nw, p = i - idm * P.nw;
    const int at = P.m == 1 ? p : (idm >> 1) * 2 * P.nw + 2 * p + (idm & 1);
    t[at] = ref_phasor(P, idm, p);
  }
  __syncthreads();
}

__host__ __device__ inline size_t sparse_table_bytes(const EncParams &P) {
  return ((size_t)P.m * P.nw * 8 + 15) & ~(size_t)15;
}

template <int OUT, int M>
__global__ void __launch_bounds__(256) k_encode_sparse(EncParams P, const uint32_t *__restrict__ dnas, int64_t n,
                                                       void *dest, float *norms, float *scales) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2 *table = reinterpret_cast<float2 *>(smem);
  sparse_table(P, table);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const SparseLayout L = sparse_layout(P.c, M, P.sp_nslot, OutT<OUT>::bytes);
  unsigned char *warea = smem + sparse_table_bytes(P) + (size_t)L.warp * warp;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const size_t rowbytes = (size_t)P.rdim * OutT<OUT>::bytes;
  int64_t f = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  uint32_t wnext = (f < n && lane < P.W) ? __ldg(dnas + f * P.W + lane) : 0u;
  for (; f < n; f += nwarps) {
    const uint32_t wreg = wnext;
    const int64_t fn = f + nwarps;
    wnext = (fn < n && lane < P.W) ? __ldg(dnas + fn * P.W + lane) : 0u;  // next fragment's words in flight
    sparse_fragment<OUT, M>(P, table, warea, wreg, reinterpret_cast<unsigned char *>(dest) + rowbytes * f,
                            norms + f * M, scales ? scales + f : nullptr);
  }
}

template <int OUT, int M>
__global__ void __launch_bounds__(256, M <= 4 ? 4 : 1) k_encode_sparse_ref(EncParams P, const uint32_t *__restrict__ genome,
                                                           const int64_t *__restrict__ win_pos, int64_t nwin,
                                                           int64_t batch, void *dest, float *norms,
                                                           float *scales) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2 *table = reinterpret_cast<float2 *>(smem);
  sparse_table(P, table);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  const SparseLayout L = sparse_layout(P.c, M, P.sp_nslot, OutT<OUT>::bytes);
  unsigned char *warea = smem + sparse_table_bytes(P) + (size_t)L.warp * warp;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const size_t rowbytes = (size_t)P.rdim * OutT<OUT>::bytes;
  const int rr = P.k & 15;
  const uint32_t tailmask = rr == 0 ? 0xFFFFFFFFu : ((1u << (2 * rr)) - 1u);
  const uint32_t shbits = (uint32_t)(32 * P.W - 2 * P.k);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; i < nwin; i += nwarps) {
    const int64_t pos = __ldg(win_pos + i);
    const int64_t q = pos >> 4;
    uint32_t fw = 0u;
    if (lane < P.W) {
      const uint32_t a = __ldg(genome + q + lane), b = __ldg(genome + q + lane + 1);
      fw = __funnelshift_r(a, b, (uint32_t)(pos & 15) << 1);
      if (lane == P.W - 1) fw &= tailmask;
    }
    // reverse complement: complement, left-align the k bases to the end of
    // the W-word stream, reverse the word order and the sixteen 2-bit lanes
    const int src = P.W - 1 - lane;
    const uint32_t xi = ~__shfl_sync(FULL, fw, src & 31), xm = ~__shfl_sync(FULL, fw, (src - 1) & 31);
    uint32_t vv = xi;
    if (shbits != 0) vv = (xi << shbits) | (src > 0 ? (xm >> (32u - shbits)) : 0u);
    const uint32_t rcw = lane < P.W ? lanerev32(vv) : 0u;
    const int64_t bt = i / batch, off = i - bt * batch;
    const int64_t nb = min(batch, nwin - bt * batch);
    const int64_t colf = 2 * bt * batch + off, colr = colf + nb;
    sparse_fragment<OUT, M>(P, table, warea, fw, reinterpret_cast<unsigned char *>(dest) + rowbytes * colf,
                            norms + colf * M, scales ? scales + colf : nullptr);
    sparse_fragment<OUT, M>(P, table, warea, rcw, reinterpret_cast<unsigned char *>(dest) + rowbytes * colr,
                            norms + colr * M, scales ? scales + colr : nullptr);
  }
}

__global__ void k_f32_to_e4m3(uint8_t *dst, const float *src, int64_t count) {
  int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  int64_t stride = (int64_t)gridDim.x * blockDim.x * 4;
  for (; i < count; i += stride) {
    if (i + 4 <= count && ((reinterpret_cast<uintptr_t>(src + i) & 15) == 0)) {
      float4 v = *reinterpret_cast<const float4 *>(src + i);
      uint32_t lo = f32x2_to_e4m3x2(v.x, v.y), hi = f32x2_to_e4m3x2(v.z, v.w);
      uint32_t w = lo | (hi << 16);
      dst[i] = w & 0xFF; dst[i + 1] = (w >> 8) & 0xFF; dst[i + 2] = (w >> 16) & 0xFF; dst[i + 3] = w >> 24;
    } else {
      for (int64_t j = i; j < i + 4 && j < count; ++j) dst[j] = f32_to_e4m3(src[j]);
    }
  }
}

__global__ void k_f16_to_e4m3(uint8_t *dst, const __half *src, int64_t count) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
    dst[i] = f32_to_e4m3(__half2float(src[i]));
}

// ------------------------------------------------------------------ host

static size_t warp_bytes_host(const EncParams &P) {
  return (size_t)P.hist_floats * 4 + (size_t)P.cs_u16 * 2 + (size_t)P.words_u32 * 4 * 2 + 32;
}

template <int OUT, typename KernelFn>
static int plan_launch(EncParams &P, KernelFn kern, int64_t nwork, int *grid, int *block,
                       size_t *smem, float2 **gtable, cudaStream_t st) {
  const size_t kSmemCap = 200 * 1024;
  size_t tb = ((size_t)P.m * P.nw * 8 + 15) & ~(size_t)15;
  size_t wb = warp_bytes_host(P);
  P.table_in_smem = (tb + wb * 2 <= 100 * 1024) ? 1 : 0;
  size_t fixed = P.table_in_smem ? tb : 0;
  int wpb = 8;
  while (wpb > 1 && fixed + wb * wpb > kSmemCap) wpb >>= 1;
  if (fixed + wb * wpb > kSmemCap) return fail(R2M_EINVAL, "encoder shared memory does not fit (k or m*4^c too large)");
  *block = 32 * wpb;
  *smem = fixed + wb * wpb;
  R2M_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
  int per_sm = 0;
  R2M_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, *block, *smem));
  if (per_sm < 1) per_sm = 1;
  int64_t want = (nwork + wpb - 1) / wpb;
  int64_t cap = (int64_t)sm_count() * per_sm;
  *grid = (int)(want < cap ? want : cap);
  if (*grid < 1) *grid = 1;
  *gtable = nullptr;
  if (!P.table_in_smem) {
    float2 *t = nullptr;
    R2M_CUDA(cudaMallocAsync(&t, (size_t)P.m * P.nw * sizeof(float2), st));
    int nchunk = (P.nw + P.Wc - 1) / P.Wc;
    int tot = nchunk * P.m;
    k_phasor_table<<<(tot + 127) / 128, 128, 0, st>>>(P, t);
    R2M_CUDA(cudaGetLastError());
    *gtable = t;
  }
  return R2M_OK;
}

// The sparse path serves normalize = 0 with m in {1, 2, 4, 8}, at most 255
// distinct c-mers per fragment, whole 16-byte output chunks per c-mer run
// and k <= 496 (the words of a fragment fit one warp's registers).  The
// environment variable R2M_ENCODER=dense (or sparse) forces a path.
static bool sparse_ok(const EncParams &P, int outb) {
  const char *force = getenv("R2M_ENCODER");
  if (force && strcmp(force, "dense") == 0) return false;
  if (P.normalize != 0) return false;
  if (P.m != 1 && P.m != 2 && P.m != 4 && P.m != 8) return false;
  const int CB = P.m * outb;
  if (CB > 16) return false;
  const long long ncm = 1LL << (2 * P.c);
  if (ncm * CB < 16) return false;
  if (P.sp_nslot > 255 || P.W > 31) return false;
  const SparseLayout L = sparse_layout(P.c, P.m, P.sp_nslot, outb);
  return sparse_table_bytes(P) + (size_t)L.warp * 2 <= 200 * 1024;
}

template <typename KernelFn>
static int sparse_grid(KernelFn kern, const EncParams &P, int outb, int64_t nwork, int *grid, int *block,
                       size_t *smem) {
  const SparseLayout L = sparse_layout(P.c, P.m, P.sp_nslot, outb);
  int wpb = 8;
  while (wpb > 1 && sparse_table_bytes(P) + (size_t)L.warp * wpb > 200 * 1024) wpb >>= 1;
  *block = 32 * wpb;
  *smem = sparse_table_bytes(P) + (size_t)L.warp * wpb;
  R2M_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
  int per_sm = 0;
  R2M_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, *block, *smem));
  if (per_sm < 1) per_sm = 1;
  const int64_t want = (nwork + wpb - 1) / wpb, cap = (int64_t)sm_count() * per_sm;
  *grid = (int)(want < cap ? want : cap);
  if (*grid < 1) *grid = 1;
  return R2M_OK;
}

template <int OUT, int M>
static int launch_sparse_frags(const EncParams &P, void *dest, float *norms, float *scales, const uint32_t *dnas,
                               int64_t n, cudaStream_t st) {
  if constexpr (M * OutT<OUT>::bytes > 16) {
    return fail(R2M_EINVAL, "sparse encoder: output run too wide");
  } else {
    int grid, block;
    size_t smem;
    int rc = sparse_grid(k_encode_sparse<OUT, M>, P, OutT<OUT>::bytes, n, &grid, &block, &smem);
    if (rc) return rc;
    k_encode_sparse<OUT, M><<<grid, block, smem, st>>>(P, dnas, n, dest, norms, scales);
    R2M_CUDA(cudaGetLastError());
    return R2M_OK;
  }
}

template <int OUT, int M>
static int launch_sparse_ref(const EncParams &P, void *dest, float *norms, float *scales, const uint32_t *genome,
                             const int64_t *pos, int64_t nwin, int64_t batch, cudaStream_t st) {
  if constexpr (M * OutT<OUT>::bytes > 16) {
    return fail(R2M_EINVAL, "sparse encoder: output run too wide");
  } else {
    int grid, block;
    size_t smem;
    int rc = sparse_grid(k_encode_sparse_ref<OUT, M>, P, OutT<OUT>::bytes, nwin, &grid, &block, &smem);
    if (rc) return rc;
    k_encode_sparse_ref<OUT, M><<<grid, block, smem, st>>>(P, genome, pos, nwin, batch, dest, norms, scales);
    R2M_CUDA(cudaGetLastError());
    return R2M_OK;
  }
}

template <int OUT>
static int launch_frags(EncParams P, void *dest, float *norms, float *scales, const uint32_t *dnas,
                        int64_t n, cudaStream_t st) {
  if (sparse_ok(P, OutT<OUT>::bytes)) {
    switch (P.m) {
      case 1: return launch_sparse_frags<OUT, 1>(P, dest, norms, scales, dnas, n, st);
      case 2: return launch_sparse_frags<OUT, 2>(P, dest, norms, scales, dnas, n, st);
      case 4: return launch_sparse_frags<OUT, 4>(P, dest, norms, scales, dnas, n, st);
      default: return launch_sparse_frags<OUT, 8>(P, dest, norms, scales, dnas, n, st);
    }
  }
  int grid, block;
  size_t smem;
  float2 *gt = nullptr;
  int rc = plan_launch<OUT>(P, k_encode_frags<OUT>, n, &grid, &block, &smem, &gt, st);
  if (rc) return rc;
  k_encode_frags<OUT><<<grid, block, smem, st>>>(P, dnas, n, dest, norms, scales, gt);
  cudaError_t e = cudaGetLastError();
  if (gt) cudaFreeAsync(gt, st);
  if (e != cudaSuccess) return cuda_fail(e, "k_encode_frags launch");
  return R2M_OK;
}

template <int OUT>
static int launch_ref(EncParams P, void *dest, float *norms, float *scales, const uint32_t *genome,
                      const int64_t *pos, int64_t nwin, int64_t batch, cudaStream_t st) {
  if (sparse_ok(P, OutT<OUT>::bytes)) {
    switch (P.m) {
      case 1: return launch_sparse_ref<OUT, 1>(P, dest, norms, scales, genome, pos, nwin, batch, st);
      case 2: return launch_sparse_ref<OUT, 2>(P, dest, norms, scales, genome, pos, nwin, batch, st);
      case 4: return launch_sparse_ref<OUT, 4>(P, dest, norms, scales, genome, pos, nwin, batch, st);
      default: return launch_sparse_ref<OUT, 8>(P, dest, norms, scales, genome, pos, nwin, batch, st);
    }
  }
  int grid, block;
  size_t smem;
  float2 *gt = nullptr;
  int rc = plan_launch<OUT>(P, k_encode_ref<OUT>, nwin, &grid, &block, &smem, &gt, st);
  if (rc) return rc;
  k_encode_ref<OUT><<<grid, block, smem, st>>>(P, genome, pos, nwin, batch, dest, norms, scales, gt);
  cudaError_t e = cudaGetLastError();
  if (gt) cudaFreeAsync(gt, st);
  if (e != cudaSuccess) return cuda_fail(e, "k_encode_ref launch");
  return R2M_OK;
}

static int check_align(const void *p, size_t a, const char *what) {
  if ((reinterpret_cast<uintptr_t>(p) % a) != 0)
    return fail(R2M_EINVAL, std::string(what) + " must be " + std::to_string(a) + "-byte aligned");
  return R2M_OK;
}

}  // namespace r2m

using namespace r2m;

extern "C" int r2m_encode_frag_real_batch(void *dest, int out_kind, float *dest_norms,
                                          float *dest_scales, const uint32_t *dnas, int64_t n,
                                          int k, int s, int m, int c, int normalize,
                                          r2m_stream_t stream) {
  EncParams P;
  int rc = make_params(P, k, s, m, c, normalize);
  if (rc) return rc;
  R2M_REQUIRE(n >= 0, "n must be >= 0");
  if (n == 0) return R2M_OK;
  R2M_REQUIRE(dest && dest_norms && dnas, "null pointer");
  R2M_REQUIRE(out_kind >= R2M_OUT_F32 && out_kind <= R2M_OUT_E4M3_SCALED, "bad out_kind");
  R2M_REQUIRE(out_kind != R2M_OUT_E4M3_SCALED || dest_scales, "scaled e4m3 needs dest_scales");
  if ((rc = check_align(dest, 16, "dest"))) return rc;
  cudaStream_t st = as_stream(stream);
  switch (out_kind) {
    case R2M_OUT_F32: return launch_frags<R2M_OUT_F32>(P, dest, dest_norms, nullptr, dnas, n, st);
    case R2M_OUT_F16: return launch_frags<R2M_OUT_F16>(P, dest, dest_norms, nullptr, dnas, n, st);
    case R2M_OUT_E4M3: return launch_frags<R2M_OUT_E4M3>(P, dest, dest_norms, nullptr, dnas, n, st);
    default: return launch_frags<R2M_OUT_E4M3_SCALED>(P, dest, dest_norms, dest_scales, dnas, n, st);
  }
}

extern "C" int r2m_encode_ref_windows(void *dest, int out_kind, float *dest_norms,
                                      float *dest_scales, const uint32_t *genome,
                                      const int64_t *win_pos, int64_t nwin, int64_t batch_size,
                                      int k, int s, int m, int c, int normalize,
                                      r2m_stream_t stream) {
  EncParams P;
  int rc = make_params(P, k, s, m, c, normalize);
  if (rc) return rc;
  R2M_REQUIRE(nwin >= 0, "nwin must be >= 0");
  R2M_REQUIRE(batch_size >= 1, "batch_size must be >= 1");
  if (nwin == 0) return R2M_OK;
  R2M_REQUIRE(dest && dest_norms && genome && win_pos, "null pointer");
  R2M_REQUIRE(out_kind >= R2M_OUT_F32 && out_kind <= R2M_OUT_E4M3_SCALED, "bad out_kind");
  R2M_REQUIRE(out_kind != R2M_OUT_E4M3_SCALED || dest_scales, "scaled e4m3 needs dest_scales");
  if ((rc = check_align(dest, 16, "dest"))) return rc;
  cudaStream_t st = as_stream(stream);
  switch (out_kind) {
    case R2M_OUT_F32:
      return launch_ref<R2M_OUT_F32>(P, dest, dest_norms, nullptr, genome, win_pos, nwin, batch_size, st);
    case R2M_OUT_F16:
      return launch_ref<R2M_OUT_F16>(P, dest, dest_norms, nullptr, genome, win_pos, nwin, batch_size, st);
    case R2M_OUT_E4M3:
      return launch_ref<R2M_OUT_E4M3>(P, dest, dest_norms, nullptr, genome, win_pos, nwin, batch_size, st);
    default:
      return launch_ref<R2M_OUT_E4M3_SCALED>(P, dest, dest_norms, dest_scales, genome, win_pos, nwin,
                                             batch_size, st);
  }
}

extern "C" int r2m_revcomp_frag_words(uint32_t *drc, const uint32_t *dnas, int k, int64_t n,
                                      r2m_stream_t stream) {
  R2M_REQUIRE(k >= 1, "k must be >= 1");
  R2M_REQUIRE(n >= 0, "n must be >= 0");
  if (n == 0) return R2M_OK;
  R2M_REQUIRE(drc && dnas, "null pointer");
  int W = (k + 15) / 16;
  uint32_t sh = (uint32_t)(32 * W - 2 * k);
  int64_t total = (int64_t)W * n;
  int64_t blocks = (total + 255) / 256;
  k_revcomp<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(drc, dnas, W, n, sh);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}

extern "C" int r2m_f32_to_e4m3(uint8_t *dst, const float *src, int64_t count, r2m_stream_t stream) {
  R2M_REQUIRE(count >= 0, "count must be >= 0");
  if (count == 0) return R2M_OK;
  R2M_REQUIRE(dst && src, "null pointer");
  int64_t blocks = (count / 4 + 255) / 256 + 1;
  if (blocks > 65535) blocks = 65535;
  k_f32_to_e4m3<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(dst, src, count);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}

extern "C" int r2m_f16_to_e4m3(uint8_t *dst, const uint16_t *src, int64_t count, r2m_stream_t stream) {
  R2M_REQUIRE(count >= 0, "count must be >= 0");
  if (count == 0) return R2M_OK;
  R2M_REQUIRE(dst && src, "null pointer");
  int64_t blocks = (count + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  k_f16_to_e4m3<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(dst, reinterpret_cast<const __half *>(src),
                                                                  count);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}

// ------------------------------------------------------------------
// FP32 exact rescoring of top-k candidates.  For each read (one warp) the
// fp32 embedding is rebuilt with the encoder's arithmetic, then every
// candidate's reference window is re-encoded on the fly from the packed
// genome (forward, or reverse complement for strand-1 columns) and scored as
// the fp32 dot product of the two unquantised embeddings (fixed lane-strided
// order + xor-tree reduction, so scores are deterministic).  The candidates
// are re-ranked by that score (descending, ties by column).
namespace r2m {

constexpr int kMaxCand = 64;

__global__ void __launch_bounds__(128) k_rescore_fp32(EncParams P, const uint32_t *__restrict__ dnas,
                                                      int nb, const int *__restrict__ cand, int kc,
                                                      const uint32_t *__restrict__ genome,
                                                      const int64_t *__restrict__ col_pos,
                                                      const uint8_t *__restrict__ strand, long long N,
                                                      float *scores, float *out_v, int *out_l, int k,
                                                      const float2 *gtable) {
  extern __shared__ __align__(16) unsigned char smem[];
  const float2 *table = block_table(P, smem, gtable);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  unsigned char *base = smem + table_bytes(P);
  const size_t per = warp_smem_bytes(P) + (size_t)P.rdim * 4 + 2 * kMaxCand * 4 + 32;
  unsigned char *mine = base + per * warp;
  WarpSmem ws = carve(P, mine, 0);
  float *emb = reinterpret_cast<float *>(mine + warp_smem_bytes(P));
  float *sc = emb + P.rdim;
  int *scol = reinterpret_cast<int *>(sc + kMaxCand);
  float *rnrm = reinterpret_cast<float *>(scol + kMaxCand);
  const int nwarps_total = gridDim.x * (blockDim.x >> 5);
  const int rstart = blockIdx.x * (blockDim.x >> 5) + warp;
  const int W = P.W;
  const int rr = P.k & 15;
  const uint32_t tailmask = rr == 0 ? 0xFFFFFFFFu : ((1u << (2 * rr)) - 1u);
  for (int row = rstart; row < nb; row += nwarps_total) {
    // read embedding
    for (int i = lane; i < W; i += 32) ws.words[i] = __ldg(dnas + (size_t)row * W + i);
    if (lane == 0) ws.words[W] = 0u;
    __syncwarp();
    fragment_hist(P, table, ws.hist, ws.cs, ws.words, ws.nrmv, rnrm);
    for (int i = lane; i < P.rdim; i += 32) emb[i] = out_value<R2M_OUT_F32>(P, ws.hist, ws.nrmv, i, 1.0f);
    __syncwarp();
    for (int j = 0; j < kc; ++j) {
      const int c1 = __ldg(cand + (size_t)row * kc + j);
      float s = -INFINITY;
      if (c1 >= 1 && c1 <= N) {
        const long long col = c1 - 1;
        const int64_t pos = __ldg(col_pos + col);
        const int64_t q = pos >> 4;
        const uint32_t sh = (uint32_t)(pos & 15) << 1;
        for (int t = lane; t < W; t += 32) {
          uint32_t a = __ldg(genome + q + t), b = __ldg(genome + q + t + 1);
          uint32_t v = sh == 0 ? a : ((a >> sh) | (b << (32u - sh)));
          if (t == W - 1) v &= tailmask;
          ws.words2[t] = v;
        }
        __syncwarp();
        const uint32_t *src = ws.words2;
        if (__ldg(strand + col)) {
          for (int t = lane; t < W; t += 32) {
            uint32_t w = 0;
            for (int b = 0; b < 16; ++b) {
              int x = 16 * t + b;
              if (x < P.k) {
                int y = P.k - 1 - x;
                w |= (3u - ((ws.words2[y >> 4] >> (2 * (y & 15))) & 3u)) << (2 * b);
              }
            }
            ws.words[t] = w;
          }
          src = ws.words;
        }
        if (lane == 0) {
          ws.words[W] = 0u;
          ws.words2[W] = 0u;
        }
        __syncwarp();
        fragment_hist(P, table, ws.hist, ws.cs, src, ws.nrmv, rnrm);
        float acc = 0.f;
        for (int i = lane; i < P.rdim; i += 32)
          acc = fmaf(emb[i], out_value<R2M_OUT_F32>(P, ws.hist, ws.nrmv, i, 1.0f), acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
        s = acc;
      }
      if (lane == 0) {
        sc[j] = s;
        scol[j] = c1;
        if (scores) scores[(size_t)row * kc + j] = s;
      }
      __syncwarp();
    }
    // re-rank (kc <= 64): lane 0 selection sort, value desc then column asc
    if (lane == 0) {
      for (int a = 0; a < k; ++a) {
        int best = a;
        for (int b = a + 1; b < kc; ++b) {
          bool better = sc[b] > sc[best] || (sc[b] == sc[best] && scol[b] < scol[best]);
          if (better) best = b;
        }
        float tv = sc[a];
        int tc = scol[a];
        sc[a] = sc[best];
        scol[a] = scol[best];
        sc[best] = tv;
        scol[best] = tc;
        out_v[(size_t)row * k + a] = sc[a];
        out_l[(size_t)row * k + a] = sc[a] == -INFINITY ? 0 : scol[a];
      }
    }
    __syncwarp();
  }
}

}  // namespace r2m

extern "C" int r2m_rescore_fp32(const uint32_t *dnas, int nb, const int32_t *cand, int kc,
                                const uint32_t *genome, const int64_t *col_pos, const uint8_t *strand,
                                int64_t N, int k, int s, int m, int c, int normalize, float *scores,
                                float *out_vals, int32_t *out_locs, int topk, r2m_stream_t stream) {
  EncParams P;
  int rc = make_params(P, k, s, m, c, normalize);
  if (rc) return rc;
  R2M_REQUIRE(nb >= 0, "nb must be >= 0");
  R2M_REQUIRE(kc >= 1 && kc <= kMaxCand, "candidates per read must be in 1..64");
  R2M_REQUIRE(topk >= 1 && topk <= kc, "need 1 <= topk <= candidates");
  if (nb == 0) return R2M_OK;
  R2M_REQUIRE(dnas && cand && genome && col_pos && strand && out_vals && out_locs, "null pointer");
  cudaStream_t st = as_stream(stream);
  size_t tb = ((size_t)P.m * P.nw * 8 + 15) & ~(size_t)15;
  size_t per = warp_bytes_host(P) + (size_t)P.rdim * 4 + 2 * kMaxCand * 4 + 32;
  P.table_in_smem = (tb + per * 4 <= 200 * 1024) ? 1 : 0;
  size_t smem = (P.table_in_smem ? tb : 0) + per * 4;
  R2M_REQUIRE(smem <= 220 * 1024, "rescoring shared memory does not fit (k or m*4^c too large)");
  R2M_CUDA(cudaFuncSetAttribute(k_rescore_fp32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  float2 *gt = nullptr;
  if (!P.table_in_smem) {
    R2M_CUDA(cudaMallocAsync(&gt, (size_t)P.m * P.nw * sizeof(float2), st));
    int nchunk = (P.nw + P.Wc - 1) / P.Wc;
    k_phasor_table<<<(nchunk * P.m + 127) / 128, 128, 0, st>>>(P, gt);
  }
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rescore_fp32, 128, smem);
  long long want = (nb + 3) / 4, cap = (long long)sm_count() * (per_sm > 0 ? per_sm : 1);
  int grid = (int)(want < cap ? want : cap);
  k_rescore_fp32<<<grid, 128, smem, st>>>(P, dnas, nb, cand, kc, genome, col_pos, strand, N, scores, out_vals,
                                          out_locs, topk, gt);
  cudaError_t e = cudaGetLastError();
  if (gt) cudaFreeAsync(gt, st);
  if (e != cudaSuccess) return cuda_fail(e, "k_rescore_fp32 launch");
  return R2M_OK;
}
