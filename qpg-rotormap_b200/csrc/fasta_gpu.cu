// fasta_gpu.cu -- device FASTA reader for read sets: the FASTA bytes already
// in HBM -> forward 2-bit words of every record's first k bases plus each
// kept record's header span.  Same records, words and headers as the host
// reader (fasta.cpp, which follows RotorMap/fasta/reader.jl:21-28,61-75,
// 120-198,204-311):
//   * a record starts at a '>' that is the first byte or follows '\n'/'\r';
//   * the header is [start, first '\n'), one trailing '\r' removed; the first
//     record whose header line is not closed before the next record start
//     (or the end) ends the parse: it and every later record are dropped;
//   * sequence bytes other than '\n'/'\r' are bases: A/C/G/T either case ->
//     0/1/2/3, anything else -> 2;
//   * records with fewer than k bases are skipped; base j of a kept record
//     sits in word j>>4 at bits 2*(j&15), the tail zero-padded.
//
// Passes (all on one stream):
//   1. k_count_starts  : 4 KB tiles (256 threads x 16 bytes), record starts
//                        counted per tile;
//   2. scan            : exclusive scan of the tile counts;
//   3. k_write_starts  : the starts written in file order;
//   4. k_parse_records : G lanes per record (8/16/32 by mean record size),
//                        windows of G aligned 16-byte chunks (one per
//                        lane): header end by ballot, then each lane's bases
//                        OR-ed as one 2-bit field into shared word staging,
//                        flushed as whole words;
//   5. scans           : exclusive scans of the kept flags and the kept
//                        header lengths, cut at the first unclosed header
//                        (one block up to 64K entries, three passes above);
//   6. compaction      : kept records' words moved to their file-order rank
//                        (skipped when every record before the cut is kept),
//                        their spans too, and their headers into one blob
//                        (each header followed by '\n').
// Passes 1, 3 read the input once each; pass 4 reads each record's header
// and its first k bases (plus line breaks), so the traffic is about
// 2 x input + kept words + headers.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "common.cuh"
#include "r2m.h"

struct r2m_dreads {
  int k = 0, W = 0;
  int64_t n = 0;
  uint32_t *words = nullptr;  // n x W
  int64_t *spans = nullptr;   // n x 2: header [start, end) byte offsets
  uint8_t *heads = nullptr;   // every header followed by '\n'
  size_t head_bytes = 0;
  bool stopped = false;  // an unclosed header ended the parse
  cudaStream_t stream = nullptr;
};

namespace {

constexpr int kTileThreads = 256;
constexpr int kTileBytes = kTileThreads * 16;
constexpr int kParseWarps = 8;
constexpr int kScanThreads = 1024;

__device__ __forceinline__ bool is_break(uint8_t b) { return b == '\n' || b == '\r'; }

__device__ __forceinline__ uint32_t base_code(uint8_t b) {
  const uint8_t c = b | 0x20;  // ASCII case fold; only 'A'/'a' land on 'a', etc.
  return c == 'a' ? 0u : c == 'c' ? 1u : c == 't' ? 3u : 2u;
}

// Bit j set when byte off+j starts a record.
__device__ __forceinline__ uint32_t start_mask(const uint8_t *__restrict__ d, size_t n, size_t off) {
  uint8_t b[16];
  if (off + 16 <= n && (((uintptr_t)(d + off)) & 15) == 0) {
    const uint4 v = *reinterpret_cast<const uint4 *>(d + off);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int j = 0; j < 16; ++j) b[j] = (uint8_t)(w[j >> 2] >> (8 * (j & 3)));
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) b[j] = off + j < n ? d[off + j] : 0;
  }
  uint8_t prev = off == 0 ? (uint8_t)'\n' : (off - 1 < n ? d[off - 1] : 0);
  uint32_t m = 0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (b[j] == '>' && is_break(prev)) m |= 1u << j;
    prev = b[j];
  }
  return m;
}

__global__ void __launch_bounds__(kTileThreads) k_count_starts(const uint8_t *__restrict__ d, size_t n,
                                                              int32_t *__restrict__ counts) {
  __shared__ int32_t ws[kTileThreads / 32];
  const size_t off = (size_t)blockIdx.x * kTileBytes + threadIdx.x * 16;
  int c = off < n ? __popc(start_mask(d, n, off)) : 0;
#pragma unroll
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < kTileThreads / 32; ++i) t += ws[i];
    counts[blockIdx.x] = t;
  }
}

constexpr int64_t kScanTile = (int64_t)kScanThreads * 4;

// Exclusive scan of in[base, base + kScanTile) (entries at or beyond lim
// count as 0) written to out[] (entries below n) offset by carry; returns
// the tile total to every thread.  Called by all kScanThreads threads.
template <class T>
__device__ __forceinline__ int64_t scan_tile(const T *__restrict__ in, int64_t *__restrict__ out, int64_t base,
                                             int64_t n, int64_t lim, int64_t carry) {
  __shared__ int64_t ws[kScanThreads / 32];
  __shared__ int64_t tile_total;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t i0 = base + (int64_t)threadIdx.x * 4;
  int64_t v[4], t = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    v[j] = i0 + j < lim ? in[i0 + j] : 0;
    t += v[j];
  }
  int64_t inc = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) ws[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const int64_t w = ws[lane];
    int64_t si = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    ws[lane] = si - w;  // exclusive warp offsets
    if (lane == 31) tile_total = si;
  }
  __syncthreads();
  int64_t run = carry + ws[wid] + inc - t;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (i0 + j < n) out[i0 + j] = run;
    run += v[j];
  }
  const int64_t tot = tile_total;
  __syncthreads();  // ws / tile_total are reused by the next call
  return tot;
}

// out[i] = sum of in[j] for j < i, out[n] = the total; entries at or beyond
// *limit (when given) count as 0.  One block walks every tile.
template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_excl(const T *__restrict__ in, int64_t *__restrict__ out,
                                                           int64_t n, const int64_t *__restrict__ limit) {
  const int64_t lim = limit ? min(*limit, n) : n;
  int64_t carry = 0;
  for (int64_t base = 0; base < n; base += kScanTile) carry += scan_tile(in, out, base, n, lim, carry);
  if (threadIdx.x == 0) out[n] = carry;
}

// Multi-block form: per-tile sums, one-block scan of the sums, then every
// tile scanned again from its offset.
template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(const T *__restrict__ in, int64_t n,
                                                           const int64_t *__restrict__ limit,
                                                           int64_t *__restrict__ sums) {
  __shared__ int64_t ws[kScanThreads / 32];
  const int64_t lim = limit ? min(*limit, n) : n;
  const int64_t i0 = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * 4;
  int64_t t = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) t += i0 + j < lim ? in[i0 + j] : 0;
#pragma unroll
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t s = 0;
    for (int i = 0; i < kScanThreads / 32; ++i) s += ws[i];
    sums[blockIdx.x] = s;
  }
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const T *__restrict__ in, int64_t *__restrict__ out,
                                                            int64_t n, const int64_t *__restrict__ limit,
                                                            const int64_t *__restrict__ tile_off, int64_t ntiles) {
  const int64_t lim = limit ? min(*limit, n) : n;
  scan_tile(in, out, (int64_t)blockIdx.x * kScanTile, n, lim, tile_off[blockIdx.x]);
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_off[ntiles];
}

__global__ void __launch_bounds__(kTileThreads) k_write_starts(const uint8_t *__restrict__ d, size_t n,
                                                              const int64_t *__restrict__ tile_off,
                                                              int64_t *__restrict__ starts) {
  __shared__ int32_t ws[kTileThreads / 32];
  const size_t off = (size_t)blockIdx.x * kTileBytes + threadIdx.x * 16;
  uint32_t m = off < n ? start_mask(d, n, off) : 0u;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int c = __popc(m);
  int inc = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) ws[wid] = inc;
  __syncthreads();
  int wbase = 0;
  for (int i = 0; i < wid; ++i) wbase += ws[i];
  int64_t pos = tile_off[blockIdx.x] + wbase + inc - c;
  while (m) {
    const int j = __ffs(m) - 1;
    m &= m - 1;
    starts[pos++] = (int64_t)off + j;
  }
}

// G lanes per record (G = 8, 16 or 32; 32 / G records per warp at once).
// A group reads its record in windows of G 16-byte-aligned chunks, one per
// lane, so a record shorter than about 16 G bytes (header and sequence)
// arrives in a single round trip; the next record's bounds are loaded while
// the current one is parsed.  In each window the header end (first '\n' at
// or after the start) is found by ballot until known; every later byte
// before the record end that is not a line break is a base.  A lane's bases
// are consecutive, so their codes form one bit field of at most 32 bits,
// OR-ed into the group's shared word staging (2 G words; two words at
// most per lane); whole words are flushed to `words` once G of them are
// staged, and the rest when the record ends.  Codes at base index >= k are
// masked out.
// flag[r]: 1 kept, 0 skipped (fewer than k bases or unclosed header); an
// unclosed header also lowers *first_unclosed to r.
template <bool kVec, int G>
__global__ void __launch_bounds__(kParseWarps * 32) k_parse_records(
    const uint8_t *__restrict__ d, size_t n, const int64_t *__restrict__ starts, int64_t R, int k, int W,
    uint32_t *__restrict__ words, int64_t *__restrict__ spans, int32_t *__restrict__ flag,
    int64_t *__restrict__ hlen, unsigned long long *__restrict__ first_unclosed) {
  static_assert(G == 8 || G == 16 || G == 32, "group of 8, 16 or 32 lanes");
  constexpr int SW = 2 * G;  // staged words per group
  __shared__ uint32_t stage_all[kParseWarps * 32 / G][SW];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int gl = lane % G, grp = lane / G;
  const uint32_t gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (grp * G));
  uint32_t *stage = stage_all[wid * (32 / G) + grp];
  const int64_t ngroups = (int64_t)gridDim.x * kParseWarps * (32 / G);
  int64_t r = ((int64_t)blockIdx.x * kParseWarps + wid) * (32 / G) + grp;
  size_t s = 0, e = 0;
  if (r < R) {
    s = (size_t)starts[r];
    e = r + 1 < R ? (size_t)starts[r + 1] : n;
  }
  for (; r < R; r += ngroups) {
    // bounds of this group's next record, loaded ahead
    const int64_t rn = r + ngroups;
    size_t sn = 0, en = 0;
    if (rn < R) {
      sn = (size_t)starts[rn];
      en = rn + 1 < R ? (size_t)starts[rn + 1] : n;
    }
    stage[gl] = 0;
    stage[gl + G] = 0;
    __syncwarp(gmask);
    bool have_h = false;
    size_t h = 0;
    int64_t total = 0, flushed = 0;
    for (size_t win = s & ~(size_t)15; win < e && total < k; win += 16 * G) {
      const size_t c0 = win + 16 * (size_t)gl;
      uint32_t q[4];
      if (kVec && c0 + 16 <= n) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(d + c0));
        q[0] = v.x, q[1] = v.y, q[2] = v.z, q[3] = v.w;
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          uint32_t w = 0;
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (c0 + 4 * i + j < n) w |= (uint32_t)d[c0 + 4 * i + j] << (8 * j);
          q[i] = w;
        }
      }
      if (!have_h) {
        int jn = 16;
#pragma unroll
        for (int j = 15; j >= 0; --j) {
          const uint8_t b = (uint8_t)(q[j >> 2] >> (8 * (j & 3)));
          if (b == '\n' && c0 + j >= s && c0 + j < e) jn = j;
        }
        const uint32_t hit = (__ballot_sync(gmask, jn < 16) & gmask) >> (grp * G);
        if (!hit) continue;  // the whole window is header
        const int src = __ffs(hit) - 1;
        h = win + 16 * (size_t)src + (size_t)__shfl_sync(gmask, jn, src, G);
        have_h = true;
      }
      uint32_t codes = 0;
      int nb = 0;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const uint8_t b = (uint8_t)(q[j >> 2] >> (8 * (j & 3)));
        if (c0 + j > h && c0 + j < e && !is_break(b)) {
          codes |= base_code(b) << (2 * nb);
          ++nb;
        }
      }
      int inc = nb;
#pragma unroll
      for (int o = 1; o < G; o <<= 1) {
        const int y = __shfl_up_sync(gmask, inc, o, G);
        if (gl >= o) inc += y;
      }
      const int64_t b0 = total + inc - nb;
      const int64_t nbk = max((int64_t)0, min((int64_t)nb, (int64_t)k - b0));
      if (nbk > 0) {
        const uint32_t field = nbk == 16 ? codes : codes & ((1u << (2 * nbk)) - 1u);
        const int li = (int)(b0 - flushed);
        const int wi = li >> 4, sh = 2 * (li & 15);
        atomicOr(&stage[wi], field << sh);
        if (sh && sh + 2 * nbk > 32) atomicOr(&stage[wi + 1], field >> (32 - sh));
      }
      total += __shfl_sync(gmask, inc, G - 1, G);
      __syncwarp(gmask);
      const int64_t have = min(total, (int64_t)k) - flushed;
      if (have >= 16 * G) {  // flush the whole words, keep the partial one
        const int full = (int)(have >> 4);
        const uint32_t w0 = stage[gl], w1 = stage[gl + G], part = stage[full];
        uint32_t *o = words + (size_t)r * W + (flushed >> 4);
        if (gl < full) o[gl] = w0;
        if (gl + G < full) o[gl + G] = w1;
        __syncwarp(gmask);
        stage[gl] = gl == 0 ? part : 0u;
        stage[gl + G] = 0;
        __syncwarp(gmask);
        flushed += 16 * full;
      }
    }
    if (!have_h) {
      if (gl == 0) {
        flag[r] = 0;
        hlen[r] = 0;
        atomicMin(first_unclosed, (unsigned long long)r);
      }
    } else {
      size_t hend = h;
      if (hend > s && d[hend - 1] == '\r') --hend;
      const bool kept = total >= k;
      if (kept) {
        const int left = W - (int)(flushed >> 4);
        uint32_t *o = words + (size_t)r * W + (flushed >> 4);
        if (gl < left) o[gl] = stage[gl];
        if (gl + G < left) o[gl + G] = stage[gl + G];
      }
      if (gl == 0) {
        flag[r] = kept ? 1 : 0;
        hlen[r] = kept ? (int64_t)(hend - s + 1) : 0;  // header + '\n' in the blob
        spans[2 * r] = (int64_t)s;
        spans[2 * r + 1] = (int64_t)hend;
      }
    }
    __syncwarp(gmask);
    s = sn;
    e = en;
  }
}

// Kept records' words to their rank (one thread per word); skipped when
// every record before the cut was kept (the slot order is then the rank).
__global__ void k_compact_words(const uint32_t *__restrict__ words, const int32_t *__restrict__ flag,
                                const int64_t *__restrict__ rank, int64_t lim, int W,
                                uint32_t *__restrict__ out_words) {
  const int64_t total = lim * W;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / W;
    if (flag[r]) out_words[rank[r] * W + (t - r * W)] = words[t];
  }
}

// Kept records' spans to their rank and their headers into the blob, each
// followed by '\n'.  One warp per 32 consecutive records: the lanes load
// the 32 records' metadata at once, then stride over the chunk's part of
// the blob (contiguous, since hoff is a scan in record order), finding each
// output byte's record by a 5-step search of the 32 offsets, so all the
// header loads are independent.
__global__ void __launch_bounds__(256) k_compact_heads(const uint8_t *__restrict__ d,
                                                       const int64_t *__restrict__ spans,
                                                       const int32_t *__restrict__ flag,
                                                       const int64_t *__restrict__ rank,
                                                       const int64_t *__restrict__ hoff, int64_t lim,
                                                       int64_t *__restrict__ out_spans,
                                                       uint8_t *__restrict__ heads) {
  __shared__ int64_t off_all[8][33], src_all[8][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t *off = off_all[wid], *src = src_all[wid];
  const int64_t nchunks = (lim + 31) / 32;
  for (int64_t c = (int64_t)blockIdx.x * 8 + wid; c < nchunks; c += (int64_t)gridDim.x * 8) {
    const int64_t r = c * 32 + lane;
    int64_t a = 0;
    if (r < lim) {
      a = spans[2 * r];
      if (flag[r]) {
        const int64_t dst = rank[r];
        out_spans[2 * dst] = a;
        out_spans[2 * dst + 1] = spans[2 * r + 1];
      }
    }
    off[lane] = hoff[min(r, lim)];
    src[lane] = a;
    if (lane == 31) off[32] = hoff[min(c * 32 + 32, lim)];
    __syncwarp();
    const int64_t o0 = off[0], o1 = off[32];
    for (int64_t o = o0 + lane; o < o1; o += 32) {
      int j = 0;  // last j with off[j] <= o
#pragma unroll
      for (int step = 16; step; step >>= 1)
        if (j + step < 32 && off[j + step] <= o) j += step;
      const int64_t rel = o - off[j];
      heads[o] = rel + 1 < off[j + 1] - off[j] ? d[src[j] + rel] : (uint8_t)'\n';
    }
    __syncwarp();
  }
}

__global__ void k_set_u64(unsigned long long *p, unsigned long long v) { *p = v; }

struct Scratch {
  static constexpr int kMax = 16;
  cudaStream_t st;
  void *p[kMax] = {};
  int n = 0;
  explicit Scratch(cudaStream_t s) : st(s) {}
  template <class T>
  cudaError_t get(T **dst, size_t count) {
    *dst = nullptr;
    if (n == kMax) return cudaErrorMemoryAllocation;
    void *q = nullptr;
    cudaError_t e = r2m::pool_alloc(&q, count * sizeof(T) + 16, st);
    if (e == cudaSuccess) p[n++] = q;
    *dst = (T *)q;
    return e;
  }
  // exclusive scan of n int32 -> n + 1 int64 (out[n] = total)
  template <class T>
  cudaError_t scan(const T *in, int64_t *out, int64_t count, const int64_t *limit) {
    if (count <= 16 * kScanTile) {
      k_scan_excl<<<1, kScanThreads, 0, st>>>(in, out, count, limit);
      return cudaGetLastError();
    }
    const int64_t nt = (count + kScanTile - 1) / kScanTile;
    int64_t *sums, *toff;
    cudaError_t e;
    if ((e = get(&sums, nt)) != cudaSuccess || (e = get(&toff, nt + 1)) != cudaSuccess) return e;
    k_scan_sums<<<(unsigned)nt, kScanThreads, 0, st>>>(in, count, limit, sums);
    k_scan_excl<<<1, kScanThreads, 0, st>>>(sums, toff, nt, nullptr);
    k_scan_apply<<<(unsigned)nt, kScanThreads, 0, st>>>(in, out, count, limit, toff, nt);
    return cudaGetLastError();
  }
  // hand an allocation over to the caller (not freed with the scratch)
  void adopt(const void *q) {
    for (int i = 0; i < n; ++i)
      if (p[i] == q) p[i] = nullptr;
  }
  ~Scratch() {
    for (int i = 0; i < n; ++i)
      if (p[i]) cudaFreeAsync(p[i], st);
  }
};

void release(r2m_dreads *r) {
  if (r->words) cudaFreeAsync(r->words, r->stream);
  if (r->spans) cudaFreeAsync(r->spans, r->stream);
  if (r->heads) cudaFreeAsync(r->heads, r->stream);
  r->words = nullptr;
  r->spans = nullptr;
  r->heads = nullptr;
}

}  // namespace

extern "C" int r2m_fasta_reads_device(const void *d_data, size_t len, int k, r2m_stream_t stream,
                                      r2m_dreads **out) {
  R2M_REQUIRE(out != nullptr, "out is null");
  *out = nullptr;
  R2M_REQUIRE(k >= 1, "k must be >= 1");
  R2M_REQUIRE(d_data != nullptr || len == 0, "data is null");
  cudaStream_t st = r2m::as_stream(stream);
  r2m_dreads *res = new r2m_dreads();
  res->k = k;
  res->W = (k + 15) / 16;
  res->stream = st;
  if (len == 0) {
    *out = res;
    return R2M_OK;
  }
  const uint8_t *d = (const uint8_t *)d_data;
  const int W = res->W;
  auto bail = [&](cudaError_t e, const char *what) {
    delete res;
    return r2m::cuda_fail(e, what);
  };
  cudaError_t e;
  {
    Scratch sc(st);
    const int64_t ntiles = (int64_t)((len + kTileBytes - 1) / kTileBytes);
    int32_t *counts;
    int64_t *tile_off;
    if ((e = sc.get(&counts, ntiles)) != cudaSuccess) return bail(e, "cudaMallocAsync");
    if ((e = sc.get(&tile_off, ntiles + 1)) != cudaSuccess) return bail(e, "cudaMallocAsync");
    k_count_starts<<<(unsigned)ntiles, kTileThreads, 0, st>>>(d, len, counts);
    if ((e = sc.scan(counts, tile_off, ntiles, nullptr)) != cudaSuccess) return bail(e, "record scan");
    int64_t R = 0;
    if ((e = cudaMemcpyAsync(&R, tile_off + ntiles, sizeof(R), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return bail(e, "record count");
    if (R == 0) {
      *out = res;
      return R2M_OK;
    }
    int64_t *starts, *spans, *rank, *hoff, *hlen;
    uint32_t *words;
    int32_t *flag;
    unsigned long long *first_unclosed;
    if ((e = sc.get(&starts, R)) != cudaSuccess || (e = sc.get(&spans, 2 * R)) != cudaSuccess ||
        (e = sc.get(&words, (size_t)R * W)) != cudaSuccess || (e = sc.get(&flag, R)) != cudaSuccess ||
        (e = sc.get(&hlen, R)) != cudaSuccess || (e = sc.get(&rank, R + 1)) != cudaSuccess ||
        (e = sc.get(&hoff, R + 1)) != cudaSuccess || (e = sc.get(&first_unclosed, 1)) != cudaSuccess)
      return bail(e, "cudaMallocAsync");
    k_write_starts<<<(unsigned)ntiles, kTileThreads, 0, st>>>(d, len, tile_off, starts);
    k_set_u64<<<1, 1, 0, st>>>(first_unclosed, (unsigned long long)R);
    // lanes per record from the mean record size: a window of 16 G bytes
    // should hold a typical record
    const size_t mean = len / (size_t)R;
    const int G = mean <= 112 ? 8 : mean <= 240 ? 16 : 32;
    const bool vec = (((uintptr_t)d) & 15) == 0;
    const int64_t per_block = (int64_t)kParseWarps * (32 / G);
    const int64_t pblocks = std::min<int64_t>((R + per_block - 1) / per_block, (int64_t)r2m::sm_count() * 8);
    auto parse = [&](auto kern) {
      kern<<<(unsigned)pblocks, kParseWarps * 32, 0, st>>>(d, len, starts, R, k, W, words, spans, flag, hlen,
                                                           first_unclosed);
    };
    if (vec) {
      if (G == 8) parse(k_parse_records<true, 8>);
      else if (G == 16) parse(k_parse_records<true, 16>);
      else parse(k_parse_records<true, 32>);
    } else {
      if (G == 8) parse(k_parse_records<false, 8>);
      else if (G == 16) parse(k_parse_records<false, 16>);
      else parse(k_parse_records<false, 32>);
    }
    const int64_t *lim = (const int64_t *)first_unclosed;
    if ((e = sc.scan(flag, rank, R, lim)) != cudaSuccess || (e = sc.scan(hlen, hoff, R, lim)) != cudaSuccess)
      return bail(e, "kept scan");
    int64_t tot[3] = {0, 0, 0};
    if ((e = cudaMemcpyAsync(&tot[0], rank + R, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot[1], hoff + R, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&tot[2], first_unclosed, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return bail(e, "kept count");
    const int64_t Kc = tot[0], cut = std::min<int64_t>(tot[2], R);
    res->n = Kc;
    res->stopped = cut < R;
    res->head_bytes = (size_t)tot[1];
    if (Kc > 0) {
      const bool all_kept = Kc == cut;  // slot order is already the rank order
      if (all_kept) {
        res->words = words;
        sc.adopt(words);
      } else if ((e = r2m::pool_alloc((void **)&res->words, (size_t)Kc * W * sizeof(uint32_t), st)) != cudaSuccess) {
        release(res);
        return bail(e, "cudaMallocAsync");
      }
      if ((e = r2m::pool_alloc((void **)&res->spans, (size_t)Kc * 2 * sizeof(int64_t), st)) != cudaSuccess ||
          (e = r2m::pool_alloc((void **)&res->heads, res->head_bytes, st)) != cudaSuccess) {
        release(res);
        return bail(e, "cudaMallocAsync");
      }
      const int sms = r2m::sm_count();
      if (!all_kept) {
        const int64_t wb = std::min<int64_t>((cut * W + 255) / 256, (int64_t)sms * 32);
        k_compact_words<<<(unsigned)std::max<int64_t>(wb, 1), 256, 0, st>>>(words, flag, rank, cut, W, res->words);
      }
      const int64_t hb = std::min<int64_t>((cut + 255) / 256, (int64_t)sms * 16);
      k_compact_heads<<<(unsigned)std::max<int64_t>(hb, 1), 256, 0, st>>>(d, spans, flag, rank, hoff, cut,
                                                                          res->spans, res->heads);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) {
      release(res);
      return bail(e, "fasta parse launch");
    }
  }
  *out = res;
  return R2M_OK;
}

extern "C" int64_t r2m_dreads_count(const r2m_dreads *r) { return r ? r->n : 0; }

extern "C" int r2m_dreads_stopped(const r2m_dreads *r) { return r && r->stopped ? 1 : 0; }

extern "C" const uint32_t *r2m_dreads_words(const r2m_dreads *r) { return r ? r->words : nullptr; }

extern "C" const int64_t *r2m_dreads_spans(const r2m_dreads *r) { return r ? r->spans : nullptr; }

extern "C" const uint8_t *r2m_dreads_header_blob(const r2m_dreads *r, size_t *total_len) {
  if (total_len) *total_len = r ? r->head_bytes : 0;
  return r ? r->heads : nullptr;
}

extern "C" void r2m_dreads_free(r2m_dreads *r) {
  if (!r) return;
  release(r);
  delete r;
}
