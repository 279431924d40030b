// compact.cu -- host-ring engine: an index held in host memory (larger than
// the device, or simply not resident) streamed through a ring of device
// chunk slots while the fused GEMM + top-k searches the chunk before.
//
// Mirror of CompactEngine / batch_gemm_topk_compact!
// (RotorMap/search/engine_compact.jl:256-343): the same ring structure -- a
// dedicated non-blocking H2D stream, `depth` device slots, per-slot events
// "copy into slot b done" (waited by the search) and "search reading slot b
// done" (waited by the next copy into b), every wait on the GPU, the host
// loop only enqueues -- with the fused kernel in place of the cuBLASLt chunk
// GEMM and its segmented top-k.
//
// Results are the resident engine's, bit for bit: chunks go in column order;
// each chunk's top-k (values exactly as the resident kernel computes them:
// f16-rounded or fp32, x the column scale for scaled scores) is merged into
// the running top-k by (value desc, column asc), and a column of an earlier
// chunk is always the smaller one, so on equal values the running entry
// wins -- the top-k of the union is the union's top-k under that total order.
// Scaled scores rank before the per-row factor (the resident split merge
// multiplies by scaleA last): chunk searches run with a unit row scale and
// one final pass multiplies by scaleA with the same single rounding.
//
// The first `resident` chunks get slots of their own: each is copied once
// and stays (an index a little larger than the device keeps most of itself in
// HBM and streams only the rest); the remaining chunks go through the ring
// of `depth` slots -- or also get slots of their own when they are no more
// than `depth`.  A search visits the chunks in column order, so the resident
// ones are searched while the first streamed ones are in flight.
#include <cuda_runtime.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"
#include "r2m.h"

using namespace r2m;

struct r2m_compact {
  const uint8_t *hB = nullptr;
  const float *d_scaleB = nullptr;
  int rdim = 0, k = 0, rows_cap = 0, score_mode = 0, depth = 0, resident = 0;
  int64_t N = 0, cap = 0;
  std::vector<int64_t> lo, wi;  // chunk column ranges
  std::vector<uint8_t *> slot;
  std::vector<int64_t> holds;   // chunk kept by each slot (-1: none)
  std::vector<cudaEvent_t> ev_h2d, ev_dev;
  std::vector<bool> used;
  int64_t next = 0;
  r2m_engine *eng = nullptr;
  cudaStream_t h2d = nullptr;
  float *tmp_vals = nullptr, *ones = nullptr;
  int32_t *tmp_locs = nullptr;
  bool registered = false;
};

namespace {

// Merge a chunk's (nb, k) top-k (1-based chunk columns, + off) into the
// running (nb, k) top-k.  One thread per row.
__global__ void k_merge_running(float *__restrict__ vals, int32_t *__restrict__ locs,
                                const float *__restrict__ cv, const int32_t *__restrict__ cl, int nb, int k,
                                int64_t off) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nb) return;
  float rv[64];
  int32_t rl[64];
  for (int t = 0; t < k; ++t) {
    rv[t] = vals[(size_t)r * k + t];
    rl[t] = locs[(size_t)r * k + t];
  }
  const float *c_v = cv + (size_t)r * k;
  const int32_t *c_l = cl + (size_t)r * k;
  int i = 0, j = 0;
  for (int t = 0; t < k; ++t) {
    bool run;
    if (j >= k) run = true;
    else if (i >= k) run = false;
    else {
      const bool run_empty = rl[i] == 0, ch_empty = c_l[j] == 0;
      // equal values: the running column is the smaller one
      run = ch_empty || (!run_empty && rv[i] >= c_v[j]);
    }
    if (run) {
      vals[(size_t)r * k + t] = rv[i];
      locs[(size_t)r * k + t] = rl[i];
      ++i;
    } else {
      vals[(size_t)r * k + t] = c_v[j];
      locs[(size_t)r * k + t] = c_l[j] == 0 ? 0 : (int32_t)(c_l[j] + off);
      ++j;
    }
  }
}

// Merge G sorted (value desc, column asc; empty = column 0) lists of k per
// row, laid out row by row as [list 0 | list 1 | ...] (nb, G*k), into the
// row's top-k.  One warp per row, one lane per list (G <= 32); k rounds of a
// warp arg-max, ties by column then by list.
__global__ void k_merge_lists(const float *__restrict__ vals, const int32_t *__restrict__ locs, int G, int nb,
                              int k, int kout, float *__restrict__ out_v, int32_t *__restrict__ out_l) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= nb) return;
  const unsigned FULL = 0xFFFFFFFFu;
  const float *rv = vals + (size_t)row * G * k;
  const int32_t *rl = locs + (size_t)row * G * k;
  int head = 0;
  auto load = [&](int h, float &v, int &c) {
    if (lane < G && h < k && rl[lane * k + h] != 0) {
      v = rv[lane * k + h];
      c = rl[lane * k + h];
    } else {
      v = -INFINITY;
      c = INT_MAX;
    }
  };
  float hv;
  int hc;
  load(0, hv, hc);
  for (int t = 0; t < kout; ++t) {
    float wv = hv;
    int wc = hc, wl = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(FULL, wv, o);
      const int oc = __shfl_xor_sync(FULL, wc, o);
      const int ol = __shfl_xor_sync(FULL, wl, o);
      const bool better = (ov > wv) || (ov == wv && oc < wc) || (ov == wv && oc == wc && ol < wl);
      wv = better ? ov : wv;
      wc = better ? oc : wc;
      wl = better ? ol : wl;
    }
    if (lane == 0) {
      const bool empty = wc == INT_MAX;
      out_v[(size_t)row * kout + t] = empty ? -INFINITY : wv;
      out_l[(size_t)row * kout + t] = empty ? 0 : wc;
    }
    if (lane == wl) load(++head, hv, hc);
  }
}

__global__ void k_scale_rows(float *__restrict__ vals, const float *__restrict__ scaleA, int nb, int k) {
  const int64_t n = (int64_t)nb * k;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = vals[i];
    vals[i] = v == -INFINITY ? v : v * scaleA[i / k];
  }
}

__global__ void k_fill_f32(float *p, float v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

void destroy(r2m_compact *c) {
  if (!c) return;
  if (c->eng) r2m_engine_destroy(c->eng);
  for (uint8_t *p : c->slot) cudaFree(p);
  for (auto e : c->ev_h2d) cudaEventDestroy(e);
  for (auto e : c->ev_dev) cudaEventDestroy(e);
  if (c->h2d) cudaStreamDestroy(c->h2d);
  cudaFree(c->tmp_vals);
  cudaFree(c->tmp_locs);
  cudaFree(c->ones);
  if (c->registered) cudaHostUnregister((void *)c->hB);
  delete c;
}

}  // namespace

extern "C" int r2m_compact_create(const uint8_t *h_B, const float *d_scaleB, int rdim, int64_t N, int k,
                                  int rows_cap, int score_mode, int64_t chunk_cols, int depth,
                                  int resident_chunks, int pin, const r2m_tuning *tune, r2m_compact **out) {
  R2M_REQUIRE(out != nullptr, "out is null");
  *out = nullptr;
  R2M_REQUIRE(h_B != nullptr, "host B is null");
  R2M_REQUIRE(rdim >= 16 && rdim % 16 == 0, "rdim must be a positive multiple of 16");
  R2M_REQUIRE(k >= 1 && k <= 64 && k <= N, "need 1 <= k <= min(N, 64)");
  R2M_REQUIRE(N <= (1LL << 31) - 1 - 256, "N out of range");
  R2M_REQUIRE(rows_cap >= 1, "rows_cap must be >= 1");
  R2M_REQUIRE(depth >= 2, "ring depth must be >= 2");
  R2M_REQUIRE(chunk_cols >= 256, "chunk_cols must be >= 256");
  R2M_REQUIRE(resident_chunks >= 0, "resident_chunks must be >= 0");
  R2M_REQUIRE(score_mode >= R2M_SCORE_F16 && score_mode <= R2M_SCORE_SCALED, "bad score_mode");
  R2M_REQUIRE(score_mode != R2M_SCORE_SCALED || d_scaleB, "scaled scores need scaleB (device)");
  R2M_REQUIRE(score_mode != R2M_SCORE_SCALED || (reinterpret_cast<uintptr_t>(d_scaleB) & 15) == 0,
              "scaleB must be 16-byte aligned");
  int rc = r2m_device_check();
  if (rc) return rc;
  r2m_compact *c = new r2m_compact();
  c->hB = h_B;
  c->d_scaleB = d_scaleB;
  c->rdim = rdim;
  c->N = N;
  c->k = k;
  c->rows_cap = rows_cap;
  c->score_mode = score_mode;
  c->depth = depth;
  // chunks of near-equal size with starts on multiples of 4 columns (16-byte
  // aligned scale slices); with two or more chunks each holds at least
  // chunk_cols / 2 - 4 >= 124 >= k columns
  const int64_t nch = (N + chunk_cols - 1) / chunk_cols;
  for (int64_t i = 0; i < nch; ++i) c->lo.push_back(i == 0 ? 0 : (i * N / nch) & ~(int64_t)3);
  for (int64_t i = 0; i < nch; ++i) {
    c->wi.push_back((i + 1 < nch ? c->lo[i + 1] : N) - c->lo[i]);
    c->cap = std::max(c->cap, c->wi.back());
  }
  cudaError_t e;
  c->resident = (int)std::min<int64_t>(resident_chunks, nch);
  const int64_t rest = nch - c->resident;
  const int nslots = c->resident + (int)std::min<int64_t>(depth, rest);
  for (int b = 0; b < nslots; ++b) {
    uint8_t *p = nullptr;
    if ((e = cudaMalloc(&p, (size_t)c->cap * rdim)) != cudaSuccess) {
      destroy(c);
      return fail(R2M_ENOMEM, "ring slot allocation failed");
    }
    c->slot.push_back(p);
    c->holds.push_back(-1);
    c->used.push_back(false);
    cudaEvent_t a, d;
    if ((e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming)) != cudaSuccess) {
      destroy(c);
      return cuda_fail(e, "cudaEventCreate");
    }
    c->ev_h2d.push_back(a);
    if ((e = cudaEventCreateWithFlags(&d, cudaEventDisableTiming)) != cudaSuccess) {
      destroy(c);
      return cuda_fail(e, "cudaEventCreate");
    }
    c->ev_dev.push_back(d);
  }
  if ((e = cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking)) != cudaSuccess) {
    destroy(c);
    return cuda_fail(e, "cudaStreamCreate");
  }
  if ((e = cudaMalloc(&c->tmp_vals, (size_t)rows_cap * k * sizeof(float))) != cudaSuccess ||
      (e = cudaMalloc(&c->tmp_locs, (size_t)rows_cap * k * sizeof(int32_t))) != cudaSuccess ||
      (e = cudaMalloc(&c->ones, (size_t)rows_cap * sizeof(float))) != cudaSuccess) {
    destroy(c);
    return fail(R2M_ENOMEM, "compact engine buffers");
  }
  k_fill_f32<<<(rows_cap + 255) / 256, 256>>>(c->ones, 1.0f, rows_cap);
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess) {
    destroy(c);
    return cuda_fail(e, "compact engine init");
  }
  rc = r2m_engine_create(c->slot[0], score_mode == R2M_SCORE_SCALED ? d_scaleB : nullptr, rdim, c->cap, k,
                         rows_cap, score_mode, tune, &c->eng);
  if (rc) {
    destroy(c);
    return rc;
  }
  if (pin) {
    cudaPointerAttributes at{};
    const bool pinned = cudaPointerGetAttributes(&at, h_B) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (!pinned) {
      // page-lock the host index for full-speed DMA; read-only so that a
      // read-only file mapping qualifies.  Left pageable if refused.
      if (cudaHostRegister((void *)h_B, (size_t)N * rdim, cudaHostRegisterReadOnly) == cudaSuccess)
        c->registered = true;
      else
        cudaGetLastError();
    }
  }
  *out = c;
  return R2M_OK;
}

extern "C" int r2m_compact_destroy(r2m_compact *c) {
  if (!c) return R2M_OK;
  cudaDeviceSynchronize();
  destroy(c);
  return R2M_OK;
}

extern "C" int r2m_merge_topk_lists(const float *d_vals, const int32_t *d_locs, int lists, int nb, int k,
                                    int kout, float *d_out_vals, int32_t *d_out_locs, r2m_stream_t stream) {
  R2M_REQUIRE(lists >= 1 && lists <= 32, "lists must be in 1..32");
  R2M_REQUIRE(k >= 1 && kout >= 1 && kout <= lists * k, "need k >= 1 and 1 <= kout <= lists * k");
  R2M_REQUIRE(nb >= 0, "nb must be >= 0");
  if (nb == 0) return R2M_OK;
  R2M_REQUIRE(d_vals && d_locs && d_out_vals && d_out_locs, "null pointer");
  const int warps = 8;
  k_merge_lists<<<(nb + warps - 1) / warps, 32 * warps, 0, as_stream(stream)>>>(d_vals, d_locs, lists, nb, k, kout,
                                                                                 d_out_vals, d_out_locs);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}

extern "C" int64_t r2m_compact_chunks(const r2m_compact *c) { return c ? (int64_t)c->lo.size() : 0; }

extern "C" int r2m_compact_is_pinned(const r2m_compact *c) { return c && c->registered ? 1 : 0; }

extern "C" int64_t r2m_compact_resident_chunks(const r2m_compact *c) { return c ? c->resident : 0; }

extern "C" int r2m_compact_batch_gemm_topk(r2m_compact *c, const uint8_t *d_A, const float *d_scaleA, int nb,
                                           float *d_vals, int32_t *d_locs, r2m_stream_t stream) {
  R2M_REQUIRE(c != nullptr, "engine is null");
  R2M_REQUIRE(nb >= 0 && nb <= c->rows_cap, "nb must be in 0..rows_cap");
  if (nb == 0) return R2M_OK;
  R2M_REQUIRE(d_A && d_vals && d_locs, "null pointer");
  const bool scaled = c->score_mode == R2M_SCORE_SCALED;
  R2M_REQUIRE(!scaled || d_scaleA, "scaled scores need scaleA");
  cudaStream_t st = as_stream(stream);
  const int64_t nch = (int64_t)c->lo.size();
  const int R = c->resident;
  const int nring = (int)c->slot.size() - R;
  const bool all_fixed = nch - R <= nring;  // the streamed chunks fit their own slots too
  for (int64_t i = 0; i < nch; ++i) {
    const bool fixed = i < R || all_fixed;
    const int b = fixed ? (int)i : R + (int)(c->next++ % nring);
    if (c->holds[b] != i) {
      if (c->used[b]) R2M_CUDA(cudaStreamWaitEvent(c->h2d, c->ev_dev[b], 0));
      R2M_CUDA(cudaMemcpyAsync(c->slot[b], c->hB + (size_t)c->lo[i] * c->rdim, (size_t)c->wi[i] * c->rdim,
                               cudaMemcpyHostToDevice, c->h2d));
      R2M_CUDA(cudaEventRecord(c->ev_h2d[b], c->h2d));
      c->holds[b] = fixed ? i : -1;  // a ring slot's content is not reused
    }
    R2M_CUDA(cudaStreamWaitEvent(st, c->ev_h2d[b], 0));
    int rc = engine_rebind(c->eng, c->slot[b], scaled ? c->d_scaleB + c->lo[i] : nullptr, c->wi[i]);
    if (rc) return rc;
    float *ov = i == 0 ? d_vals : c->tmp_vals;
    int32_t *ol = i == 0 ? d_locs : c->tmp_locs;
    rc = r2m_batch_gemm_topk(c->eng, d_A, scaled ? c->ones : nullptr, nb, ov, ol, stream);
    if (rc) return rc;
    if (i > 0) {
      k_merge_running<<<(nb + 127) / 128, 128, 0, st>>>(d_vals, d_locs, c->tmp_vals, c->tmp_locs, nb, c->k,
                                                        c->lo[i]);
      R2M_CUDA(cudaGetLastError());
    }
    R2M_CUDA(cudaEventRecord(c->ev_dev[b], st));
    c->used[b] = true;
  }
  if (scaled) {
    const int64_t n = (int64_t)nb * c->k;
    k_scale_rows<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(d_vals, d_scaleA, nb, c->k);
    R2M_CUDA(cudaGetLastError());
  }
  return R2M_OK;
}
