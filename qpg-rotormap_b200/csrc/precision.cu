// precision.cu -- the FP64 sampled-row check of the precision form.
//
// For a sample of reads it computes the exact (fp64) top-k over ALL index
// columns and the fp64 score of any given candidate lists, so the fp8 bulk
// scores and the fp32 rescored top-k can be stated against it (score error,
// top-k recall).  Embeddings follow the golden fp64 encoder
// _ref_rope_frag / _ref_rope_frag_real (RotorMap/encode/reference.jl:37-105,
// normalize = 0): phasors cis(theta*p) in fp64, G-homopolymer bins zeroed,
// norm sqrt(sum |h|^2) + 1e-16.  Index columns are re-encoded on the fly from
// the packed genome (forward / reverse-complement window per column), chunk
// by chunk; the read x chunk scores come from a cuBLASLt fp64 GEMM (a plain
// library GEMM, called only) and feed this file's fp64 top-k merge.
#include <float.h>
#include <limits.h>

#include <string>

#include "common.cuh"
#include "lt_api.cuh"

namespace r2m {

struct P64 {
  int k, s, m, c, W, nw, nbin, rdim;
  uint32_t bmask, cbmask, csmerG;
  double theta[8];
};

static int make_p64(P64 &P, int k, int s, int m, int c) {
  R2M_REQUIRE(s >= 1 && s <= 16 && c >= 1 && c <= s && m >= 1 && m <= 8 && k >= s, "bad encoder parameters");
  R2M_REQUIRE(((long long)m << (2 * c)) <= 1024, "the fp64 check supports m*4^c <= 1024");
  P.k = k; P.s = s; P.m = m; P.c = c;
  P.W = (k + 15) / 16;
  P.nw = k - s + 1;
  P.nbin = m << (2 * c);
  P.rdim = 2 * P.nbin;
  P.bmask = s == 16 ? 0xFFFFFFFFu : ((1u << (2 * s)) - 1u);
  P.cbmask = (1u << (2 * c)) - 1u;
  uint32_t allones = 0;
  for (int i = 0; i < c; ++i) allones += 1u << (2 * i);
  P.csmerG = 2u * allones;
  for (int i = 0; i < 8; ++i) {
    double f = m == 1 ? 1.0 : 2.0 * i / (double)(m - 1) + 1.0;
    P.theta[i] = f * (2.0 * M_PI / (double)k);
  }
  return R2M_OK;
}

__global__ void k_phasor64(P64 P, double2 *t) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.m * P.nw) return;
  int idm = i / P.nw, p = i % P.nw;
  double a = P.theta[idm] * p;
  t[i] = make_double2(cos(a), sin(a));
}

constexpr int kWarps64 = 4;

struct Smem64 {
  double *hist;
  uint16_t *cs;
  uint32_t *w0, *w1;
};

__host__ __device__ __forceinline__ size_t smem64_per_warp(const P64 &P) {
  return (size_t)P.rdim * 8 + (((size_t)P.nw * 2 + 15) & ~(size_t)15) + 2 * (((size_t)P.W + 2) * 4 + 12);
}

__device__ __forceinline__ Smem64 carve64(const P64 &P, unsigned char *base, int warp) {
  unsigned char *p = base + smem64_per_warp(P) * warp;
  Smem64 s;
  s.hist = reinterpret_cast<double *>(p);
  p += (size_t)P.rdim * 8;
  s.cs = reinterpret_cast<uint16_t *>(p);
  p += ((size_t)P.nw * 2 + 15) & ~(size_t)15;
  s.w0 = reinterpret_cast<uint32_t *>(p);
  p += ((size_t)P.W + 2) * 4 + 12;
  s.w1 = reinterpret_cast<uint32_t *>(p);
  return s;
}

// Stage the k bases of a read (dnas != null) or of index column `col`.
__device__ const uint32_t *stage64(const P64 &P, Smem64 &sm, const uint32_t *dnas, long long row,
                                   const uint32_t *genome, const int64_t *col_pos, const uint8_t *strand) {
  const int lane = threadIdx.x & 31;
  if (dnas) {
    for (int t = lane; t < P.W; t += 32) sm.w0[t] = dnas[row * P.W + t];
    if (lane == 0) sm.w0[P.W] = 0u;
    __syncwarp();
    return sm.w0;
  }
  const int64_t pos = col_pos[row];
  const int64_t q = pos >> 4;
  const uint32_t sh = (uint32_t)(pos & 15) << 1;
  const int r = P.k & 15;
  const uint32_t tail = r == 0 ? 0xFFFFFFFFu : ((1u << (2 * r)) - 1u);
  for (int t = lane; t < P.W; t += 32) {
    uint32_t a = genome[q + t], b = genome[q + t + 1];
    uint32_t v = sh == 0 ? a : ((a >> sh) | (b << (32u - sh)));
    sm.w0[t] = t == P.W - 1 ? (v & tail) : v;
  }
  if (lane == 0) sm.w0[P.W] = 0u;
  __syncwarp();
  if (!strand[row]) return sm.w0;
  for (int t = lane; t < P.W; t += 32) {
    uint32_t w = 0;
    for (int b = 0; b < 16; ++b) {
      int x = 16 * t + b;
      if (x < P.k) {
        int y = P.k - 1 - x;
        w |= (3u - ((sm.w0[y >> 4] >> (2 * (y & 15))) & 3u)) << (2 * b);
      }
    }
    sm.w1[t] = w;
  }
  if (lane == 0) sm.w1[P.W] = 0u;
  __syncwarp();
  return sm.w1;
}

// fp64 histogram (interleaved re/im), normalised in place (mode 0).
__device__ void hist64(const P64 &P, const double2 *table, Smem64 &sm, const uint32_t *words) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  for (int i = lane; i < P.rdim; i += 32) sm.hist[i] = 0.0;
  for (int p = lane; p < P.nw; p += 32) {
    int wo = p >> 4;
    uint32_t sh = (uint32_t)(p & 15) << 1;
    uint32_t v = sh == 0 ? words[wo] : ((words[wo] >> sh) | (words[wo + 1] << (32u - sh)));
    uint32_t smer = v & P.bmask;
    uint32_t upper = (2 * P.c >= 32) ? 0u : (smer >> (2 * P.c));
    sm.cs[p] = (uint16_t)((smer & P.cbmask) ^ ((upper * 0x9E3779B1u) & P.cbmask));
  }
  __syncwarp();
  for (int b0 = 0; b0 < P.nw; b0 += 32) {
    int p = b0 + lane;
    bool act = p < P.nw;
    unsigned amask = __ballot_sync(FULL, act);
    if (act) {
      uint32_t cb = sm.cs[p];
      unsigned grp = __match_any_sync(amask, cb);
      if (lane == __ffs(grp) - 1) {
        for (int idm = 0; idm < P.m; ++idm) {
          double *h = sm.hist + 2 * (cb * P.m + idm);
          double re = h[0], im = h[1];
          unsigned g = grp;
          while (g) {
            int j = __ffs(g) - 1;
            g &= g - 1;
            double2 ph = table[(size_t)idm * P.nw + b0 + j];
            re += ph.x;
            im += ph.y;
          }
          h[0] = re;
          h[1] = im;
        }
      }
    }
    __syncwarp();
  }
  if (lane < P.m) {
    double *h = sm.hist + 2 * (P.csmerG * P.m + lane);
    h[0] = 0.0;
    h[1] = 0.0;
  }
  __syncwarp();
  double acc = 0.0;
  for (int i = lane; i < P.rdim; i += 32) acc += sm.hist[i] * sm.hist[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
  const double nrm = sqrt(acc) + 1e-16;
  for (int i = lane; i < P.rdim; i += 32) sm.hist[i] /= nrm;
  __syncwarp();
}

// Dense fp64 rows (split [Re; Im] layout) of reads or of a column range.
__global__ void __launch_bounds__(32 * kWarps64) k_encode64(P64 P, const double2 *table, const uint32_t *dnas,
                                                          const uint32_t *genome, const int64_t *col_pos,
                                                          const uint8_t *strand, long long row0, long long n,
                                                          double *dest) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Smem64 sm = carve64(P, smem, warp);
  const long long nw = (long long)gridDim.x * kWarps64;
  for (long long i = (long long)blockIdx.x * kWarps64 + warp; i < n; i += nw) {
    const uint32_t *w = stage64(P, sm, dnas, row0 + i, genome, col_pos, strand);
    hist64(P, table, sm, w);
    double *out = dest + i * P.rdim;
    for (int b = lane; b < P.nbin; b += 32) {
      out[b] = sm.hist[2 * b];
      out[P.nbin + b] = sm.hist[2 * b + 1];
    }
    __syncwarp();
  }
}

// fp64 score of (sampled read, candidate column) pairs: one warp per pair.
__global__ void __launch_bounds__(32 * kWarps64) k_pair64(P64 P, const double2 *table, const double *A64, int S,
                                                        const int *cand, int kc, const uint32_t *genome,
                                                        const int64_t *col_pos, const uint8_t *strand,
                                                        long long N, double *out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  Smem64 sm = carve64(P, smem, warp);
  const long long total = (long long)S * kc;
  const long long nw = (long long)gridDim.x * kWarps64;
  for (long long i = (long long)blockIdx.x * kWarps64 + warp; i < total; i += nw) {
    const int s = (int)(i / kc);
    const int c1 = cand[i];
    double sc = -INFINITY;
    if (c1 >= 1 && c1 <= N) {
      const uint32_t *w = stage64(P, sm, nullptr, c1 - 1, genome, col_pos, strand);
      hist64(P, table, sm, w);
      const double *a = A64 + (size_t)s * P.rdim;
      double acc = 0.0;
      for (int b = lane; b < P.nbin; b += 32) acc += a[b] * sm.hist[2 * b] + a[P.nbin + b] * sm.hist[2 * b + 1];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
      sc = acc;
    }
    if (lane == 0) out[i] = sc;
    __syncwarp();
  }
}

// Merge a (S x nc) fp64 score chunk (row-major) into the running top-K of
// every row: one warp per row, per-lane sorted lists, k rounds of warp argmax.
template <int K>
__global__ void k_topk64(const double *sc, int S, int nc, long long col0, double *rv, int *rl) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= S) return;
  const unsigned FULL = 0xFFFFFFFFu;
  double v[K];
  long long c[K];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    v[i] = -INFINITY;
    c[i] = LLONG_MAX;
  }
  // lane 0 also carries the running list (it precedes every chunk column)
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < K; ++i) {
      v[i] = rv[(size_t)row * K + i];
      c[i] = rl[(size_t)row * K + i] == 0 ? LLONG_MAX : (long long)rl[(size_t)row * K + i] - 1;
    }
  const double *r = sc + (size_t)row * nc;
  for (int j = lane; j < nc; j += 32) {
    double x = r[j];
    long long col = col0 + j;
    if (x > v[K - 1] || (x == v[K - 1] && col < c[K - 1])) {
      int p = 0;
#pragma unroll
      for (int i = 0; i < K; ++i) p += (v[i] > x || (v[i] == x && c[i] < col)) ? 1 : 0;
#pragma unroll
      for (int i = K - 1; i > 0; --i) {
        bool shift = i > p, here = i == p;
        v[i] = shift ? v[i - 1] : (here ? x : v[i]);
        c[i] = shift ? c[i - 1] : (here ? col : c[i]);
      }
      if (p == 0) {
        v[0] = x;
        c[0] = col;
      }
    }
  }
  int h = 0;
  for (int t = 0; t < K; ++t) {
    double bv = h < K ? v[0] : -INFINITY;
    long long bc = h < K ? c[0] : LLONG_MAX;
#pragma unroll
    for (int i = 0; i < K; ++i)
      if (i == h) {
        bv = v[i];
        bc = c[i];
      }
    if (h >= K) {
      bv = -INFINITY;
      bc = LLONG_MAX;
    }
    double wv = bv;
    long long wc = bc;
    int wl = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(FULL, wv, o);
      long long oc = __shfl_xor_sync(FULL, wc, o);
      int ol = __shfl_xor_sync(FULL, wl, o);
      bool better = ov > wv || (ov == wv && (oc < wc || (oc == wc && ol < wl)));
      wv = better ? ov : wv;
      wc = better ? oc : wc;
      wl = better ? ol : wl;
    }
    if (lane == 0) {
      rv[(size_t)row * K + t] = wv;
      rl[(size_t)row * K + t] = wc == LLONG_MAX ? 0 : (int)(wc + 1);
    }
    if (lane == wl) ++h;
  }
}

__global__ void k_fill64(double *v, int *l, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    v[i] = -INFINITY;
    l[i] = 0;
  }
}

static int lt_check(cublasStatus_t s, const char *what) {
  if (s == CUBLAS_STATUS_SUCCESS) return R2M_OK;
  return fail(R2M_ECUDA, std::string("cuBLASLt ") + what + " failed (status " + std::to_string((int)s) + ")");
}

}  // namespace r2m

using namespace r2m;

extern "C" int r2m_check_fp64(const uint32_t *d_read_words, int S, const uint32_t *d_genome,
                              const int64_t *d_col_pos, const uint8_t *d_strand, int64_t N, int k, int s, int m,
                              int c, const int32_t *d_cand, int kc, double *d_cand_scores, double *d_vals,
                              int32_t *d_locs, r2m_stream_t stream) {
  P64 P;
  int rc = make_p64(P, k, s, m, c);
  if (rc) return rc;
  R2M_REQUIRE(S >= 1 && N >= 20, "need S >= 1 sampled reads and N >= 20 columns");
  R2M_REQUIRE(d_read_words && d_genome && d_col_pos && d_strand && d_vals && d_locs, "null pointer");
  R2M_REQUIRE(!d_cand || (kc >= 1 && d_cand_scores), "candidate lists need kc >= 1 and an output");
  LtApi *api = nullptr;
  if ((rc = lt_api(&api))) return rc;
  cudaStream_t st = as_stream(stream);
  const long long NC = 32768;
  const size_t smem = smem64_per_warp(P) * kWarps64;
  R2M_CUDA(cudaFuncSetAttribute(k_encode64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  R2M_CUDA(cudaFuncSetAttribute(k_pair64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  double2 *table = nullptr;
  double *A = nullptr, *Bc = nullptr, *Sc = nullptr;
  void *ws = nullptr;
  const size_t wsb = 32u << 20;
  cudaError_t ce = cudaMalloc(&table, (size_t)P.m * P.nw * sizeof(double2));
  if (ce == cudaSuccess) ce = cudaMalloc(&A, (size_t)S * P.rdim * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&Bc, (size_t)NC * P.rdim * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&Sc, (size_t)S * NC * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&ws, wsb);
  cublasLtHandle_t lt = nullptr;
  cublasLtMatmulDesc_t desc = nullptr;
  cublasLtMatrixLayout_t la = nullptr, lb = nullptr, lc = nullptr;
  auto cleanup = [&]() {
    cudaStreamSynchronize(st);
    if (la) api->layout_destroy(la);
    if (lb) api->layout_destroy(lb);
    if (lc) api->layout_destroy(lc);
    if (desc) api->desc_destroy(desc);
    if (lt) api->destroy(lt);
    cudaFree(table); cudaFree(A); cudaFree(Bc); cudaFree(Sc); cudaFree(ws);
  };
  if (ce != cudaSuccess) {
    cleanup();
    return fail(R2M_ENOMEM, "fp64 check workspace allocation failed");
  }
  const int grid_enc = 4 * sm_count();
  k_phasor64<<<(P.m * P.nw + 127) / 128, 128, 0, st>>>(P, table);
  k_encode64<<<grid_enc, 32 * kWarps64, smem, st>>>(P, table, d_read_words, nullptr, nullptr, nullptr, 0, S, A);
  k_fill64<<<64, 256, 0, st>>>(d_vals, d_locs, (long long)S * 20);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    cleanup();
    return cuda_fail(ce, "fp64 check encode");
  }
  if (d_cand) {
    k_pair64<<<grid_enc, 32 * kWarps64, smem, st>>>(P, table, A, S, d_cand, kc, d_genome, d_col_pos, d_strand, N,
                                                  d_cand_scores);
  }
  if ((rc = lt_check(api->create(&lt), "create"))) { cleanup(); return rc; }
  if ((rc = lt_check(api->desc_create(&desc, CUBLAS_COMPUTE_64F, CUDA_R_64F), "desc"))) { cleanup(); return rc; }
  cublasOperation_t ta = CUBLAS_OP_T, tb = CUBLAS_OP_N;
  api->desc_set(desc, CUBLASLT_MATMUL_DESC_TRANSA, &ta, sizeof(ta));
  api->desc_set(desc, CUBLASLT_MATMUL_DESC_TRANSB, &tb, sizeof(tb));
  if ((rc = lt_check(api->layout_create(&lb, CUDA_R_64F, P.rdim, S, P.rdim), "layout reads"))) { cleanup(); return rc; }
  const double one = 1.0, zero = 0.0;
  long long cur_w = -1;
  cublasLtMatmulAlgo_t algo;
  for (long long c0 = 0; c0 < N; c0 += NC) {
    const long long nc = (N - c0) < NC ? (N - c0) : NC;
    k_encode64<<<grid_enc, 32 * kWarps64, smem, st>>>(P, table, nullptr, d_genome, d_col_pos, d_strand, c0, nc, Bc);
    if (nc != cur_w) {
      if (la) api->layout_destroy(la);
      if (lc) api->layout_destroy(lc);
      la = lc = nullptr;
      if ((rc = lt_check(api->layout_create(&la, CUDA_R_64F, P.rdim, nc, P.rdim), "layout cols"))) { cleanup(); return rc; }
      if ((rc = lt_check(api->layout_create(&lc, CUDA_R_64F, nc, S, nc), "layout scores"))) { cleanup(); return rc; }
      cublasLtMatmulPreference_t pref;
      api->pref_create(&pref);
      uint64_t w64 = wsb;
      api->pref_set(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES, &w64, sizeof(w64));
      cublasLtMatmulHeuristicResult_t res;
      int nres = 0;
      cublasStatus_t hs = api->heuristic(lt, desc, la, lb, lc, lc, pref, 1, &res, &nres);
      api->pref_destroy(pref);
      if (hs != CUBLAS_STATUS_SUCCESS || nres == 0) { cleanup(); return fail(R2M_ECUDA, "no fp64 GEMM algorithm"); }
      algo = res.algo;
      cur_w = nc;
    }
    if ((rc = lt_check(api->matmul(lt, desc, &one, Bc, la, A, lb, &zero, Sc, lc, Sc, lc, &algo, ws, wsb, st),
                       "fp64 matmul"))) { cleanup(); return rc; }
    k_topk64<20><<<(S + 7) / 8, 256, 0, st>>>(Sc, S, (int)nc, c0, d_vals, d_locs);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) { cleanup(); return cuda_fail(ce, "fp64 check chunk"); }
  }
  cleanup();
  return R2M_OK;
}
