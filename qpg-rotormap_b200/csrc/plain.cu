// plain.cu -- the plain batch path: the reference engine's structure on the
// B200, kept as the throughput / recall reference for the fused kernel.
//
// batch_gemm_topk! (RotorMap/search/engine_fp8.jl:399-437): for every chunk of
// w index columns, a cuBLASLt fp8 GEMM writes the (rows x w) fp16 score chunk
// to HBM (fp8_lt.jl:128-168: e4m3 x e4m3, fp32 compute, fp16 D, A "T" /
// B "N"), and a segmented per-row top-k merges the chunk into the running
// top-k (gemm/topk_kernels.jl:213-347).  Two C buffers, a GEMM stream and a
// top-k stream with event pairs double-buffer the loop exactly like the
// reference.  cuBLASLt is a closed library and is only called (dlopen).
//
// The top-k kernel restates seg_rowtopk_merge_kernel!'s algorithm and tie
// rules: PS threads per row each keep a K-reservoir of their column segment
// (strict `v > threshold`, replace the first minimum), insertion-sort it
// descending (stable), and the block's first warp merges the segment heads
// against the running list (the running entry wins ties, then the lowest
// segment); ids are 1-based, 0 = empty with value -Inf.
#include <cublasLt.h>
#include <dlfcn.h>

#include <mutex>

#include "common.cuh"
#include "lt_api.cuh"

namespace r2m {

// ------------------------------------------------------------- cuBLASLt

int lt_api(LtApi **out) {
  static std::mutex mu;
  static LtApi api;
  static bool ok = false;
  std::lock_guard<std::mutex> lk(mu);
  if (!ok) {
    const char *names[] = {"libcublasLt.so.12", "libcublasLt.so", "/usr/local/cuda/lib64/libcublasLt.so.12"};
    for (const char *n : names)
      if ((api.so = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
    if (!api.so) return fail(R2M_ESTATE, "plain path: libcublasLt.so.12 could not be loaded");
#define R2M_SYM(field, name)                                                        \
  api.field = reinterpret_cast<decltype(api.field)>(dlsym(api.so, #name));          \
  if (!api.field) return fail(R2M_ESTATE, "plain path: cuBLASLt lacks " #name);
    R2M_SYM(create, cublasLtCreate)
    R2M_SYM(destroy, cublasLtDestroy)
    R2M_SYM(desc_create, cublasLtMatmulDescCreate)
    R2M_SYM(desc_destroy, cublasLtMatmulDescDestroy)
    R2M_SYM(desc_set, cublasLtMatmulDescSetAttribute)
    R2M_SYM(layout_create, cublasLtMatrixLayoutCreate)
    R2M_SYM(layout_destroy, cublasLtMatrixLayoutDestroy)
    R2M_SYM(pref_create, cublasLtMatmulPreferenceCreate)
    R2M_SYM(pref_destroy, cublasLtMatmulPreferenceDestroy)
    R2M_SYM(pref_set, cublasLtMatmulPreferenceSetAttribute)
    R2M_SYM(heuristic, cublasLtMatmulAlgoGetHeuristic)
    R2M_SYM(matmul, cublasLtMatmul)
#undef R2M_SYM
    ok = true;
  }
  *out = &api;
  return R2M_OK;
}

static int lt_fail(cublasStatus_t s, const char *what) {
  return fail(R2M_ECUDA, std::string("cuBLASLt ") + what + " failed (status " + std::to_string((int)s) + ")");
}
#define R2M_LT(call, what)                              \
  do {                                                  \
    cublasStatus_t s_ = (call);                         \
    if (s_ != CUBLAS_STATUS_SUCCESS) return lt_fail(s_, what); \
  } while (0)

// ------------------------------------------------------------- seg top-k

template <int K>
struct SegRes {
  float v[K];
  int l[K];
  float thr;
  int minpos;
  __device__ __forceinline__ void reset() {
#pragma unroll
    for (int i = 0; i < K; ++i) {
      v[i] = -INFINITY;
      l[i] = 0;
    }
    thr = -INFINITY;
    minpos = 0;
  }
  // replace the tracked minimum; the new minimum is the FIRST smallest
  __device__ __forceinline__ void insert(float x, int loc) {
#pragma unroll
    for (int i = 0; i < K; ++i)
      if (i == minpos) {
        v[i] = x;
        l[i] = loc;
      }
    float mv = v[0];
    int mp = 0;
#pragma unroll
    for (int i = 1; i < K; ++i) {
      bool less = v[i] < mv;
      mv = less ? v[i] : mv;
      mp = less ? i : mp;
    }
    thr = mv;
    minpos = mp;
  }
  // stable insertion sort, descending (`while lk[j-1] < v` moves)
  __device__ __forceinline__ void sort() {
#pragma unroll
    for (int i = 1; i < K; ++i) {
#pragma unroll
      for (int j = i; j > 0; --j) {
        bool mv = v[j - 1] < v[j];
        float a = v[j - 1], b = v[j];
        int la = l[j - 1], lb = l[j];
        v[j - 1] = mv ? b : a;
        v[j] = mv ? a : b;
        l[j - 1] = mv ? lb : la;
        l[j] = mv ? la : lb;
      }
    }
  }
};

// One block per 32 rows; thread (row mt, segment s0).  C is the chunk in
// column-major order (ldc = rows per column), wi columns, global column of
// chunk column 0 = offset; D_val / D_loc are (nb, K) row-major running lists.
template <int K, int PS>
__global__ void __launch_bounds__(32 * PS) k_seg_topk(const __half *__restrict__ C, long long ldc, int nb,
                                                    int wi, long long offset, float *Dv, int *Dl) {
  __shared__ float shv[PS][32][K];
  __shared__ int shi[PS][32][K];
  __shared__ short shp[PS][32];
  __shared__ float shrv[32][K];
  __shared__ int shri[32][K];
  const int tid = threadIdx.x;
  const int mt = tid & 31, s0 = tid >> 5;
  const int row = blockIdx.x * 32 + mt;
  const bool valid = row < nb;
  const int segw = (wi + PS - 1) / PS;
  const int seg_lo = s0 * segw;
  const int count = max(0, min(wi, (s0 + 1) * segw) - seg_lo);
  SegRes<K> R;
  R.reset();
  if (valid && count > 0) {
    const __half *col = C + (long long)seg_lo * ldc + row;
#pragma unroll 4
    for (int c = 0; c < count; ++c) {
      float x = __half2float(col[(long long)c * ldc]);
      if (x > R.thr) R.insert(x, c + 1);
    }
    R.sort();
  }
  if (valid) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      shv[s0][mt][j] = R.v[j];
      shi[s0][mt][j] = R.l[j];
    }
  }
  if (valid && tid < 32) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      shrv[mt][j] = Dv[(size_t)row * K + j];
      shri[mt][j] = Dl[(size_t)row * K + j];
    }
  }
  __syncthreads();
  if (valid && tid < 32) {
    for (int s = 0; s < PS; ++s) shp[s][mt] = 0;
    int pa = 0;
    for (int j = 0; j < K; ++j) {
      float va = pa < K ? shrv[mt][pa] : -INFINITY;
      float bv = -INFINITY;
      int bs = -1, bli = 0;
      for (int s = 0; s < PS; ++s) {
        int h = shp[s][mt];
        if (h < K) {
          float v = shv[s][mt][h];
          if (bv < v) {  // ties keep the lowest segment
            bv = v;
            bs = s;
            bli = shi[s][mt][h];
          }
        }
      }
      if (va >= bv) {  // the running list wins ties (or both are exhausted)
        Dv[(size_t)row * K + j] = va;
        Dl[(size_t)row * K + j] = pa < K ? shri[mt][pa] : 0;
        ++pa;
      } else {
        Dv[(size_t)row * K + j] = bv;
        Dl[(size_t)row * K + j] = bli == 0 ? 0 : (int)(offset + (long long)bs * segw + bli);
        shp[bs][mt] += 1;
      }
    }
  }
}

__global__ void k_fill_running(float *Dv, int *Dl, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    Dv[i] = -INFINITY;
    Dl[i] = 0;
  }
}

}  // namespace r2m

using namespace r2m;

struct r2m_plain_engine {
  const uint8_t *B;
  int rdim;
  long long N;
  int k, rows_cap, w, segs;
  __half *buf[2];
  void *ws;
  size_t ws_bytes;
  cudaStream_t sg, st;
  cudaEvent_t evg[2], evt[2], ev_in, ev_out;
  cublasLtHandle_t lt;
  cublasLtMatmulDesc_t desc;
  LtApi *api;
  // cached layouts/algos per (rows, width)
  int cached_rows;
  int cached_w[2];
  cublasLtMatrixLayout_t la, lb[2], lc[2];
  cublasLtMatmulAlgo_t algo[2];
  bool has_algo[2];
};

static int plain_layouts(r2m_plain_engine *e, int rows, int wi, int slot) {
  LtApi *a = e->api;
  if (e->cached_rows != rows) {
    if (e->la) a->layout_destroy(e->la);
    e->la = nullptr;
    R2M_LT(a->layout_create(&e->la, CUDA_R_8F_E4M3, e->rdim, rows, e->rdim), "layout A");
    for (int s = 0; s < 2; ++s) {
      if (e->lb[s]) a->layout_destroy(e->lb[s]);
      if (e->lc[s]) a->layout_destroy(e->lc[s]);
      e->lb[s] = e->lc[s] = nullptr;
      e->cached_w[s] = -1;
      e->has_algo[s] = false;
    }
    e->cached_rows = rows;
  }
  if (e->cached_w[slot] != wi) {
    if (e->lb[slot]) a->layout_destroy(e->lb[slot]);
    if (e->lc[slot]) a->layout_destroy(e->lc[slot]);
    R2M_LT(a->layout_create(&e->lb[slot], CUDA_R_8F_E4M3, e->rdim, wi, e->rdim), "layout B");
    R2M_LT(a->layout_create(&e->lc[slot], CUDA_R_16F, rows, wi, rows), "layout C");
    cublasLtMatmulPreference_t pref;
    R2M_LT(a->pref_create(&pref), "preference");
    uint64_t wsb = e->ws_bytes;
    a->pref_set(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES, &wsb, sizeof(wsb));
    cublasLtMatmulHeuristicResult_t res;
    int nres = 0;
    cublasStatus_t s = a->heuristic(e->lt, e->desc, e->la, e->lb[slot], e->lc[slot], e->lc[slot], pref, 1, &res, &nres);
    a->pref_destroy(pref);
    if (s != CUBLAS_STATUS_SUCCESS || nres == 0) return lt_fail(s, "algo heuristic (no fp8 algorithm)");
    e->algo[slot] = res.algo;
    e->has_algo[slot] = true;
    e->cached_w[slot] = wi;
  }
  return R2M_OK;
}

extern "C" int r2m_plain_engine_create(const uint8_t *d_B, int rdim, int64_t N, int k, int rows_cap, int w,
                                       int segs, r2m_plain_engine **out) {
  R2M_REQUIRE(out, "out is null");
  *out = nullptr;
  R2M_REQUIRE(d_B, "B is null");
  R2M_REQUIRE(rdim >= 16 && rdim % 16 == 0, "cuBLASLt fp8 needs K % 16 == 0");
  R2M_REQUIRE(k == 20, "the plain path is built for k = 20 (the reference default)");
  R2M_REQUIRE(segs == 8, "the plain path is built for segs = 8 (the reference default)");
  R2M_REQUIRE(rows_cap >= 1 && w >= k && w <= N, "need k <= w <= N and rows_cap >= 1");
  LtApi *api = nullptr;
  int rc = lt_api(&api);
  if (rc) return rc;
  r2m_plain_engine *e = new r2m_plain_engine();
  e->B = d_B;
  e->rdim = rdim;
  e->N = N;
  e->k = k;
  e->rows_cap = (rows_cap + 15) / 16 * 16;
  e->w = w;
  e->segs = segs;
  e->api = api;
  e->ws_bytes = 32u << 20;
  cudaError_t ce = cudaMalloc(&e->buf[0], (size_t)e->rows_cap * w * sizeof(__half));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->buf[1], (size_t)e->rows_cap * w * sizeof(__half));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->ws, e->ws_bytes);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->sg, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking);
  for (int i = 0; i < 2 && ce == cudaSuccess; ++i) {
    ce = cudaEventCreateWithFlags(&e->evg[i], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->evt[i], cudaEventDisableTiming);
  }
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_in, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming);
  if (ce != cudaSuccess) {
    delete e;
    return cuda_fail(ce, "plain engine allocation");
  }
  R2M_LT(api->create(&e->lt), "create");
  R2M_LT(api->desc_create(&e->desc, CUBLAS_COMPUTE_32F, CUDA_R_32F), "matmul desc");
  cublasOperation_t ta = CUBLAS_OP_T, tb = CUBLAS_OP_N;
  api->desc_set(e->desc, CUBLASLT_MATMUL_DESC_TRANSA, &ta, sizeof(ta));
  api->desc_set(e->desc, CUBLASLT_MATMUL_DESC_TRANSB, &tb, sizeof(tb));
  e->cached_rows = -1;
  *out = e;
  return R2M_OK;
}

extern "C" int r2m_plain_engine_destroy(r2m_plain_engine *e) {
  if (!e) return R2M_OK;
  cudaStreamSynchronize(e->sg);
  cudaStreamSynchronize(e->st);
  LtApi *a = e->api;
  if (e->la) a->layout_destroy(e->la);
  for (int s = 0; s < 2; ++s) {
    if (e->lb[s]) a->layout_destroy(e->lb[s]);
    if (e->lc[s]) a->layout_destroy(e->lc[s]);
    cudaEventDestroy(e->evg[s]);
    cudaEventDestroy(e->evt[s]);
  }
  a->desc_destroy(e->desc);
  a->destroy(e->lt);
  cudaEventDestroy(e->ev_in);
  cudaEventDestroy(e->ev_out);
  cudaStreamDestroy(e->sg);
  cudaStreamDestroy(e->st);
  cudaFree(e->buf[0]);
  cudaFree(e->buf[1]);
  cudaFree(e->ws);
  delete e;
  return R2M_OK;
}

extern "C" int r2m_plain_batch_gemm_topk(r2m_plain_engine *e, const uint8_t *d_A, int nb, float *d_vals,
                                         int32_t *d_locs, r2m_stream_t stream) {
  R2M_REQUIRE(e, "engine is null");
  R2M_REQUIRE(nb >= 0 && nb <= e->rows_cap, "nb must be in 0..rows_cap");
  if (nb == 0) return R2M_OK;
  R2M_REQUIRE(d_A && d_vals && d_locs, "null pointer");
  const int rows = (nb + 15) / 16 * 16;  // cuBLASLt fp8: rows multiple of 16 (padmul)
  cudaStream_t cs = as_stream(stream);
  LtApi *a = e->api;
  R2M_CUDA(cudaEventRecord(e->ev_in, cs));
  R2M_CUDA(cudaStreamWaitEvent(e->sg, e->ev_in, 0));
  R2M_CUDA(cudaStreamWaitEvent(e->st, e->ev_in, 0));
  k_fill_running<<<64, 256, 0, e->st>>>(d_vals, d_locs, (long long)nb * e->k);
  R2M_CUDA(cudaGetLastError());
  const float alpha = 1.0f, beta = 0.0f;
  const long long nchunks = (e->N + e->w - 1) / e->w;
  for (long long i = 0; i < nchunks; ++i) {
    const int b = (int)(i & 1);
    const long long lo = i * e->w;
    const int wi = (int)((e->N < lo + e->w ? e->N : lo + e->w) - lo);
    const int slot = wi == e->w ? 0 : 1;
    int rc = plain_layouts(e, rows, wi, slot);
    if (rc) return rc;
    if (i >= 2) R2M_CUDA(cudaStreamWaitEvent(e->sg, e->evt[b], 0));  // buffer b's top-k done
    R2M_LT(a->matmul(e->lt, e->desc, &alpha, d_A, e->la, e->B + lo * e->rdim, e->lb[slot], &beta, e->buf[b],
                     e->lc[slot], e->buf[b], e->lc[slot], &e->algo[slot], e->ws, e->ws_bytes, e->sg),
           "matmul");
    R2M_CUDA(cudaEventRecord(e->evg[b], e->sg));
    R2M_CUDA(cudaStreamWaitEvent(e->st, e->evg[b], 0));
    k_seg_topk<20, 8><<<(nb + 31) / 32, 32 * 8, 0, e->st>>>(e->buf[b], rows, nb, wi, lo, d_vals, d_locs);
    R2M_CUDA(cudaGetLastError());
    R2M_CUDA(cudaEventRecord(e->evt[b], e->st));
  }
  R2M_CUDA(cudaEventRecord(e->ev_out, e->st));
  R2M_CUDA(cudaStreamWaitEvent(cs, e->ev_out, 0));
  return R2M_OK;
}
