// common.cu -- host side of the C ABI plumbing: thread-local last error,
// cached device properties and the per-device error word that bounded
// device-side waits report through.
#include <mutex>
#include <string>

#include "common.cuh"

namespace r2m {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                 cudaGetErrorString(e) + ")";
  return R2M_ECUDA;
}

static const int kMaxDev = 64;
static std::mutex g_mu;
static int g_sm[kMaxDev];
static uint32_t *g_errword[kMaxDev];

int sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return 148;
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_sm[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    g_sm[dev] = n;
  }
  return g_sm[dev];
}

// Stream-ordered scratch comes from one library pool per device that keeps
// up to kPoolKeepBytes mapped across synchronisations (the default pool
// returns freed memory to the OS at every sync, so a call that allocates
// after a sync would otherwise map its scratch afresh each time).
static constexpr uint64_t kPoolKeepBytes = 1ull << 30;
static cudaMemPool_t g_pool[kMaxDev] = {};

cudaError_t pool_alloc(void **p, size_t bytes, cudaStream_t st) {
  *p = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaMallocAsync(p, bytes, st);
  cudaMemPool_t pool;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_pool[dev]) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      cudaMemPool_t np;
      if ((e = cudaMemPoolCreate(&np, &props)) != cudaSuccess) return e;
      uint64_t keep = kPoolKeepBytes;
      if ((e = cudaMemPoolSetAttribute(np, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
        cudaMemPoolDestroy(np);
        return e;
      }
      g_pool[dev] = np;
    }
    pool = g_pool[dev];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

int device_error_word(uint32_t **out) {
  int dev = 0;
  R2M_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDev) return fail(R2M_ESTATE, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_errword[dev] == nullptr) {
    uint32_t *p = nullptr;
    R2M_CUDA(cudaMalloc(&p, sizeof(uint32_t)));
    R2M_CUDA(cudaMemset(p, 0, sizeof(uint32_t)));
    R2M_CUDA(cudaDeviceSynchronize());
    g_errword[dev] = p;
  }
  *out = g_errword[dev];
  return R2M_OK;
}

int check_device_error(cudaStream_t stream, const char *what) {
  uint32_t *w = nullptr;
  int rc = device_error_word(&w);
  if (rc) return rc;
  uint32_t h = 0;
  R2M_CUDA(cudaMemcpyAsync(&h, w, sizeof(h), cudaMemcpyDeviceToHost, stream));
  R2M_CUDA(cudaStreamSynchronize(stream));
  if (h != 0) {
    R2M_CUDA(cudaMemsetAsync(w, 0, sizeof(uint32_t), stream));
    R2M_CUDA(cudaStreamSynchronize(stream));
    return fail(R2M_ETIMEOUT, std::string(what) + ": a bounded device wait gave up (code " +
                                  std::to_string(h) + "); the kernel aborted its work");
  }
  return R2M_OK;
}

// One CTA waits, through the same bounded wait the pipelined kernels use, on
// an mbarrier that nothing arrives on (or, with `arrive`, that its own thread
// completed first); a wait that gives up records its code in the device
// error word like a kernel's would.
__global__ void k_selftest_wait(long long limit, int arrive, uint32_t *err) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (arrive) mbar_arrive(&bar);
    if (!mbar_wait_bounded(&bar, 0, &abort_flag, limit)) atomicExch(err, kErrTimeoutSelfTest);
  }
  __syncthreads();
}

int launch_selftest_wait(long long limit, int arrive, uint32_t *err, cudaStream_t st) {
  k_selftest_wait<<<1, 32, 0, st>>>(limit, arrive ? 1 : 0, err);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}

}  // namespace r2m

extern "C" {

int r2m_selftest_bounded_wait(int64_t limit_cycles, int arrive, r2m_stream_t stream) {
  if (limit_cycles < 0 || limit_cycles > (int64_t)4000000000LL)
    return r2m::fail(R2M_EINVAL, "limit_cycles must be in 0..4e9");
  uint32_t *w = nullptr;
  int rc = r2m::device_error_word(&w);
  if (rc) return rc;
  r2m::k_selftest_wait<<<1, 32, 0, r2m::as_stream(stream)>>>((long long)limit_cycles, arrive ? 1 : 0, w);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}

const char *r2m_last_error(void) { return r2m::g_last_error.c_str(); }

int r2m_version(void) { return 10000; }

int r2m_check_device_error(r2m_stream_t stream) {
  return r2m::check_device_error(r2m::as_stream(stream), "r2m_check_device_error");
}

int r2m_device_check(void) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return r2m::cuda_fail(e, "cudaGetDevice");
  int major = 0;
  e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (e != cudaSuccess) return r2m::cuda_fail(e, "cudaDeviceGetAttribute");
  if (major != 10)
    return r2m::fail(R2M_ESTATE, "librotormap_b200 needs an sm_100 (B200) device, found cc " +
                                     std::to_string(major) + ".x");
  return R2M_OK;
}

}  // extern "C"
