// server.cpp -- the serving form behind the C ABI: a continuous-batching
// request loop over one fused engine.
//
// The reference maps one read file at a time: map.jl (RotorMap/tools/map.jl:
// 100-184) iterates rope_topk_stream_compact, whose batches are formed from
// that file alone and run synchronously per batch.  Here requests (packed
// read words of any count, or FASTA bytes) arrive at any time from any
// thread; one loop thread on the library's two streams
//   * admits requests in arrival order while their device state (words and
//     result lists) fits both the byte budget and the device's free memory
//     measured at that moment (cudaMemGetInfo plus what the stream-ordered
//     pool holds unused), and uploads their words on the copy stream;
//   * forms every GPU batch from segments of all admitted requests, so a
//     request that arrives while others run joins the next batch;
//   * per batch, on the compute stream: one encoder launch per segment, one
//     fused search, and a device copy of each segment's rows into its
//     request's result lists;
//   * downloads a request's results when its last rows are done.
// A read's result does not depend on the batch it lands in (the encoder and
// the fused top-k are deterministic per row and the top-k order is total).
// Cancelling a waiting request drops it; cancelling an admitted one stops
// scheduling its remaining rows, lets its rows already in flight finish and
// then frees its state -- other requests in the same batches are untouched.
// A failed CUDA call fails every unfinished request with that first error
// and closes the server to new requests (the reference's first-error-wins
// err_out teardown, RotorMap/encode/stream.jl:95-110).
#include <cuda_runtime.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "r2m.h"

namespace r2m {
int fail(int code, const std::string &msg);
}  // namespace r2m

namespace {

double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

bool is_pinned(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

struct Req {
  int64_t id = 0;
  int64_t n = 0;
  int state = R2M_REQ_QUEUED;
  bool cancel = false;
  std::string error;
  double t_arrival = 0, t_admit = 0, t_done = 0;
  // host side: caller-owned buffers, or owned here for FASTA requests
  const uint32_t *h_words = nullptr;
  float *h_vals = nullptr;
  int32_t *h_locs = nullptr;
  bool pinned_in = false, pinned_out = false;
  std::vector<uint32_t> own_words;
  std::vector<float> own_vals;
  std::vector<int32_t> own_locs;
  r2m_reads *reads = nullptr;  // FASTA requests: the parsed reads (headers)
  // device side
  void *d_mem = nullptr;
  size_t d_bytes = 0;
  uint32_t *d_words = nullptr;
  float *d_vals = nullptr;
  int32_t *d_locs = nullptr;
  cudaEvent_t uploaded = nullptr;
  int64_t scheduled = 0, completed = 0;
};

struct Seg {
  std::shared_ptr<Req> r;
  int64_t lo, n;
};

struct Batch {
  cudaEvent_t done;
  std::vector<Seg> segs;
};

struct Download {
  cudaEvent_t done;
  std::shared_ptr<Req> r;
};

}  // namespace

struct r2m_server {
  r2m_engine *eng = nullptr;
  int k = 0, rdim = 0, score_mode = 0, cap = 0;
  int fk = 0, s = 0, m = 0, c = 0, normalize = 0, W = 0;
  int64_t budget = 0, reserve = 0;
  int max_inflight = 2;
  int dev = 0;
  cudaStream_t comp = nullptr, copy = nullptr;
  uint8_t *a8 = nullptr;
  float *scaleA = nullptr, *norms = nullptr, *vals = nullptr;
  int32_t *locs = nullptr;
  std::mutex mu;
  std::condition_variable cv;    // wakes the loop
  std::condition_variable done_cv;  // wakes waiters
  std::thread th;
  bool stop = false;
  std::string failure;
  int64_t next_id = 1;
  std::unordered_map<int64_t, std::shared_ptr<Req>> reqs;
  std::deque<std::shared_ptr<Req>> waiting;
  std::vector<std::shared_ptr<Req>> active;
  std::deque<Batch> inflight;
  std::deque<Download> downloads;
  std::vector<cudaEvent_t> free_events;
  int64_t in_use = 0, peak_in_use = 0;
  r2m_server_stats st{};

  int64_t request_bytes(int64_t n) const { return n * ((int64_t)W * 4 + (int64_t)k * 8) + 512; }

  cudaEvent_t take_event() {
    if (!free_events.empty()) {
      cudaEvent_t e = free_events.back();
      free_events.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    return e;
  }
  void give_event(cudaEvent_t e) {
    if (e) free_events.push_back(e);
  }

  // first error wins: fail every unfinished request, refuse new ones
  void fail_all(const std::string &msg) {
    if (failure.empty()) failure = msg;
    auto fin = [&](const std::shared_ptr<Req> &r) {
      if (r->state == R2M_REQ_QUEUED || r->state == R2M_REQ_ACTIVE) {
        r->state = R2M_REQ_FAILED;
        r->error = failure;
        r->t_done = now_s();
        st.requests_failed++;
      }
    };
    for (auto &r : waiting) fin(r);
    for (auto &r : active) fin(r);
    for (auto &b : inflight)
      for (auto &sg : b.segs) fin(sg.r);
    for (auto &d : downloads) fin(d.r);
    waiting.clear();
    active.clear();
    done_cv.notify_all();
  }

  void release_device(Req &r) {
    if (r.d_mem) cudaFreeAsync(r.d_mem, copy);
    r.d_mem = nullptr;
    r.d_words = nullptr;
    r.d_vals = nullptr;
    r.d_locs = nullptr;
    if (r.uploaded) give_event(r.uploaded);
    r.uploaded = nullptr;
    in_use -= (int64_t)r.d_bytes;
    r.d_bytes = 0;
  }

  // device memory free now: the driver's count plus what the stream-ordered
  // pool holds without using
  int64_t free_bytes() {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return 0;
    int64_t f = (int64_t)fr;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t resv = 0, used = 0;
      if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &resv) == cudaSuccess &&
          cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && resv > used)
        f += (int64_t)(resv - used);
    }
    return f;
  }

  bool admit() {
    bool any = false;
    // cancelled requests leave the queue at once, wherever they wait
    for (auto it = waiting.begin(); it != waiting.end();) {
      if ((*it)->cancel) {
        (*it)->state = R2M_REQ_CANCELLED;
        (*it)->t_done = now_s();
        st.requests_cancelled++;
        it = waiting.erase(it);
        any = true;
      } else {
        ++it;
      }
    }
    if (any) done_cv.notify_all();
    while (!waiting.empty()) {
      std::shared_ptr<Req> r = waiting.front();
      if (r->cancel) {
        waiting.pop_front();
        r->state = R2M_REQ_CANCELLED;
        r->t_done = now_s();
        st.requests_cancelled++;
        done_cv.notify_all();
        any = true;
        continue;
      }
      const int64_t need = request_bytes(r->n);
      if (budget > 0 && in_use + need > budget) break;
      if (need > free_bytes() - reserve) {
        if (active.empty() && inflight.empty() && downloads.empty()) {
          // nothing will free memory: this request cannot be served
          waiting.pop_front();
          r->state = R2M_REQ_FAILED;
          r->error = "not enough free device memory for a request of " + std::to_string(r->n) + " reads";
          r->t_done = now_s();
          st.requests_failed++;
          done_cv.notify_all();
          any = true;
          continue;
        }
        break;
      }
      waiting.pop_front();
      cudaError_t e = cudaMallocAsync(&r->d_mem, (size_t)need, copy);
      if (e != cudaSuccess) {
        cudaGetLastError();
        r->d_mem = nullptr;
        if (active.empty() && inflight.empty() && downloads.empty()) {
          // nothing will free memory: fail it rather than wait forever
          r->state = R2M_REQ_FAILED;
          r->error = std::string("device allocation for the request failed: ") + cudaGetErrorString(e);
          r->t_done = now_s();
          st.requests_failed++;
          done_cv.notify_all();
          any = true;
          continue;
        }
        waiting.push_front(r);
        break;  // try again when memory frees up
      }
      r->d_bytes = (size_t)need;
      in_use += need;
      peak_in_use = std::max(peak_in_use, in_use);
      unsigned char *p = static_cast<unsigned char *>(r->d_mem);
      r->d_vals = reinterpret_cast<float *>(p);
      r->d_locs = reinterpret_cast<int32_t *>(p + ((r->n * k * 4 + 255) & ~(int64_t)255));
      r->d_words = reinterpret_cast<uint32_t *>(p + 2 * ((r->n * k * 4 + 255) & ~(int64_t)255));
      e = cudaMemcpyAsync(r->d_words, r->h_words, (size_t)r->n * W * 4, cudaMemcpyHostToDevice, copy);
      r->uploaded = take_event();
      if (e != cudaSuccess || !r->uploaded || cudaEventRecord(r->uploaded, copy) != cudaSuccess) {
        fail_all(std::string("serving: request upload failed: ") + cudaGetErrorString(e));
        return true;
      }
      r->state = R2M_REQ_ACTIVE;
      r->t_admit = now_s();
      active.push_back(r);
      any = true;
    }
    return any;
  }

  bool launch() {
    if ((int)inflight.size() >= max_inflight) return false;
    Batch b;
    int64_t off = 0;
    for (auto &r : active) {
      if (off >= cap) break;
      if (r->cancel) continue;
      const int64_t left = r->n - r->scheduled;
      if (left <= 0) continue;
      const int64_t take = std::min<int64_t>(left, cap - off);
      b.segs.push_back(Seg{r, r->scheduled, take});
      r->scheduled += take;
      off += take;
    }
    if (b.segs.empty()) return false;
    const int nb = (int)off;
    const int kind = score_mode == R2M_SCORE_SCALED ? R2M_OUT_E4M3_SCALED : R2M_OUT_E4M3;
    int rc = R2M_OK;
    int64_t o = 0;
    for (auto &sg : b.segs) {
      if (cudaStreamWaitEvent(comp, sg.r->uploaded, 0) != cudaSuccess) rc = R2M_ECUDA;
      if (!rc)
        rc = r2m_encode_frag_real_batch(a8 + o * rdim, kind, norms + o * m,
                                        kind == R2M_OUT_E4M3_SCALED ? scaleA + o : nullptr,
                                        sg.r->d_words + sg.lo * W, sg.n, fk, s, m, c, normalize, comp);
      o += sg.n;
      if (rc) break;
    }
    if (!rc)
      rc = r2m_batch_gemm_topk(eng, a8, score_mode == R2M_SCORE_SCALED ? scaleA : nullptr, nb, vals, locs, comp);
    o = 0;
    for (auto &sg : b.segs) {
      if (rc) break;
      if (cudaMemcpyAsync(sg.r->d_vals + sg.lo * k, vals + o * k, (size_t)sg.n * k * 4, cudaMemcpyDeviceToDevice,
                          comp) != cudaSuccess ||
          cudaMemcpyAsync(sg.r->d_locs + sg.lo * k, locs + o * k, (size_t)sg.n * k * 4, cudaMemcpyDeviceToDevice,
                          comp) != cudaSuccess)
        rc = R2M_ECUDA;
      o += sg.n;
    }
    b.done = take_event();
    if (rc || !b.done || cudaEventRecord(b.done, comp) != cudaSuccess) {
      const char *msg = r2m_last_error();
      fail_all(std::string("serving: batch launch failed: ") + (rc && msg ? msg : "event"));
      return true;
    }
    inflight.push_back(std::move(b));
    st.batches++;
    st.rows += nb;
    st.max_rows = std::max<int64_t>(st.max_rows, nb);
    return true;
  }

  bool retire() {
    bool any = false;
    while (!inflight.empty()) {
      cudaError_t q = cudaEventQuery(inflight.front().done);
      if (q == cudaErrorNotReady) break;
      if (q != cudaSuccess) {
        fail_all(std::string("serving: a batch failed: ") + cudaGetErrorString(q));
        return true;
      }
      Batch b = std::move(inflight.front());
      inflight.pop_front();
      give_event(b.done);
      any = true;
      for (auto &sg : b.segs) {
        Req &r = *sg.r;
        r.completed += sg.n;
        if (r.state != R2M_REQ_ACTIVE) continue;
        if (r.cancel && r.completed == r.scheduled) {  // its rows in flight are done: drop it
          r.state = R2M_REQ_CANCELLED;
          r.t_done = now_s();
          release_device(r);
          st.requests_cancelled++;
          done_cv.notify_all();
        } else if (!r.cancel && r.completed == r.n) {
          Download d{nullptr, sg.r};
          cudaError_t e1 = cudaMemcpyAsync(r.h_vals, r.d_vals, (size_t)r.n * k * 4, cudaMemcpyDeviceToHost, copy);
          cudaError_t e2 = cudaMemcpyAsync(r.h_locs, r.d_locs, (size_t)r.n * k * 4, cudaMemcpyDeviceToHost, copy);
          d.done = take_event();
          if (e1 != cudaSuccess || e2 != cudaSuccess || !d.done || cudaEventRecord(d.done, copy) != cudaSuccess) {
            fail_all("serving: result download failed");
            return true;
          }
          downloads.push_back(d);
        }
      }
    }
    // cancelled requests with nothing in flight
    for (auto &r : active) {
      if (r->cancel && r->state == R2M_REQ_ACTIVE && r->completed == r->scheduled) {
        r->state = R2M_REQ_CANCELLED;
        r->t_done = now_s();
        release_device(*r);
        st.requests_cancelled++;
        done_cv.notify_all();
        any = true;
      }
    }
    // finished, cancelled, or with every row done (a download may still run)
    active.erase(std::remove_if(active.begin(), active.end(),
                                [](const std::shared_ptr<Req> &r) {
                                  return r->state != R2M_REQ_ACTIVE || r->completed == r->n;
                                }),
                 active.end());
    while (!downloads.empty()) {
      cudaError_t q = cudaEventQuery(downloads.front().done);
      if (q == cudaErrorNotReady) break;
      if (q != cudaSuccess) {
        fail_all(std::string("serving: a download failed: ") + cudaGetErrorString(q));
        return true;
      }
      Download d = downloads.front();
      downloads.pop_front();
      give_event(d.done);
      Req &r = *d.r;
      if (r.state == R2M_REQ_ACTIVE) {
        r.state = R2M_REQ_DONE;
        r.t_done = now_s();
        st.requests_done++;
      }
      release_device(r);
      done_cv.notify_all();
      any = true;
    }
    return any;
  }

  bool busy() const { return !waiting.empty() || !active.empty() || !inflight.empty() || !downloads.empty(); }

  void loop() {
    cudaSetDevice(dev);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      if (stop && !busy()) return;
      bool progressed = retire();
      if (failure.empty()) {
        progressed |= admit();
        progressed |= launch();
      }
      if (!failure.empty() && (!inflight.empty() || !downloads.empty())) {
        // after a failure: let the queued GPU work drain, then free it
        cudaStreamSynchronize(comp);
        cudaStreamSynchronize(copy);
        for (auto &b : inflight) give_event(b.done);
        for (auto &d : downloads) give_event(d.done);
        inflight.clear();
        downloads.clear();
        for (auto &kv : reqs)
          if (kv.second->d_mem) release_device(*kv.second);
        progressed = true;
      }
      if (progressed) continue;
      if (inflight.empty() && downloads.empty())
        cv.wait(lk);  // idle: a submit, cancel or shutdown wakes us
      else
        cv.wait_for(lk, std::chrono::microseconds(200));
    }
  }
};

namespace {

int submit_locked(r2m_server *srv, std::shared_ptr<Req> r, int64_t *id) {
  if (!srv->failure.empty()) return r2m::fail(R2M_ESTATE, "server failed earlier: " + srv->failure);
  if (srv->stop) return r2m::fail(R2M_ESTATE, "server is shutting down");
  const int64_t need = srv->request_bytes(r->n);
  if (srv->budget > 0 && need > srv->budget)
    return r2m::fail(R2M_ENOMEM, "request of " + std::to_string(r->n) + " reads needs " + std::to_string(need) +
                                     " B > the HBM budget " + std::to_string(srv->budget) + " B");
  r->id = srv->next_id++;
  if (r->t_arrival <= 0) r->t_arrival = now_s();
  srv->reqs[r->id] = r;
  if (r->n == 0) {
    r->state = R2M_REQ_DONE;
    r->t_done = now_s();
    srv->st.requests_done++;
  } else {
    srv->waiting.push_back(r);
    srv->cv.notify_all();
  }
  *id = r->id;
  return R2M_OK;
}

}  // namespace

extern "C" int r2m_server_create(r2m_engine *eng, int k, int s, int m, int c, int normalize, int64_t hbm_budget,
                                 int64_t hbm_reserve, int max_inflight, r2m_server **out) {
  if (!out || !eng) return r2m::fail(R2M_EINVAL, "null argument");
  *out = nullptr;
  std::unique_ptr<r2m_server> srv(new r2m_server());
  int rc = r2m_engine_info(eng, &srv->k, &srv->rdim, &srv->score_mode, &srv->cap, nullptr);
  if (rc) return rc;
  if (2 * m * (1 << (2 * c)) != srv->rdim)
    return r2m::fail(R2M_EINVAL, "encoder (m, c) does not match the engine's row width");
  if (k < s || s < 1 || normalize < 0 || normalize > 3) return r2m::fail(R2M_EINVAL, "bad encoder parameters");
  srv->eng = eng;
  srv->fk = k;
  srv->s = s;
  srv->m = m;
  srv->c = c;
  srv->normalize = normalize;
  srv->W = (k + 15) / 16;
  srv->budget = hbm_budget > 0 ? hbm_budget : 0;
  srv->reserve = hbm_reserve >= 0 ? hbm_reserve : 0;
  srv->max_inflight = max_inflight > 0 ? max_inflight : 2;
  if (cudaGetDevice(&srv->dev) != cudaSuccess) return r2m::fail(R2M_ECUDA, "cudaGetDevice failed");
  const size_t cap = (size_t)srv->cap;
  cudaError_t e = cudaStreamCreateWithFlags(&srv->comp, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&srv->copy, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&srv->a8, cap * srv->rdim);
  if (e == cudaSuccess) e = cudaMalloc(&srv->scaleA, cap * 4);
  if (e == cudaSuccess) e = cudaMalloc(&srv->norms, cap * m * 4);
  if (e == cudaSuccess) e = cudaMalloc(&srv->vals, cap * srv->k * 4);
  if (e == cudaSuccess) e = cudaMalloc(&srv->locs, cap * srv->k * 4);
  if (e == cudaSuccess) e = cudaMemset(srv->a8, 0, cap * srv->rdim);
  if (e != cudaSuccess) {
    cudaFree(srv->a8);
    cudaFree(srv->scaleA);
    cudaFree(srv->norms);
    cudaFree(srv->vals);
    cudaFree(srv->locs);
    if (srv->comp) cudaStreamDestroy(srv->comp);
    if (srv->copy) cudaStreamDestroy(srv->copy);
    return r2m::fail(R2M_ENOMEM, std::string("server buffers: ") + cudaGetErrorString(e));
  }
  srv->th = std::thread([p = srv.get()] { p->loop(); });
  *out = srv.release();
  return R2M_OK;
}

extern "C" int r2m_server_submit(r2m_server *srv, const uint32_t *h_words, int64_t n, float *h_vals,
                                 int32_t *h_locs, double t_arrival, int64_t *id) {
  if (!srv || !id) return r2m::fail(R2M_EINVAL, "null argument");
  if (n < 0) return r2m::fail(R2M_EINVAL, "n must be >= 0");
  if (n > 0 && (!h_words || !h_vals || !h_locs)) return r2m::fail(R2M_EINVAL, "null buffer");
  auto r = std::make_shared<Req>();
  r->n = n;
  r->h_words = h_words;
  r->h_vals = h_vals;
  r->h_locs = h_locs;
  r->t_arrival = t_arrival;
  r->pinned_in = is_pinned(h_words);
  r->pinned_out = is_pinned(h_vals) && is_pinned(h_locs);
  std::lock_guard<std::mutex> lk(srv->mu);
  return submit_locked(srv, r, id);
}

extern "C" int r2m_server_submit_fasta(r2m_server *srv, const char *data, size_t len, int nthreads,
                                       double t_arrival, int64_t *id, int64_t *n_reads) {
  if (!srv || !id) return r2m::fail(R2M_EINVAL, "null argument");
  if (!data && len) return r2m::fail(R2M_EINVAL, "data is null");
  size_t i = 0;
  while (i < len && (data[i] == '\n' || data[i] == '\r' || data[i] == ' ' || data[i] == '\t')) ++i;
  if (i == len) return r2m::fail(R2M_EIO, "malformed FASTA request: no record");
  if (data[i] != '>') return r2m::fail(R2M_EIO, "malformed FASTA request: data before the first '>' header");
  r2m_reads *reads = nullptr;
  int rc = r2m_fasta_reads(data, len, srv->fk, nthreads > 0 ? nthreads : 1, &reads);
  if (rc) return rc;
  const int64_t n = r2m_reads_count(reads);
  if (n == 0) {
    r2m_reads_free(reads);
    return r2m::fail(R2M_EIO, "malformed FASTA request: no record has " + std::to_string(srv->fk) + " bases");
  }
  auto r = std::make_shared<Req>();
  r->n = n;
  r->reads = reads;
  r->h_words = r2m_reads_words(reads);
  r->own_vals.resize((size_t)n * srv->k);
  r->own_locs.resize((size_t)n * srv->k);
  r->h_vals = r->own_vals.data();
  r->h_locs = r->own_locs.data();
  r->t_arrival = t_arrival;
  std::lock_guard<std::mutex> lk(srv->mu);
  rc = submit_locked(srv, r, id);
  if (rc) {
    r2m_reads_free(reads);
    r->reads = nullptr;
    return rc;
  }
  if (n_reads) *n_reads = n;
  return R2M_OK;
}

static std::shared_ptr<Req> find_req(r2m_server *srv, int64_t id) {
  auto it = srv->reqs.find(id);
  return it == srv->reqs.end() ? nullptr : it->second;
}

extern "C" int r2m_server_cancel(r2m_server *srv, int64_t id) {
  if (!srv) return r2m::fail(R2M_EINVAL, "server is null");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto r = find_req(srv, id);
  if (!r) return r2m::fail(R2M_EINVAL, "unknown request id " + std::to_string(id));
  if (r->state != R2M_REQ_QUEUED && r->state != R2M_REQ_ACTIVE)
    return r2m::fail(R2M_ESTATE, "request " + std::to_string(id) + " has already finished");
  r->cancel = true;
  srv->cv.notify_all();
  return R2M_OK;
}

extern "C" int r2m_server_wait(r2m_server *srv, int64_t id, double timeout_s, int *state) {
  if (!srv) return r2m::fail(R2M_EINVAL, "server is null");
  std::unique_lock<std::mutex> lk(srv->mu);
  auto r = find_req(srv, id);
  if (!r) return r2m::fail(R2M_EINVAL, "unknown request id " + std::to_string(id));
  auto fin = [&] { return r->state != R2M_REQ_QUEUED && r->state != R2M_REQ_ACTIVE; };
  if (timeout_s < 0) {
    srv->done_cv.wait(lk, fin);
  } else {
    srv->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), fin);
  }
  if (state) *state = r->state;
  if (!fin()) return r2m::fail(R2M_ETIMEOUT, "request " + std::to_string(id) + " not finished in time");
  return R2M_OK;
}

extern "C" int r2m_server_request(r2m_server *srv, int64_t id, int *state, int64_t *n, double *t_arrival,
                                  double *t_admit, double *t_done) {
  if (!srv) return r2m::fail(R2M_EINVAL, "server is null");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto r = find_req(srv, id);
  if (!r) return r2m::fail(R2M_EINVAL, "unknown request id " + std::to_string(id));
  if (state) *state = r->state;
  if (n) *n = r->n;
  if (t_arrival) *t_arrival = r->t_arrival;
  if (t_admit) *t_admit = r->t_admit;
  if (t_done) *t_done = r->t_done;
  return R2M_OK;
}

extern "C" const char *r2m_server_request_error(r2m_server *srv, int64_t id) {
  if (!srv) return "";
  std::lock_guard<std::mutex> lk(srv->mu);
  auto r = find_req(srv, id);
  return r ? r->error.c_str() : "";
}

extern "C" int r2m_server_copy_result(r2m_server *srv, int64_t id, float *h_vals, int32_t *h_locs) {
  if (!srv) return r2m::fail(R2M_EINVAL, "server is null");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto r = find_req(srv, id);
  if (!r) return r2m::fail(R2M_EINVAL, "unknown request id " + std::to_string(id));
  if (r->state == R2M_REQ_FAILED) return r2m::fail(R2M_ECUDA, "request failed: " + r->error);
  if (r->state == R2M_REQ_CANCELLED) return r2m::fail(R2M_ESTATE, "request was cancelled");
  if (r->state != R2M_REQ_DONE) return r2m::fail(R2M_ESTATE, "request has not finished");
  const size_t cnt = (size_t)r->n * srv->k;
  if (cnt && h_vals && h_vals != r->h_vals) memcpy(h_vals, r->h_vals, cnt * 4);
  if (cnt && h_locs && h_locs != r->h_locs) memcpy(h_locs, r->h_locs, cnt * 4);
  return R2M_OK;
}

extern "C" const r2m_reads *r2m_server_reads(r2m_server *srv, int64_t id) {
  if (!srv) return nullptr;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto r = find_req(srv, id);
  return r ? r->reads : nullptr;
}

extern "C" int r2m_server_release(r2m_server *srv, int64_t id) {
  if (!srv) return r2m::fail(R2M_EINVAL, "server is null");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) return r2m::fail(R2M_EINVAL, "unknown request id " + std::to_string(id));
  auto r = it->second;
  if (r->state == R2M_REQ_QUEUED || r->state == R2M_REQ_ACTIVE)
    return r2m::fail(R2M_ESTATE, "request " + std::to_string(id) + " is still running: cancel it first");
  if (r->reads) r2m_reads_free(r->reads);
  r->reads = nullptr;
  srv->reqs.erase(it);
  return R2M_OK;
}

extern "C" int r2m_server_get_stats(r2m_server *srv, r2m_server_stats *out) {
  if (!srv || !out) return r2m::fail(R2M_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(srv->mu);
  *out = srv->st;
  out->in_use_bytes = srv->in_use;
  out->peak_in_use_bytes = srv->peak_in_use;
  out->queued = (int64_t)srv->waiting.size();
  int64_t act = 0;  // admitted and unfinished (rows in flight or results downloading)
  for (auto &kv : srv->reqs) act += kv.second->state == R2M_REQ_ACTIVE;
  out->active = act;
  return R2M_OK;
}

extern "C" int64_t r2m_server_request_bytes(const r2m_server *srv, int64_t n) {
  return srv ? srv->request_bytes(n) : -1;
}

extern "C" int r2m_server_destroy(r2m_server *srv, int cancel_pending) {
  if (!srv) return R2M_OK;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    if (cancel_pending) {
      for (auto &r : srv->waiting) r->cancel = true;
      for (auto &r : srv->active) r->cancel = true;
    }
    srv->stop = true;
    srv->cv.notify_all();
  }
  if (srv->th.joinable()) srv->th.join();
  cudaStreamSynchronize(srv->comp);
  cudaStreamSynchronize(srv->copy);
  const std::string failure = srv->failure;
  for (auto &kv : srv->reqs) {
    if (kv.second->reads) r2m_reads_free(kv.second->reads);
    kv.second->reads = nullptr;
  }
  for (cudaEvent_t e : srv->free_events) cudaEventDestroy(e);
  cudaFree(srv->a8);
  cudaFree(srv->scaleA);
  cudaFree(srv->norms);
  cudaFree(srv->vals);
  cudaFree(srv->locs);
  cudaStreamDestroy(srv->comp);
  cudaStreamDestroy(srv->copy);
  delete srv;
  if (!failure.empty()) return r2m::fail(R2M_ECUDA, "server failed: " + failure);
  return R2M_OK;
}
