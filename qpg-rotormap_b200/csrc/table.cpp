// table.cpp -- host writer of the mapping table of RotorMap/tools/map.jl:
// 141-151: per read and per top-k hit one line
//   <read header without its leading '>'> <+|-> <score> <window start - 1> <record name>
// where + / - is the column's strand, the score is Julia's string(::Float32)
// and the record name is the first token of the record's header.
//
// Julia prints a Float32 with its shortest round-trip digits, in decimal
// form when the first significant digit's decimal exponent e satisfies
// -5 < e < 6 ("0.0001", "123456.0") and as d.ddd e<exp> otherwise ("1.0e-5",
// "1.2345678e8"); NaN / Inf / -Inf and 0.0 / -0.0 are literal.  The shortest
// digits come from std::to_chars, which returns the shortest string that
// reads back to the same float (ties resolved to the closest).
//
// Rows are split into blocks; each thread writes its block's lines through a
// raw pointer into its own buffer (sized by an upper bound per line), then
// the threads copy their blocks side by side into the output buffer.  The
// buffers come from a small pool that keeps them mapped between calls, so a
// batch does not pay page faults on 100 MB of fresh memory every time.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <charconv>
#include <cmath>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "r2m.h"

namespace r2m {
int fail(int code, const std::string &msg);
}  // namespace r2m

namespace {

struct Buf {
  char *p = nullptr;
  size_t cap = 0;
};

// Free buffers kept for reuse: at most kPoolBufs of them and kPoolBytes in all.
constexpr size_t kPoolBufs = 64;
constexpr size_t kPoolBytes = size_t(1) << 30;
std::mutex g_pool_mu;
std::vector<Buf> g_pool;

// A buffer of at least `need` bytes: the smallest pooled one that fits, else
// a new one (nullptr p on allocation failure).
Buf take_buf(size_t need) {
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    size_t best = g_pool.size();
    for (size_t i = 0; i < g_pool.size(); ++i)
      if (g_pool[i].cap >= need && (best == g_pool.size() || g_pool[i].cap < g_pool[best].cap)) best = i;
    if (best < g_pool.size()) {
      Buf b = g_pool[best];
      g_pool.erase(g_pool.begin() + (long)best);
      return b;
    }
  }
  Buf b;
  b.p = static_cast<char *>(malloc(need ? need : 1));
  b.cap = b.p ? need : 0;
  return b;
}

void give_buf(Buf b) {
  if (!b.p) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  size_t tot = b.cap;
  for (auto &x : g_pool) tot += x.cap;
  if (g_pool.size() < kPoolBufs && tot <= kPoolBytes) {
    g_pool.push_back(b);
    return;
  }
  free(b.p);
}

}  // namespace

struct r2m_text {
  Buf b;
  size_t n = 0;
};

namespace {

// Julia's string(::Float32) into out (at least 32 bytes); returns the length.
int julia_f32(float x, char *out) {
  if (std::isnan(x)) {
    memcpy(out, "NaN", 3);
    return 3;
  }
  if (std::isinf(x)) {
    if (x > 0) {
      memcpy(out, "Inf", 3);
      return 3;
    }
    memcpy(out, "-Inf", 4);
    return 4;
  }
  if (x == 0.0f) {
    if (std::signbit(x)) {
      memcpy(out, "-0.0", 4);
      return 4;
    }
    memcpy(out, "0.0", 3);
    return 3;
  }
  char buf[48];
  auto r = std::to_chars(buf, buf + sizeof(buf), x, std::chars_format::scientific);
  // buf: [-]d[.ddd]e(+|-)xx
  const char *p = buf, *end = r.ptr;
  int n = 0;
  if (*p == '-') {
    out[n++] = '-';
    ++p;
  }
  char dig[16];
  int nd = 0;
  while (p < end && *p != 'e') {
    if (*p != '.') dig[nd++] = *p;
    ++p;
  }
  int e10 = 0;
  if (p < end && *p == 'e') {
    ++p;
    const bool neg = *p == '-';
    if (*p == '+' || *p == '-') ++p;
    while (p < end) e10 = 10 * e10 + (*p++ - '0');
    if (neg) e10 = -e10;
  }
  while (nd > 1 && dig[nd - 1] == '0') --nd;  // shortest digits carry no trailing zero
  if (e10 > -5 && e10 < 6) {
    if (e10 >= 0) {
      for (int i = 0; i <= e10; ++i) out[n++] = i < nd ? dig[i] : '0';
      out[n++] = '.';
      if (nd > e10 + 1)
        for (int i = e10 + 1; i < nd; ++i) out[n++] = dig[i];
      else
        out[n++] = '0';
    } else {
      out[n++] = '0';
      out[n++] = '.';
      for (int i = 0; i < -e10 - 1; ++i) out[n++] = '0';
      for (int i = 0; i < nd; ++i) out[n++] = dig[i];
    }
    return n;
  }
  out[n++] = dig[0];
  out[n++] = '.';
  if (nd > 1)
    for (int i = 1; i < nd; ++i) out[n++] = dig[i];
  else
    out[n++] = '0';
  out[n++] = 'e';
  auto q = std::to_chars(out + n, out + n + 8, e10);
  return (int)(q.ptr - out);
}

// Split a blob of '\n'-terminated strings into (offset, length) pairs.
bool split_lines(const char *blob, size_t len, int64_t want, std::vector<std::pair<size_t, size_t>> &out) {
  out.clear();
  size_t s = 0;
  for (size_t i = 0; i < len; ++i)
    if (blob[i] == '\n') {
      out.emplace_back(s, i - s);
      s = i + 1;
    }
  return s == len && (want < 0 || (int64_t)out.size() == want);
}

}  // namespace

extern "C" int r2m_format_f32(float x, char *out, size_t cap) {
  if (!out || cap < 32) return r2m::fail(R2M_EINVAL, "format buffer needs 32 bytes");
  int n = julia_f32(x, out);
  out[n] = 0;
  return n;
}

extern "C" int r2m_format_table(const float *vals, const int32_t *locs, int64_t nb, int k, const char *heads,
                                size_t heads_len, const uint8_t *strand, const int64_t *starts,
                                const int32_t *col_rec, int64_t ncols, const char *rec_names, size_t rec_names_len,
                                int nthreads, r2m_text **out) {
  if (!out) return r2m::fail(R2M_EINVAL, "out is null");
  *out = nullptr;
  if (nb < 0 || k < 1) return r2m::fail(R2M_EINVAL, "need nb >= 0 and k >= 1");
  if (nb > 0 && (!vals || !locs || !heads)) return r2m::fail(R2M_EINVAL, "null batch pointer");
  if (ncols < 1 || !strand || !starts || !col_rec) return r2m::fail(R2M_EINVAL, "null index column table");
  std::vector<std::pair<size_t, size_t>> hd, rn;
  if (!split_lines(heads, heads_len, nb, hd))
    return r2m::fail(R2M_EINVAL, "heads must hold nb '\\n'-terminated headers");
  if (!split_lines(rec_names, rec_names_len, -1, rn) || rn.empty())
    return r2m::fail(R2M_EINVAL, "rec_names must hold '\\n'-terminated record names");
  const int64_t nrec = (int64_t)rn.size();
  size_t max_rec = 0;
  for (auto &x : rn) max_rec = std::max(max_rec, x.second);
  if (nthreads < 1) nthreads = 1;
  const int64_t nblk = nb < 2048 ? 1 : std::min<int64_t>(nthreads, (nb + 1023) / 1024);
  // per line: header + " + " + score (<= 32) + ' ' + start (<= 20) + ' ' + record name + '\n'
  const size_t line_extra = 3 + 32 + 1 + 20 + 1 + max_rec + 1;
  std::vector<Buf> part((size_t)nblk);
  std::vector<size_t> used((size_t)nblk, 0);
  std::atomic<int> bad{0};  // 1 = location out of range, 2 = record id out of range, 3 = no memory,
                           // 4 = location -1 (rows of a search whose device wait gave up)
  auto format = [&](int64_t b) {
    const int64_t r0 = nb * b / nblk, r1 = nb * (b + 1) / nblk;
    size_t bound = 0;
    for (int64_t r = r0; r < r1; ++r) bound += (size_t)k * (hd[(size_t)r].second + line_extra);
    Buf buf = take_buf(bound);
    if (!buf.p) {
      bad = 3;
      return;
    }
    char *w = buf.p;
    for (int64_t r = r0; r < r1 && !bad.load(std::memory_order_relaxed); ++r) {
      const char *h = heads + hd[(size_t)r].first;
      size_t hl = hd[(size_t)r].second;
      if (hl && h[0] == '>') {
        ++h;
        --hl;
      }
      for (int j = 0; j < k; ++j) {
        const int64_t c = (int64_t)locs[r * k + j] - 1;
        if (c < 0 || c >= ncols) {
          bad = locs[r * k + j] == -1 ? 4 : 1;
          break;
        }
        const int32_t rec = col_rec[c];
        if (rec < 0 || rec >= nrec) {
          bad = 2;
          break;
        }
        memcpy(w, h, hl);
        w += hl;
        w[0] = ' ';
        w[1] = strand[c] == 0 ? '+' : '-';
        w[2] = ' ';
        w += 3;
        w += julia_f32(vals[r * k + j], w);
        *w++ = ' ';
        w = std::to_chars(w, w + 20, starts[c] - 1).ptr;
        *w++ = ' ';
        const auto &nm = rn[(size_t)rec];
        memcpy(w, rec_names + nm.first, nm.second);
        w += nm.second;
        *w++ = '\n';
      }
    }
    part[(size_t)b] = buf;
    used[(size_t)b] = (size_t)(w - buf.p);
  };
  auto run = [&](auto &&fn) {
    if (nblk == 1) {
      fn(0);
      return;
    }
    std::vector<std::thread> th;
    for (int64_t b = 0; b < nblk; ++b) th.emplace_back(fn, b);
    for (auto &t : th) t.join();
  };
  run(format);
  if (bad) {
    for (auto &b : part) give_buf(b);
    if (bad == 4)
      return r2m::fail(R2M_ETIMEOUT, "location -1: the search that produced this batch gave up on a "
                                     "device-side wait (device timeout); its rows hold no result");
    if (bad == 1) return r2m::fail(R2M_EINVAL, "location out of range (1-based, 1..N)");
    if (bad == 2) return r2m::fail(R2M_EINVAL, "column record id out of range");
    return r2m::fail(R2M_ENOMEM, "table buffer allocation failed");
  }
  std::vector<size_t> off((size_t)nblk + 1, 0);
  for (int64_t b = 0; b < nblk; ++b) off[(size_t)b + 1] = off[(size_t)b] + used[(size_t)b];
  r2m_text *t = new r2m_text();
  t->b = take_buf(off.back());
  t->n = off.back();
  if (!t->b.p) {
    for (auto &b : part) give_buf(b);
    delete t;
    return r2m::fail(R2M_ENOMEM, "table buffer allocation failed");
  }
  run([&](int64_t b) {
    memcpy(t->b.p + off[(size_t)b], part[(size_t)b].p, used[(size_t)b]);
    give_buf(part[(size_t)b]);
  });
  *out = t;
  return R2M_OK;
}

extern "C" const char *r2m_text_data(const r2m_text *t, size_t *len) {
  if (len) *len = t ? t->n : 0;
  return t ? t->b.p : nullptr;
}

extern "C" void r2m_text_free(r2m_text *t) {
  if (!t) return;
  give_buf(t->b);
  delete t;
}
