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
// Rows are split into blocks formatted by separate threads and concatenated
// in order.
#include <string.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <string>
#include <thread>
#include <vector>

#include "r2m.h"

namespace r2m {
int fail(int code, const std::string &msg);
}  // namespace r2m

struct r2m_text {
  std::string s;
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
  for (int64_t i = 0; i < nb * (int64_t)k; ++i) {
    const int64_t c = (int64_t)locs[i] - 1;
    if (c < 0 || c >= ncols) return r2m::fail(R2M_EINVAL, "location out of range (1-based, 1..N)");
    if (col_rec[c] < 0 || col_rec[c] >= nrec) return r2m::fail(R2M_EINVAL, "column record id out of range");
  }
  if (nthreads < 1) nthreads = 1;
  const int64_t nblk = nb < 2048 ? 1 : std::min<int64_t>(nthreads, (nb + 1023) / 1024);
  std::vector<std::string> part((size_t)nblk);
  auto work = [&](int64_t b) {
    const int64_t r0 = nb * b / nblk, r1 = nb * (b + 1) / nblk;
    std::string &s = part[(size_t)b];
    s.reserve((size_t)(r1 - r0) * k * 64);
    char num[48];
    for (int64_t r = r0; r < r1; ++r) {
      const char *h = heads + hd[(size_t)r].first;
      size_t hl = hd[(size_t)r].second;
      if (hl && h[0] == '>') {
        ++h;
        --hl;
      }
      for (int j = 0; j < k; ++j) {
        const int64_t c = (int64_t)locs[r * k + j] - 1;
        s.append(h, hl);
        s.append(strand[c] == 0 ? " + " : " - ");
        s.append(num, (size_t)julia_f32(vals[r * k + j], num));
        s.push_back(' ');
        auto q = std::to_chars(num, num + sizeof(num), starts[c] - 1);
        s.append(num, (size_t)(q.ptr - num));
        s.push_back(' ');
        const auto &nm = rn[(size_t)col_rec[c]];
        s.append(rec_names + nm.first, nm.second);
        s.push_back('\n');
      }
    }
  };
  if (nblk == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int64_t b = 0; b < nblk; ++b) th.emplace_back(work, b);
    for (auto &t : th) t.join();
  }
  r2m_text *t = new r2m_text();
  size_t tot = 0;
  for (auto &p : part) tot += p.size();
  t->s.reserve(tot);
  for (auto &p : part) t->s.append(p);
  *out = t;
  return R2M_OK;
}

extern "C" const char *r2m_text_data(const r2m_text *t, size_t *len) {
  if (len) *len = t ? t->s.size() : 0;
  return t ? t->s.data() : nullptr;
}

extern "C" void r2m_text_free(r2m_text *t) { delete t; }
