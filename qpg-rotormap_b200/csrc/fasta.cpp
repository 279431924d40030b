// fasta.cpp -- host FASTA reader: records -> forward 2-bit words, trimmed
// to the first k bases (records shorter than k are skipped).
//
// Semantics of fasta_reads / _next_rec3 / _collect3! / _emit3!
// (RotorMap/fasta/reader.jl:21-28,61-75,120-198,204-311):
//   * a record starts at a '>' that is the first byte of the input or
//     follows '\n' or '\r'; bytes before the first record are ignored;
//   * the header is the '>' line up to (excluding) the first '\n', one
//     trailing '\r' removed; a header line that is not closed by '\n' before
//     the next record start (or the end of input) ends the parse;
//   * every sequence byte except '\n'/'\r' is a base: A/C/G/T (either case)
//     -> 0/1/2/3, anything else -> 2 (G);
//   * base j sits in word j>>4 at bits 2*(j&15); the tail is zero-padded.
// Records come back in file order.  Large inputs are split at record
// boundaries and parsed by several threads; the result does not depend on
// the thread count.
#include <string.h>

#include <string>
#include <thread>
#include <vector>

#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "r2m.h"

namespace r2m {
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
}  // namespace r2m

struct r2m_reads {
  int k = 0, W = 0;
  std::vector<uint32_t> words;
  std::vector<size_t> hoff;  // header offsets into `heads` (n+1 entries)
  std::string heads;         // every header followed by '\n'
};

namespace {

// code[b]: the base's 2-bit code; '\n' and '\r' map to kSkip (not a base)
constexpr uint8_t kSkip = 0x80;
struct Lut {
  uint8_t code[256];
  Lut() {
    for (int i = 0; i < 256; ++i) code[i] = 2;
    code[(int)'A'] = 0; code[(int)'C'] = 1; code[(int)'G'] = 2; code[(int)'T'] = 3;
    code[(int)'a'] = 0; code[(int)'c'] = 1; code[(int)'g'] = 2; code[(int)'t'] = 3;
    code[(int)'\n'] = kSkip; code[(int)'\r'] = kSkip;
  }
};
const Lut kLut;

// 16 sequence bytes -> their 2-bit codes packed into one word (byte j at
// bits 2j); false when the block holds a line break (the caller then walks
// it byte by byte).  For A/C/G/T in either case ((c >> 1) ^ (c >> 2)) & 3 is
// the code; every other byte becomes 2 (G).
inline bool pack16(const uint8_t *q, uint32_t &out) {
#if defined(__SSE2__)
  const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i *>(q));
  const __m128i brk = _mm_or_si128(_mm_cmpeq_epi8(c, _mm_set1_epi8('\n')), _mm_cmpeq_epi8(c, _mm_set1_epi8('\r')));
  if (_mm_movemask_epi8(brk)) return false;
  __m128i code = _mm_and_si128(_mm_xor_si128(_mm_srli_epi16(c, 1), _mm_srli_epi16(c, 2)), _mm_set1_epi8(3));
  const __m128i lc = _mm_or_si128(c, _mm_set1_epi8(0x20));  // case fold
  const __m128i valid =
      _mm_or_si128(_mm_or_si128(_mm_cmpeq_epi8(lc, _mm_set1_epi8('a')), _mm_cmpeq_epi8(lc, _mm_set1_epi8('c'))),
                   _mm_or_si128(_mm_cmpeq_epi8(lc, _mm_set1_epi8('g')), _mm_cmpeq_epi8(lc, _mm_set1_epi8('t'))));
  code = _mm_or_si128(_mm_and_si128(valid, code), _mm_andnot_si128(valid, _mm_set1_epi8(2)));
  // pack: byte pairs -> 4 bits, 16-bit pairs -> 8 bits, 32-bit pairs -> 16 bits
  __m128i x = _mm_and_si128(_mm_or_si128(code, _mm_srli_epi16(code, 6)), _mm_set1_epi16(0x00FF));
  x = _mm_and_si128(_mm_or_si128(x, _mm_srli_epi32(x, 12)), _mm_set1_epi32(0x000000FF));
  x = _mm_or_si128(x, _mm_srli_epi64(x, 24));
  out = ((uint32_t)_mm_cvtsi128_si32(x) & 0xFFFFu) | (((uint32_t)_mm_extract_epi16(x, 4) & 0xFFFFu) << 16);
  return true;
#else
  uint32_t v = 0;
  uint8_t any = 0;
  for (int j = 0; j < 16; ++j) {
    const uint8_t c = kLut.code[q[j]];
    any |= c;
    v |= (uint32_t)(c & 3) << (2 * j);
  }
  out = v;
  return !(any & kSkip);
#endif
}

inline bool is_rec_start(const char *d, size_t i) {
  return d[i] == '>' && (i == 0 || d[i - 1] == '\n' || d[i - 1] == '\r');
}

// first record start in [from, hi), or hi
size_t next_rec(const char *d, size_t from, size_t hi) {
  size_t p = from;
  while (p < hi) {
    const void *q = memchr(d + p, '>', hi - p);
    if (!q) return hi;
    size_t t = (size_t)((const char *)q - d);
    if (is_rec_start(d, t)) return t;
    p = t + 1;
  }
  return hi;
}

struct Part {
  std::vector<uint32_t> words;
  std::vector<size_t> hlen;
  std::string heads;
  bool stop = false;  // an unterminated header line ended the parse here
};

// Parse the records whose starts lie in [lo, hi) (lo is a record start or
// hi); sequences may run to `end` (the record's own next start).
void parse_range(const char *d, size_t n, size_t lo, size_t hi, int k, Part &out) {
  const int W = (k + 15) / 16;
  std::vector<uint32_t> w(W);
  size_t s = lo;
  while (s < hi) {
    size_t e = next_rec(d, s + 1, n);
    const void *nl = memchr(d + s, '\n', e - s);
    if (!nl) {  // header not closed before the next record / EOF
      out.stop = true;
      return;
    }
    size_t h = (size_t)((const char *)nl - d);
    size_t hend = h;  // exclusive
    if (hend > s && d[hend - 1] == '\r') --hend;
    // collect the first k bases of [h+1, e): 16 bytes per step while none
    // of them is a line break, byte by byte otherwise
    std::fill(w.begin(), w.end(), 0u);
    int bases = 0;
    size_t p = h + 1;
    const uint8_t *code = kLut.code;
    while (bases < k && p < e) {
      if (bases + 16 <= k && p + 16 <= e) {
        uint32_t v;
        if (pack16((const uint8_t *)d + p, v)) {
          int wi = bases >> 4, sh = 2 * (bases & 15);
          w[wi] |= v << sh;
          if (sh) w[wi + 1] |= v >> (32 - sh);
          bases += 16;
          p += 16;
          continue;
        }
      }
      uint8_t c = code[(uint8_t)d[p++]];
      if (c & kSkip) continue;
      w[bases >> 4] |= (uint32_t)c << (2 * (bases & 15));
      ++bases;
    }
    if (bases >= k) {
      out.words.insert(out.words.end(), w.begin(), w.end());
      out.hlen.push_back(hend - s);
      out.heads.append(d + s, hend - s);
    }
    s = e;
  }
}

}  // namespace

extern "C" int r2m_fasta_reads(const char *data, size_t len, int k, int nthreads, r2m_reads **out) {
  if (!out) return r2m::fail(R2M_EINVAL, "out is null");
  *out = nullptr;
  if (k < 1) return r2m::fail(R2M_EINVAL, "k must be >= 1");
  if (!data && len) return r2m::fail(R2M_EINVAL, "data is null");
  r2m_reads *r = new r2m_reads();
  r->k = k;
  r->W = (k + 15) / 16;
  r->hoff.push_back(0);
  if (len == 0) {
    *out = r;
    return R2M_OK;
  }
  if (nthreads < 1) nthreads = 1;
  if (len < (size_t)(1 << 22)) nthreads = 1;
  // split points at record starts
  std::vector<size_t> cuts;
  cuts.push_back(next_rec(data, 0, len));
  for (int t = 1; t < nthreads; ++t) {
    size_t guess = len * (size_t)t / (size_t)nthreads;
    if (guess <= cuts.back()) continue;
    size_t c = next_rec(data, guess, len);
    if (c > cuts.back() && c < len) cuts.push_back(c);
  }
  cuts.push_back(len);
  size_t np = cuts.size() - 1;
  std::vector<Part> parts(np);
  if (np == 1) {
    parse_range(data, len, cuts[0], cuts[1], k, parts[0]);
  } else {
    std::vector<std::thread> th;
    for (size_t i = 0; i < np; ++i)
      th.emplace_back(parse_range, data, len, cuts[i], cuts[i + 1], k, std::ref(parts[i]));
    for (auto &t : th) t.join();
  }
  // the parse ends at the first part that met an unclosed header (that part
  // keeps the records before it); place every kept part at its offset
  size_t keep = 0;
  while (keep < np && !parts[keep].stop) ++keep;
  if (keep < np) ++keep;
  std::vector<size_t> wofs(keep + 1, 0), hofs(keep + 1, 0), rofs(keep + 1, 0);
  for (size_t i = 0; i < keep; ++i) {
    wofs[i + 1] = wofs[i] + parts[i].words.size();
    hofs[i + 1] = hofs[i] + parts[i].heads.size() + parts[i].hlen.size();  // + one '\n' per header
    rofs[i + 1] = rofs[i] + parts[i].hlen.size();
  }
  r->words.resize(wofs[keep]);
  r->heads.resize(hofs[keep]);
  r->hoff.resize(rofs[keep] + 1);
  r->hoff[0] = 0;
  auto place = [&](size_t i) {
    const Part &p = parts[i];
    if (!p.words.empty()) memcpy(r->words.data() + wofs[i], p.words.data(), p.words.size() * sizeof(uint32_t));
    char *dst = &r->heads[0] + hofs[i];
    size_t src = 0, o = hofs[i];
    for (size_t j = 0; j < p.hlen.size(); ++j) {
      memcpy(dst, p.heads.data() + src, p.hlen[j]);
      dst += p.hlen[j];
      *dst++ = '\n';
      src += p.hlen[j];
      o += p.hlen[j] + 1;
      r->hoff[rofs[i] + j + 1] = o;
    }
  };
  if (keep <= 1) {
    if (keep) place(0);
  } else {
    std::vector<std::thread> th;
    for (size_t i = 0; i < keep; ++i) th.emplace_back(place, i);
    for (auto &t : th) t.join();
  }
  *out = r;
  return R2M_OK;
}

extern "C" int64_t r2m_reads_count(const r2m_reads *r) {
  return r ? (int64_t)(r->hoff.size() - 1) : 0;
}

extern "C" const uint32_t *r2m_reads_words(const r2m_reads *r) {
  return (r && !r->words.empty()) ? r->words.data() : nullptr;
}

extern "C" const char *r2m_reads_header(const r2m_reads *r, int64_t i, size_t *len) {
  if (!r || i < 0 || i >= r2m_reads_count(r)) {
    if (len) *len = 0;
    return nullptr;
  }
  if (len) *len = r->hoff[i + 1] - r->hoff[i] - 1;
  return r->heads.data() + r->hoff[i];
}

extern "C" const char *r2m_reads_header_blob(const r2m_reads *r, size_t *total_len) {
  if (total_len) *total_len = r ? r->heads.size() : 0;
  return r ? r->heads.data() : nullptr;
}

extern "C" const size_t *r2m_reads_header_offsets(const r2m_reads *r) {
  return r ? r->hoff.data() : nullptr;
}

extern "C" void r2m_reads_free(r2m_reads *r) { delete r; }
