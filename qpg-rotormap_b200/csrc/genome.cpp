// genome.cpp -- host reference-genome packer: FASTA -> every record's bases
// as 2-bit words (base j of a record in word j>>4 at bits 2*(j&15); each
// record starts on a word boundary and is followed by one zero guard word),
// the record headers, word offsets and base counts.
//
// Record walk of the index builder (RotorMap/index/build.jl:291-324, with
// the record table of RotorMap/test/harness.jl:52-91):
//   * a record starts at a '>' that is the first byte or follows '\n'/'\r';
//     bytes before the first record are ignored;
//   * the header is [start, first '\n' at or after the start), one trailing
//     '\r' removed (no '\n' at all: the header runs to the end);
//   * the sequence is (header '\n', next record start); every byte in it
//     other than '\n'/'\r' is a base: A/C/G/T either case -> 0/1/2/3,
//     anything else -> 2; a header whose '\n' lies at or past the next
//     record start leaves an empty sequence.
// Work split for multi-gigabase inputs: record starts by memchr over
// per-thread byte ranges; the sequence bytes cut into items of at most
// kItem bytes; a parallel base count per item gives every item its first
// base within its record; a parallel pack writes each item's words, with an
// atomic OR only on the (at most two) words an item shares with its
// neighbours.
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "r2m.h"

namespace r2m {
int fail(int code, const std::string &msg);
}  // namespace r2m

struct r2m_genome {
  std::vector<uint32_t> words;
  std::vector<int64_t> word_off, nbases;
  std::string heads;  // every header followed by '\n'
};

namespace {

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

constexpr size_t kItem = size_t(8) << 20;

template <class F>
void parallel_for(int64_t n, int nthreads, F f) {
  if (n <= 0) return;
  const int nt = (int)std::min<int64_t>(std::max(nthreads, 1), n);
  if (nt == 1) {
    for (int64_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (int64_t i = t; i < n; i += nt) f(i);
    });
  for (auto &x : th) x.join();
}

void rec_starts(const char *d, size_t lo, size_t hi, std::vector<size_t> &out) {
  size_t p = lo;
  while (p < hi) {
    const void *q = memchr(d + p, '>', hi - p);
    if (!q) return;
    const size_t t = (size_t)((const char *)q - d);
    if (t == 0 || d[t - 1] == '\n' || d[t - 1] == '\r') out.push_back(t);
    p = t + 1;
  }
}

struct Item {
  int64_t rec;
  size_t lo, hi;       // bytes
  int64_t base0 = 0;   // first base of the item within its record
  int64_t nb = 0;      // bases in the item
};

int64_t count_bases(const uint8_t *p, size_t n) {
  int64_t c = 0;
  for (size_t i = 0; i < n; ++i) c += (kLut.code[p[i]] & kSkip) ? 0 : 1;
  return c;
}

inline void or_word(uint32_t *w, uint32_t v, bool shared) {
  if (!v) return;
  if (shared)
    __atomic_fetch_or(w, v, __ATOMIC_RELAXED);
  else
    *w |= v;
}

// Pack the item's bases into out (the record's first word), which starts
// zeroed; words [first, last] may be shared with the neighbouring items.
void pack_item(const uint8_t *p, size_t n, int64_t base0, int64_t nb, uint32_t *out) {
  if (nb == 0) return;
  const int64_t first = base0 >> 4, last = (base0 + nb - 1) >> 4;
  int64_t b = base0;
  uint32_t acc = 0;
  int64_t cur = first;
  auto emit = [&](int64_t wi, uint32_t v) { or_word(out + wi, v, wi == first || wi == last); };
  size_t i = 0;
  while (i < n) {
    // 16 bytes without a line break starting on a word boundary: one word
    if ((b & 15) == 0 && i + 16 <= n) {
      uint32_t v = 0;
      uint8_t any = 0;
      for (int j = 0; j < 16; ++j) {
        const uint8_t c = kLut.code[p[i + j]];
        any |= c;
        v |= (uint32_t)(c & 3) << (2 * j);
      }
      if (!(any & kSkip)) {
        emit(cur, acc);  // the word the slow path just completed, if any
        acc = 0;
        emit(b >> 4, v);
        b += 16;
        cur = b >> 4;
        i += 16;
        continue;
      }
    }
    const uint8_t c = kLut.code[p[i++]];
    if (c & kSkip) continue;
    if ((b >> 4) != cur) {
      emit(cur, acc);
      acc = 0;
      cur = b >> 4;
    }
    acc |= (uint32_t)c << (2 * (b & 15));
    ++b;
  }
  emit(cur, acc);
}

}  // namespace

extern "C" int r2m_fasta_genome(const char *data, size_t len, int nthreads, r2m_genome **out) {
  if (!out) return r2m::fail(R2M_EINVAL, "out is null");
  *out = nullptr;
  if (!data && len) return r2m::fail(R2M_EINVAL, "data is null");
  if (nthreads < 1) nthreads = 1;
  r2m_genome *g = new r2m_genome();
  const uint8_t *u = (const uint8_t *)data;
  // record starts, in order
  std::vector<size_t> starts;
  {
    const int nt = len < (size_t(1) << 24) ? 1 : nthreads;
    std::vector<std::vector<size_t>> part(nt);
    parallel_for(nt, nt, [&](int64_t t) {
      rec_starts(data, len * (size_t)t / nt, len * (size_t)(t + 1) / nt, part[t]);
    });
    for (auto &v : part) starts.insert(starts.end(), v.begin(), v.end());
  }
  const int64_t R = (int64_t)starts.size();
  std::vector<size_t> seq_lo(R), seq_hi(R);
  std::vector<Item> items;
  for (int64_t r = 0; r < R; ++r) {
    const size_t s = starts[r], e = r + 1 < R ? starts[r + 1] : len;
    const void *nl = memchr(data + s, '\n', len - s);
    const size_t h = nl ? (size_t)((const char *)nl - data) : len;
    size_t hend = h;
    if (hend > s && data[hend - 1] == '\r') --hend;
    g->heads.append(data + s, hend - s);
    g->heads.push_back('\n');
    seq_lo[r] = h + 1 < e ? h + 1 : e;
    seq_hi[r] = e;
    for (size_t lo = seq_lo[r]; lo < seq_hi[r]; lo += kItem) items.push_back({r, lo, std::min(lo + kItem, seq_hi[r])});
  }
  const int64_t NI = (int64_t)items.size();
  parallel_for(NI, nthreads, [&](int64_t i) { items[i].nb = count_bases(u + items[i].lo, items[i].hi - items[i].lo); });
  g->nbases.assign(R, 0);
  for (int64_t i = 0; i < NI; ++i) {
    items[i].base0 = g->nbases[items[i].rec];
    g->nbases[items[i].rec] += items[i].nb;
  }
  g->word_off.resize(R);
  int64_t cur = 0;
  for (int64_t r = 0; r < R; ++r) {
    g->word_off[r] = cur;
    cur += (g->nbases[r] + 15) / 16 + 1;  // + zero guard word
  }
  try {
    g->words.assign((size_t)std::max<int64_t>(cur, 1), 0u);
  } catch (const std::bad_alloc &) {
    delete g;
    return r2m::fail(R2M_ENOMEM, "genome words");
  }
  parallel_for(NI, nthreads, [&](int64_t i) {
    const Item &it = items[i];
    pack_item(u + it.lo, it.hi - it.lo, it.base0, it.nb, g->words.data() + g->word_off[it.rec]);
  });
  *out = g;
  return R2M_OK;
}

extern "C" int64_t r2m_genome_count(const r2m_genome *g) { return g ? (int64_t)g->nbases.size() : 0; }

extern "C" const uint32_t *r2m_genome_words(const r2m_genome *g, size_t *nwords) {
  if (nwords) *nwords = g ? g->words.size() : 0;
  return g ? g->words.data() : nullptr;
}

extern "C" const int64_t *r2m_genome_word_off(const r2m_genome *g) {
  return (g && !g->word_off.empty()) ? g->word_off.data() : nullptr;
}

extern "C" const int64_t *r2m_genome_nbases(const r2m_genome *g) {
  return (g && !g->nbases.empty()) ? g->nbases.data() : nullptr;
}

extern "C" const char *r2m_genome_header_blob(const r2m_genome *g, size_t *total_len) {
  if (total_len) *total_len = g ? g->heads.size() : 0;
  return g ? g->heads.data() : nullptr;
}

extern "C" void r2m_genome_free(r2m_genome *g) { delete g; }
