/*
 * rotormap_oracle.c -- CPU restatement of RotorMap's read-mapping hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the parity tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg compare the CUDA
 * library against; nothing in the product path links or calls it.
 *
 * Parity status: pinned against the reference's own outputs.  The
 * reference (Julia, not installed here) commits three encoder sweep curves
 * (RotorMap/experiments/out/rope_*_sweep.csv: its fp64 encoder at k =
 * 20,000, s5 m1 c5, on Julia-Xoshiro fixtures); with the same fixtures drawn
 * here (rotormap.jlrandom), orc_rope_frag_f64 reproduces their float64 inner
 * products to within 1e-12 (tests/golden/rope_sweeps.json).  The
 * reference's known-answer properties (unit energy, window /
 * reverse-complement word identities, e4m3 == host conversion, exact top-k
 * multisets) and the hand-derived vectors under tests/golden/ cover what
 * those curves do not exercise (the scramble at s > c, m > 1).
 *
 * Functions and the reference code each one restates:
 *   orc_rope_frag_f64   _ref_rope_frag / _ref_rope_frag_real
 *                       (RotorMap/encode/reference.jl:37-105), fp64, modes 0-3
 *   orc_rope_frag_f32   kernel_rope_frag_real's fp32 arithmetic
 *                       (RotorMap/encode/kernel.jl:115-290): fp32 theta,
 *                       cos/sin at the owning thread's first window and the
 *                       fp32 complex recurrence, sums in window order
 *   orc_f32_to_f16      IEEE binary16 round-to-nearest-even (the fp16 output
 *                       of kernel.jl:285-286)
 *   orc_f32_to_e4m3     e4m3fn RNE + satfinite, the published OCP FP8 E4M3
 *                       definition (bias 7, max 448, no Inf) -- the
 *                       conversion DLFP8Types 0.1.0 Float8_E4M3FN() applies
 *                       on the host (RotorMap/index/build.jl:730) and
 *                       cvt.rn.satfinite on the device (gemm/fp8_ptx.jl:161)
 *   orc_e4m3_to_f32     exact widening (gemm/fp8_convert.jl:105)
 *   orc_topk_e4m3       brute-force scores of e4m3 reads x e4m3 index columns
 *                       (the reference's own CPU check `Bh' * hrefq`,
 *                       RotorMap/search/engine_fp8.jl:873-883) with the
 *                       score rounding of cout = :f16 / :f32
 *                       (engine_fp8.jl:20-27, fp8_lt.jl:128-168) and the
 *                       exact top-k ordering of _assert_topk_rows
 *                       (engine_fp8.jl:826-838): score desc, ties by column asc
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* Minimal parallel-for over [0, n): `nthreads` pthreads pull indices from a
 * shared counter (libgomp is not available in this toolchain). */
typedef void (*orc_body_fn)(int64_t i, void *ctx);
typedef struct {
  int64_t n;
  int64_t next;
  pthread_mutex_t mu;
  orc_body_fn fn;
  void *ctx;
} orc_pool;

static void *orc_worker(void *arg) {
  orc_pool *p = (orc_pool *)arg;
  for (;;) {
    pthread_mutex_lock(&p->mu);
    int64_t i = p->next++;
    pthread_mutex_unlock(&p->mu);
    if (i >= p->n) break;
    p->fn(i, p->ctx);
  }
  return NULL;
}

static void orc_parallel_for(int64_t n, int nthreads, orc_body_fn fn, void *ctx) {
  orc_pool p;
  p.n = n;
  p.next = 0;
  p.fn = fn;
  p.ctx = ctx;
  pthread_mutex_init(&p.mu, NULL);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  int started = 0;
  for (int t = 1; t < nthreads; ++t)
    if (pthread_create(&th[started], NULL, orc_worker, &p) == 0) ++started;
  orc_worker(&p);
  for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
  pthread_mutex_destroy(&p.mu);
}

/* ------------------------------------------------------------ fp16 / e4m3 */

uint16_t orc_f32_to_f16(float f) {
  uint32_t x;
  memcpy(&x, &f, 4);
  uint32_t sign = (x >> 16) & 0x8000u;
  uint32_t ax = x & 0x7FFFFFFFu;
  if (ax >= 0x7F800000u) return (uint16_t)(sign | (ax > 0x7F800000u ? 0x7E00u : 0x7C00u));
  /* exponent of the value, unbiased */
  int e = (int)(ax >> 23) - 127;
  uint32_t mant = (ax & 0x7FFFFFu) | (ax >= 0x800000u ? 0x800000u : 0);
  if (e > 15) return (uint16_t)(sign | 0x7C00u); /* overflow -> Inf */
  if (e >= -14) {
    /* normal half: keep 10 mantissa bits of the 24-bit significand */
    uint32_t shift = 13;
    uint32_t q = mant >> shift, rem = mant & ((1u << shift) - 1), half = 1u << (shift - 1);
    if (rem > half || (rem == half && (q & 1))) q++;
    /* q has 11 significant bits (implicit one); may carry into 12 */
    uint32_t he = (uint32_t)(e + 15);
    if (q >= 0x800u) {
      q >>= 1;
      he++;
    }
    if (he >= 31) return (uint16_t)(sign | 0x7C00u);
    return (uint16_t)(sign | (he << 10) | (q & 0x3FFu));
  }
  /* subnormal half: value = q * 2^-24 */
  if (ax < 0x33000000u) { /* < 2^-25: rounds to zero (ties-to-even at 2^-25) */
    return (uint16_t)sign;
  }
  {
    int shift = 13 + (-14 - e); /* bits dropped from the 24-bit significand */
    uint32_t q, rem, half;
    if (shift >= 32) return (uint16_t)sign;
    q = mant >> shift;
    rem = mant & ((1u << shift) - 1);
    half = 1u << (shift - 1);
    if (rem > half || (rem == half && (q & 1))) q++;
    return (uint16_t)(sign | q); /* q may reach 0x400 = smallest normal: correct encoding */
  }
}

float orc_f16_to_f32(uint16_t h) {
  uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  uint32_t e = (h >> 10) & 0x1F, m = h & 0x3FF;
  float v;
  if (e == 0) {
    v = ldexpf((float)m, -24);
  } else if (e == 31) {
    v = m ? NAN : INFINITY;
  } else {
    v = ldexpf((float)(m | 0x400), (int)e - 25);
  }
  uint32_t x;
  memcpy(&x, &v, 4);
  x |= sign;
  memcpy(&v, &x, 4);
  return v;
}

/* e4m3fn: s eeee mmm, bias 7; normals 2^-6 .. 448, subnormals m * 2^-9;
 * 0x7F / 0xFF are NaN; satfinite clamps finite overflow (and Inf) to 448. */
uint8_t orc_f32_to_e4m3(float f) {
  uint32_t x;
  memcpy(&x, &f, 4);
  uint8_t sign = (uint8_t)((x >> 24) & 0x80u);
  uint32_t ax = x & 0x7FFFFFFFu;
  if (ax > 0x7F800000u) return 0x7F; /* NaN */
  if (ax == 0x7F800000u) return (uint8_t)(sign | 0x7E); /* Inf -> 448 (satfinite) */
  double a = (double)fabsf(f);
  if (a == 0.0) return sign;
  /* scale so that the representable grid near `a` has unit spacing */
  int e;
  frexp(a, &e); /* a = fr * 2^e, fr in [0.5, 1) -> unbiased exponent e-1 */
  int ue = e - 1;
  if (ue < -6) ue = -6; /* subnormal range shares the 2^-9 spacing */
  double step = ldexp(1.0, ue - 3);
  double q = a / step; /* exact: power-of-two scaling */
  double fl = floor(q);
  double rem = q - fl;
  double r;
  if (rem > 0.5) r = fl + 1.0;
  else if (rem < 0.5) r = fl;
  else r = (fmod(fl, 2.0) == 0.0) ? fl : fl + 1.0;
  double v = r * step;
  if (v > 448.0) return (uint8_t)(sign | 0x7E);
  /* encode v */
  if (v < ldexp(1.0, -6)) { /* subnormal: v = mm * 2^-9 */
    int mm = (int)(v / ldexp(1.0, -9));
    return (uint8_t)(sign | mm);
  }
  {
    int ve;
    frexp(v, &ve);
    int be = ve - 1 + 7;
    int mm = (int)(v / ldexp(1.0, ve - 1 - 3)) - 8;
    return (uint8_t)(sign | (be << 3) | mm);
  }
}

float orc_e4m3_to_f32(uint8_t b) {
  int s = b >> 7, e = (b >> 3) & 0xF, m = b & 7;
  float v;
  if (e == 0xF && m == 7) return NAN;
  if (e == 0) v = ldexpf((float)m, -9);
  else v = ldexpf((float)(8 + m), e - 7 - 3);
  return s ? -v : v;
}

void orc_f32_to_e4m3_array(const float *src, uint8_t *dst, int64_t n) {
  for (int64_t i = 0; i < n; ++i) dst[i] = orc_f32_to_e4m3(src[i]);
}
void orc_f32_to_f16_array(const float *src, uint16_t *dst, int64_t n) {
  for (int64_t i = 0; i < n; ++i) dst[i] = orc_f32_to_f16(src[i]);
}

/* ------------------------------------------------------------ rope encoder */

static uint32_t smer_at(const uint8_t *codes, int p, int s) {
  uint32_t v = 0;
  for (int j = 0; j < s; ++j) v |= (uint32_t)codes[p + j] << (2 * j); /* little-endian field */
  return v;
}

static uint32_t scramble(uint32_t smer, int c) {
  uint32_t cb = (c >= 16) ? 0xFFFFFFFFu : ((1u << (2 * c)) - 1u);
  uint32_t lower = smer & cb;
  uint32_t upper = (2 * c >= 32) ? 0u : (smer >> (2 * c));
  return lower ^ ((upper * 0x9E3779B1u) & cb);
}

static uint32_t g_bin(int c) {
  uint32_t allones = 0;
  for (int i = 0; i < c; ++i) allones += 1u << (2 * i);
  return 2u * allones; /* 0-based csmer of the reference's 2*allones+1 */
}

/* fp64 golden encoder: out[2D] split [Re; Im], norms[m].  Returns 0. */
int orc_rope_frag_f64(const uint8_t *codes, int k, int s, int m, int c, int normalize, double *out,
                      double *norms) {
  int nbin = m << (2 * c);
  int nw = k - s + 1;
  double *hr = (double *)calloc((size_t)nbin, sizeof(double));
  double *hi = (double *)calloc((size_t)nbin, sizeof(double));
  if (!hr || !hi) return -1;
  for (int p = 0; p < nw; ++p) {
    uint32_t cs = scramble(smer_at(codes, p, s), c);
    for (int idm = 0; idm < m; ++idm) {
      double f = (m == 1) ? 1.0 : 2.0 * idm / (double)(m - 1) + 1.0;
      double th = f * (2.0 * M_PI / (double)k);
      hr[cs * m + idm] += cos(th * p);
      hi[cs * m + idm] += sin(th * p);
    }
  }
  uint32_t gb = g_bin(c);
  for (int idm = 0; idm < m; ++idm) hr[gb * m + idm] = hi[gb * m + idm] = 0.0;
  for (int t = 0; t < m; ++t) norms[t] = 0.0;
  if (normalize == 0) {
    double acc = 0.0;
    for (int b = 0; b < nbin; ++b) acc += hr[b] * hr[b] + hi[b] * hi[b];
    double nrm = sqrt(acc) + 1e-16;
    for (int b = 0; b < nbin; ++b) {
      hr[b] /= nrm;
      hi[b] /= nrm;
    }
    norms[0] = nrm;
  } else {
    const double eps = 2.220446049250313e-16;
    if (normalize >= 2) {
      for (int b = 0; b < nbin; ++b) {
        double a = hypot(hr[b], hi[b]);
        double d = (normalize == 2) ? (a + eps) : sqrt(a + eps);
        hr[b] /= d;
        hi[b] /= d;
      }
    }
    for (int idm = 0; idm < m; ++idm) {
      double acc = 0.0;
      for (int b = idm; b < nbin; b += m) acc += hr[b] * hr[b] + hi[b] * hi[b];
      double nrm = sqrt(acc) + (normalize == 1 ? 1e-7 : eps);
      for (int b = idm; b < nbin; b += m) {
        hr[b] /= nrm;
        hi[b] /= nrm;
      }
      norms[idm] = nrm;
    }
  }
  for (int b = 0; b < nbin; ++b) {
    out[b] = hr[b];
    out[nbin + b] = hi[b];
  }
  free(hr);
  free(hi);
  return 0;
}

/* fp32 restatement of the GPU kernel's arithmetic (see file header). */
int orc_rope_frag_f32(const uint8_t *codes, int k, int s, int m, int c, int normalize, float *out,
                      float *norms) {
  int nbin = m << (2 * c);
  int nw = k - s + 1;
  int wc = (nw + 511) / 512;
  if ((wc & 1) == 0) wc += 1;
  float *h = (float *)calloc((size_t)2 * nbin, sizeof(float));
  if (!h) return -1;
  float base = (float)(2.0 * M_PI / (double)k);
  for (int idm = 0; idm < m; ++idm) {
    float f = (m == 1) ? 1.0f : (float)(2.0 * idm / (double)(m - 1) + 1.0);
    float th = f * base;
    float xr = cosf(th), xi = sinf(th);
    float re = 0.f, im = 0.f;
    for (int p = 0; p < nw; ++p) {
      if (p % wc == 0) {
        float a = th * (float)p;
        re = cosf(a);
        im = sinf(a);
      } else {
        volatile float t1 = re * xr, t2 = im * xi, t3 = re * xi, t4 = im * xr;
        float nr = t1 - t2, ni = t3 + t4;
        re = nr;
        im = ni;
      }
      uint32_t cs = scramble(smer_at(codes, p, s), c);
      size_t b = (size_t)cs * m + idm;
      h[2 * b] += re;
      h[2 * b + 1] += im;
    }
  }
  uint32_t gb = g_bin(c);
  for (int idm = 0; idm < m; ++idm) h[2 * (gb * m + idm)] = h[2 * (gb * m + idm) + 1] = 0.f;
  if (normalize >= 2) {
    for (int b = 0; b < nbin; ++b) {
      double a = (double)hypotf(h[2 * b], h[2 * b + 1]);
      double d = (normalize == 2) ? (a + 2.220446049250313e-16) : sqrt(a + 2.220446049250313e-16);
      h[2 * b] = (float)((double)h[2 * b] / d);
      h[2 * b + 1] = (float)((double)h[2 * b + 1] / d);
    }
  }
  float part[64];
  for (int idm = 0; idm < m; ++idm) {
    float acc = 0.f;
    for (int b = idm; b < nbin; b += m) acc += h[2 * b] * h[2 * b] + h[2 * b + 1] * h[2 * b + 1];
    part[idm] = acc;
  }
  float nrmv[64];
  if (normalize == 0) {
    float acc = part[0];
    for (int idm = 1; idm < m; ++idm) acc += part[idm];
    float nrm = (float)((double)sqrtf(acc) + 1e-16);
    for (int idm = 0; idm < m; ++idm) nrmv[idm] = nrm;
    norms[0] = nrm;
    for (int idm = 1; idm < m; ++idm) norms[idm] = part[idm];
  } else {
    for (int idm = 0; idm < m; ++idm) {
      float nrm = (normalize == 1) ? sqrtf(part[idm]) + 1e-7f
                                   : (float)((double)sqrtf(part[idm]) + 2.220446049250313e-16);
      nrmv[idm] = nrm;
      norms[idm] = nrm;
    }
  }
  for (int b = 0; b < nbin; ++b) {
    out[b] = h[2 * b] / nrmv[b % m];
    out[nbin + b] = h[2 * b + 1] / nrmv[b % m];
  }
  free(h);
  return 0;
}

/* Batch wrappers over forward-packed words (n x W words). */
static void unpack(const uint32_t *w, int k, uint8_t *codes) {
  for (int j = 0; j < k; ++j) codes[j] = (uint8_t)((w[j >> 4] >> (2 * (j & 15))) & 3u);
}

typedef struct {
  const uint32_t *words;
  int k, s, m, c, normalize, W, rdim, f32;
  void *out, *norms;
  volatile int err;
} rope_ctx;

static void rope_body(int64_t f, void *vctx) {
  rope_ctx *x = (rope_ctx *)vctx;
  uint8_t *codes = (uint8_t *)malloc((size_t)x->k);
  unpack(x->words + f * x->W, x->k, codes);
  int e;
  if (x->f32)
    e = orc_rope_frag_f32(codes, x->k, x->s, x->m, x->c, x->normalize, (float *)x->out + f * x->rdim,
                          (float *)x->norms + f * x->m);
  else
    e = orc_rope_frag_f64(codes, x->k, x->s, x->m, x->c, x->normalize, (double *)x->out + f * x->rdim,
                          (double *)x->norms + f * x->m);
  if (e) x->err = e;
  free(codes);
}

static int rope_batch(const uint32_t *words, int64_t n, int k, int s, int m, int c, int normalize,
                      void *out, void *norms, int nthreads, int f32) {
  rope_ctx x = {words, k, s, m, c, normalize, (k + 15) / 16, 2 * (m << (2 * c)), f32, out, norms, 0};
  orc_parallel_for(n, nthreads, rope_body, &x);
  return x.err;
}

int orc_rope_batch_f64(const uint32_t *words, int64_t n, int k, int s, int m, int c, int normalize,
                       double *out, double *norms, int nthreads) {
  return rope_batch(words, n, k, s, m, c, normalize, out, norms, nthreads, 0);
}

int orc_rope_batch_f32(const uint32_t *words, int64_t n, int k, int s, int m, int c, int normalize,
                       float *out, float *norms, int nthreads) {
  return rope_batch(words, n, k, s, m, c, normalize, out, norms, nthreads, 1);
}

/* ------------------------------------------------------------ brute top-k */

/* score = fp32(exact dot of the widened e4m3 operands), then per mode:
 * 0 = fp16-rounded, 1 = fp32, 2 = fp32 * scaleA[row] * scaleB[col]
 * (column scale applied first, as the device epilogue does).  Output
 * (nb, k) descending, ties by ascending column; locs 1-based. */
typedef struct {
  const uint8_t *A, *B;
  int64_t N;
  int rdim, k, mode;
  const float *scaleA, *scaleB;
  float *vals;
  int32_t *locs;
  float lut[256];
} topk_ctx;

static void topk_body(int64_t r, void *vctx) {
  topk_ctx *x = (topk_ctx *)vctx;
  const uint8_t *A = x->A, *B = x->B;
  const int64_t N = x->N;
  const int rdim = x->rdim, k = x->k, mode = x->mode;
  const float *lut = x->lut, *scaleA = x->scaleA, *scaleB = x->scaleB;
  float *vals = x->vals;
  int32_t *locs = x->locs;
  {
    double *a = (double *)malloc(sizeof(double) * rdim);
    float *bv = (float *)malloc(sizeof(float) * k);
    int64_t *bc = (int64_t *)malloc(sizeof(int64_t) * k);
    for (int j = 0; j < k; ++j) {
      bv[j] = -INFINITY;
      bc[j] = INT64_MAX;
    }
    for (int i = 0; i < rdim; ++i) a[i] = lut[A[r * rdim + i]];
    for (int64_t col = 0; col < N; ++col) {
      const uint8_t *b = B + col * rdim;
      double acc = 0.0;
      for (int i = 0; i < rdim; ++i) acc += a[i] * (double)lut[b[i]];
      float sc = (float)acc;
      if (mode == 0) sc = orc_f16_to_f32(orc_f32_to_f16(sc));
      else if (mode == 2) sc = (sc * scaleB[col]);
      /* insert if better than the worst (value desc, column asc) */
      if (sc > bv[k - 1] || (sc == bv[k - 1] && col < bc[k - 1])) {
        int j = k - 1;
        while (j > 0 && (sc > bv[j - 1] || (sc == bv[j - 1] && col < bc[j - 1]))) {
          bv[j] = bv[j - 1];
          bc[j] = bc[j - 1];
          --j;
        }
        bv[j] = sc;
        bc[j] = col;
      }
    }
    for (int j = 0; j < k; ++j) {
      float v = bv[j];
      if (mode == 2) v = v * scaleA[r];
      vals[r * k + j] = v;
      locs[r * k + j] = (bc[j] == INT64_MAX) ? 0 : (int32_t)(bc[j] + 1);
    }
    free(a);
    free(bv);
    free(bc);
  }
}

int orc_topk_e4m3(const uint8_t *A, const uint8_t *B, int64_t nb, int64_t N, int rdim, int k,
                  int mode, const float *scaleA, const float *scaleB, float *vals, int32_t *locs,
                  int nthreads) {
  topk_ctx x;
  x.A = A; x.B = B; x.N = N; x.rdim = rdim; x.k = k; x.mode = mode;
  x.scaleA = scaleA; x.scaleB = scaleB; x.vals = vals; x.locs = locs;
  for (int i = 0; i < 256; ++i) x.lut[i] = orc_e4m3_to_f32((uint8_t)i);
  orc_parallel_for(nb, nthreads, topk_body, &x);
  return 0;
}

/* All scores of one read against every column (mode as above, before the
 * row scale), for tolerance checks of individual values. */
int orc_scores_e4m3(const uint8_t *a8, const uint8_t *B, int64_t N, int rdim, int mode,
                    const float *scaleB, float *scores) {
  float lut[256];
  for (int i = 0; i < 256; ++i) lut[i] = orc_e4m3_to_f32((uint8_t)i);
  for (int64_t col = 0; col < N; ++col) {
    double acc = 0.0;
    for (int i = 0; i < rdim; ++i) acc += (double)lut[a8[i]] * (double)lut[B[col * rdim + i]];
    float sc = (float)acc;
    if (mode == 0) sc = orc_f16_to_f32(orc_f32_to_f16(sc));
    else if (mode == 2) sc = sc * scaleB[col];
    scores[col] = sc;
  }
  return 0;
}
