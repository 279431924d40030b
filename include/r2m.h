/*
 * r2m.h -- C ABI of librotormap_b200.so, the B200 (sm_100a) read-mapping hot
 * path of RotorMap: rope encode -> fp8 read x index GEMM -> per-row top-k.
 *
 * Conventions (every entry point):
 *   - return 0 on success, a negative R2M_E* code on failure; the message of
 *     the last failure on the calling thread is r2m_last_error();
 *   - device pointers are plain CUDA device addresses owned by the caller;
 *     an engine owns only its own workspace;
 *   - `stream` is a cudaStream_t (NULL = the legacy default stream); every
 *     device call is stream-ordered and returns without synchronizing unless
 *     its comment says otherwise (the device FASTA reader learns its record
 *     counts on the host; destroying an engine waits for its work);
 *   - an engine or reader handle serves one thread at a time (its workspace,
 *     events and rebound tensor maps are per handle); different handles may
 *     be used from different threads and streams concurrently;
 *   - index conventions follow the reference: global column ids are 1-based,
 *     0 marks an empty slot whose value is -Inf.
 *
 * Each declaration names the reference function it replaces (file:line in
 * q4bio-qpg/qpg-rotormap, RotorMap/ tree).
 */
#ifndef R2M_H
#define R2M_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *r2m_stream_t; /* cudaStream_t */

enum {
  R2M_OK = 0,
  R2M_EINVAL = -1,   /* bad argument (shape, alignment, range) */
  R2M_ECUDA = -2,    /* a CUDA runtime/driver call failed */
  R2M_ENOMEM = -3,   /* device or host allocation failed */
  R2M_ETIMEOUT = -4, /* a bounded device-side wait gave up (kernel aborted) */
  R2M_ESTATE = -5,   /* wrong object state (e.g. no device, not initialised) */
  R2M_EIO = -6       /* host input could not be read/parsed */
};

/* Output element kinds of the encoders. */
enum {
  R2M_OUT_F32 = 0,        /* fp32 [Re; Im] rows (the kernel's compute type) */
  R2M_OUT_F16 = 1,        /* fp16 RNE rows (the reference stream's fp16 = true) */
  R2M_OUT_E4M3 = 2,       /* e4m3(fp32(fp16(x))): the reference's quantisation, scale 1 */
  R2M_OUT_E4M3_SCALED = 3 /* e4m3(x * 448/amax_row) + fp32 row scale amax_row/448 */
};

/* Score semantics of the fused GEMM + top-k. */
enum {
  R2M_SCORE_F16 = 0,   /* fp32 accumulate, rounded to fp16 (reference cout = :f16) */
  R2M_SCORE_F32 = 1,   /* fp32 accumulate, unrounded (reference cout = :f32) */
  R2M_SCORE_SCALED = 2 /* fp32 accumulate x scaleA[row] x scaleB[col] (per-row scales) */
};

/* Library identity and last error (thread-local). */
const char *r2m_last_error(void);
int r2m_version(void);
/* 0 when a CUDA device of compute capability 10.x is current, else an error. */
int r2m_device_check(void);
/* Synchronizes `stream`, then reports (R2M_ETIMEOUT) and clears a bounded
 * device-side wait that gave up in a kernel of this library since the last
 * check on the current device.  No reference counterpart: the reference's
 * kernels have no bounded waits. */
int r2m_check_device_error(r2m_stream_t stream);
/* Self-check of that mechanism: one CTA waits, with the kernels' bounded
 * wait and a limit of `limit_cycles` SM clocks (<= 4e9), on an mbarrier that
 * nothing arrives on (arrive = 0: the wait gives up and the next
 * r2m_check_device_error reports R2M_ETIMEOUT) or that it completed itself
 * (arrive = 1: no error).  Stream-ordered; touches no caller memory. */
int r2m_selftest_bounded_wait(int64_t limit_cycles, int arrive, r2m_stream_t stream);

/* ---------------------------------------------------------------- encode */

/* Replaces encode_frag_real_batch! (RotorMap/encode/kernel.jl:298-325) and
 * the kernel kernel_rope_frag_real (kernel.jl:86-290).
 * dnas: n * cld(k,16) forward 2-bit words (base j at word j>>4, bits
 * 2*(j&15), zero-padded tail).  dest: (n, 2*m*4^c) row-major of `out_kind`
 * ([Re; Im] split layout).  dest_norms: (n, m) fp32 (row = fragment), the
 * reference's embeds_norms column per fragment.  dest_scales: n fp32 row
 * scales, required for R2M_OUT_E4M3_SCALED, ignored otherwise (may be NULL).
 * normalize in 0..3.  Requires s <= 16, c <= s, 1 <= m <= 8, k >= s. */
int r2m_encode_frag_real_batch(void *dest, int out_kind, float *dest_norms,
                               float *dest_scales, const uint32_t *dnas,
                               int64_t n, int k, int s, int m, int c,
                               int normalize, r2m_stream_t stream);

/* Replaces revcomp_frag_words! / kernel_revcomp_words!
 * (RotorMap/index/build.jl:448-476): drc = reverse complement of each
 * fragment's k bases, forward-packed with a zero tail. */
int r2m_revcomp_frag_words(uint32_t *drc, const uint32_t *dnas, int k,
                           int64_t n, r2m_stream_t stream);

/* Replaces the index builder's encode step (ref_rope_real_stream +
 * build_index_matrix, RotorMap/index/build.jl:547-749): encodes the
 * forward and reverse-complement k-window of every window start into index
 * columns.  genome: packed 2-bit words of all records (each record starting
 * at a word boundary, followed by at least one zero guard word);
 * win_pos[i] = absolute base position (16 * record word offset + 0-based
 * window offset) of window i.  Column layout is the reference's: windows are
 * grouped in batches of `batch_size`; batch b (nb windows) fills columns
 * [2*b*batch_size, 2*b*batch_size + nb) with forward windows and the next nb
 * columns with their reverse complements.  dest: (2*nwin, 2*m*4^c) rows of
 * `out_kind`; dest_norms (2*nwin, m); dest_scales 2*nwin (SCALED only). */
int r2m_encode_ref_windows(void *dest, int out_kind, float *dest_norms,
                           float *dest_scales, const uint32_t *genome,
                           const int64_t *win_pos, int64_t nwin,
                           int64_t batch_size, int k, int s, int m, int c,
                           int normalize, r2m_stream_t stream);

/* Replaces f32_to_f8! (RotorMap/gemm/fp8_convert.jl:100,
 * fp8_ptx.jl:161-166) and the fp16 -> fp32 -> e4m3 step of
 * upload_fp16_as_f8! (RotorMap/search/engine_fp8.jl:355-371):
 * cvt.rn.satfinite e4m3, element-wise over `count` values. */
int r2m_f32_to_e4m3(uint8_t *dst, const float *src, int64_t count,
                    r2m_stream_t stream);
int r2m_f16_to_e4m3(uint8_t *dst, const uint16_t *src, int64_t count,
                    r2m_stream_t stream);

/* ---------------------------------------------------------------- search */

typedef struct r2m_engine r2m_engine;

/* Schedule knobs of the fused GEMM + top-k (0 = automatic). */
typedef struct {
  int splits;  /* column splits per read tile (k-split of the top-k); 0:
                  the CTA-pair kernel with at least half the pairs' worth of
                  read tiles takes 1..8 splits by wave use less ~9% per
                  doubling, smaller batches enough for every CTA */
  int ctas;    /* persistent CTAs (default: SM count) */
  int reserved[6]; /* reserved[0] = 1: record CUDA events around the kernels
                      of every r2m_batch_gemm_topk (see r2m_engine_kernel_ms);
                      reserved[1]: kernel, 0 auto (CTA pairs above 128 reads),
                      1 single-CTA, 2 CTA-pair;
                      reserved[2]: epilogue form of either kernel, 0 auto
                      (CTA-pair kernel: 8 warps for k <= 32; single-CTA
                      kernel: 8 warps for work units of at most 8192 column
                      tiles, else 4), 1 four warps, 2 eight warps (k <= 32);
                      reserved[3]: pacing of the CTA-pair kernel, 0 default
                      (a pair naps while it is more than 16 column tiles
                      ahead of the slowest pair, so the pairs share index
                      tiles through L2), > 0 that window in tiles, < 0 off;
                      reserved[4]: top-k reservoir size per row, 0 auto
                      (the smallest of 8/16/20/32/64 that holds k), else one
                      of those sizes (ignored when smaller than k) */
} r2m_tuning;

/* Replaces TopKEngine(B; k, w, rows_cap, segs, engine, cout)
 * (RotorMap/search/engine_fp8.jl:309-337).  d_B: the resident e4m3 index,
 * N columns of rdim bytes each (the reference's (rdim, N) column-major
 * embeds8; 16-byte aligned).  d_scaleB: N fp32 column scales
 * (R2M_SCORE_SCALED only, else NULL).  rows_cap: largest batch height.
 * 1 <= k <= min(N, 64); rdim % 16 == 0. */
int r2m_engine_create(const uint8_t *d_B, const float *d_scaleB, int rdim,
                      int64_t N, int k, int rows_cap, int score_mode,
                      const r2m_tuning *tune, r2m_engine **out);
int r2m_engine_destroy(r2m_engine *eng);
/* Change an engine's schedule (column splits, persistent CTAs) -- the knob
 * the autotuner of the batching form turns; grows the split workspace when
 * the new schedule needs more (synchronizes the device in that case, so call
 * it outside stream capture).  No reference counterpart (the reference's
 * schedule knobs are the constructor's w / segs). */
int r2m_engine_set_tuning(r2m_engine *eng, const r2m_tuning *tune);
/* The engine's top-k size, row width, score mode, batch height and column
 * count (any pointer may be NULL).  No reference counterpart (the reference
 * reads these from the TopKEngine struct's fields). */
int r2m_engine_info(const r2m_engine *eng, int *k, int *rdim, int *score_mode, int *rows_cap, int64_t *N);
/* Bytes of device workspace the engine holds. */
int64_t r2m_engine_workspace_bytes(const r2m_engine *eng);
/* Device time of the last r2m_batch_gemm_topk's GEMM+top-k kernel and of
 * its split-merge kernel (engines created with tuning.reserved[0] = 1);
 * waits for that call to finish.  No reference counterpart (the reference
 * times whole chunks with _timed_gpu, RotorMap/common/util.jl:67). */
int r2m_engine_kernel_ms(r2m_engine *eng, float *gemm_ms, float *merge_ms, int *splits);

/* Replaces batch_gemm_topk! (RotorMap/search/engine_fp8.jl:399-437) with the
 * cuBLASLt GEMM (fp8_lt.jl:128-168) and seg_rowtopk_merge_kernel!
 * (gemm/topk_kernels.jl:213-329) fused into one tcgen05 kernel plus a
 * split-merge kernel; the score matrix never reaches HBM.
 * d_A: nb rows of rdim e4m3 bytes (row-major, 16-byte aligned rows).
 * d_scaleA: nb fp32 row scales (SCALED only).  Outputs (nb, k) row-major:
 * d_vals fp32 descending, d_locs int32 1-based global column ids.
 * Ties are ordered by ascending column. */
int r2m_batch_gemm_topk(r2m_engine *eng, const uint8_t *d_A,
                        const float *d_scaleA, int nb, float *d_vals,
                        int32_t *d_locs, r2m_stream_t stream);

/* Allocation-free variant of r2m_batch_gemm_topk for callers that cannot
 * allocate device memory when they search: a serving loop where cudaMalloc
 * would synchronize the device and stall its other streams, or a host whose
 * memory pool (CUDA.jl's, PyTorch's caching allocator) already owns the free
 * device memory, so a side allocation can fail.  No counterpart in
 * the reference.  Takes the engine's arguments directly (B, scaleB, rdim, N,
 * k, score_mode as r2m_engine_create; A, scaleA, nb, outputs as
 * r2m_batch_gemm_topk) and calls no cudaMalloc/cudaFree: the pacing slots and
 * the split scratch are a 32 MiB array inside the library that every GPU
 * loading the library holds until exit.  It runs the engine's automatic
 * schedule (CTA pairs above 128 reads, paced), with the column splits cut to
 * what the array holds, so its results equal an automatic engine's.  Limit:
 * ceil(nb/256)*256 rows x the top-k list size (k rounded up to
 * 8/16/20/32/64) x 8 bytes must fit 32 MiB less 8 KiB (nb <= 209,664 at
 * k = 20); larger nb returns R2M_EINVAL.  The first call on a device (and
 * the first after a device reset, which loads the array anew) looks up the
 * array's address and should come before any stream capture.  All calls
 * share the array: calls that overlap on the GPU (other streams, other
 * threads) race and must be serialized by the caller.  A device-side wait
 * that gave up marks every output row with NaN values and location -1. */
int r2m_batch_gemm_topk_noalloc(const uint8_t *d_B, const float *d_scaleB,
                                int rdim, int64_t N, const uint8_t *d_A,
                                const float *d_scaleA, int nb, int k,
                                int score_mode, float *d_vals,
                                int32_t *d_locs, r2m_stream_t stream);
/* Self-check of the allocation-free path's give-up handling, without a
 * fault: the kernels' bounded wait (limit_cycles SM clocks, <= 4e9) on an
 * mbarrier that nothing arrives on gives up and records its code in that
 * path's error word, then the pass that marks a failed search's rows writes
 * NaN / -1 into the (nb, k) outputs.  No reference counterpart. */
int r2m_selftest_noalloc_timeout(int64_t limit_cycles, int nb, int k, float *d_vals, int32_t *d_locs,
                                 r2m_stream_t stream);

/* ------------------------------------------------------- precision form */

/* FP32 exact rescoring of top-k candidates.  No single reference
 * counterpart: the reference scores only in fp8 (RotorMap/search/
 * engine_fp8.jl:20-27) and checks against a CPU fp64 encode
 * (_ref_rope_frag_real, RotorMap/encode/reference.jl:96-105).  For each of
 * nb reads (forward words, as r2m_encode_frag_real_batch) and its kc <= 64
 * candidate columns (1-based ids, e.g. an fp8 top-kc), re-encode the read and
 * every candidate's reference window on the fly from the packed genome
 * (genome / col_pos / strand as r2m_encode_ref_windows writes them; strand 1
 * = reverse complement) in fp32 and score the unquantised embeddings' dot
 * product.  scores (nb, kc) in candidate order (may be NULL); out_vals /
 * out_locs (nb, topk) re-ranked, descending, ties by column. */
int r2m_rescore_fp32(const uint32_t *dnas, int nb, const int32_t *cand, int kc,
                     const uint32_t *genome, const int64_t *col_pos,
                     const uint8_t *strand, int64_t N, int k, int s, int m,
                     int c, int normalize, float *scores, float *out_vals,
                     int32_t *out_locs, int topk, r2m_stream_t stream);

/* FP64 sampled-row check: exact fp64 top-20 of S reads over all N index
 * columns (re-encoded on the fly with the golden fp64 encoder semantics,
 * RotorMap/encode/reference.jl:37-105, normalize = 0) -> d_vals / d_locs
 * (S, 20), descending, ties by column; and, when d_cand is given, the fp64
 * score of each (read, candidate) pair -> d_cand_scores (S, kc).  Allocates
 * its own workspace; synchronizes the stream before returning. */
int r2m_check_fp64(const uint32_t *d_read_words, int S, const uint32_t *d_genome,
                   const int64_t *d_col_pos, const uint8_t *d_strand, int64_t N,
                   int k, int s, int m, int c, const int32_t *d_cand, int kc,
                   double *d_cand_scores, double *d_vals, int32_t *d_locs,
                   r2m_stream_t stream);

/* ------------------------------------------------------------ plain path */

/* The reference engine's own structure on the B200 -- the plain batch path
 * and the GPU bar of the fused kernel.  Replaces the same calls as
 * r2m_engine_create / r2m_batch_gemm_topk (TopKEngine(B; engine = :lt,
 * cout = :f16), RotorMap/search/engine_fp8.jl:309-437) but keeps their
 * mechanics: a cuBLASLt fp8 GEMM (RotorMap/gemm/fp8_lt.jl:128-168) into
 * double-buffered (rows x w) fp16 score chunks in HBM and the segmented top-k
 * merge (RotorMap/gemm/topk_kernels.jl:213-347, segs = 8, k = 20) on a second
 * stream.  d_A must hold ceil(nb/16)*16 rows (the pad rows are scored and
 * dropped).  Outputs (nb, 20) row-major, 1-based ids, the reference's tie
 * order. */
typedef struct r2m_plain_engine r2m_plain_engine;
int r2m_plain_engine_create(const uint8_t *d_B, int rdim, int64_t N, int k,
                            int rows_cap, int w, int segs,
                            r2m_plain_engine **out);
int r2m_plain_engine_destroy(r2m_plain_engine *eng);
int r2m_plain_batch_gemm_topk(r2m_plain_engine *eng, const uint8_t *d_A,
                              int nb, float *d_vals, int32_t *d_locs,
                              r2m_stream_t stream);

/* ---------------------------------------------------------- top-k merge */

/* The merge of a column-sharded search (one rank per index shard, each with
 * its local top-k shifted to global 1-based columns, gathered side by side):
 * d_vals / d_locs hold per row `lists` sorted lists of k entries, laid out
 * [list 0 | list 1 | ...] (nb, lists*k); the row's top-kout under the
 * engine's order (value descending, ties by ascending column; column 0 =
 * empty, last) goes to (nb, kout).  lists <= 32.  Extends the reference's
 * single-device merge (RotorMap/gemm/topk_kernels.jl:213-347) across
 * devices; stream-ordered. */
int r2m_merge_topk_lists(const float *d_vals, const int32_t *d_locs, int lists, int nb, int k, int kout,
                         float *d_out_vals, int32_t *d_out_locs, r2m_stream_t stream);

/* ----------------------------------------------------------- match table */

typedef struct r2m_text r2m_text;

/* Replaces the table writer of run_map (RotorMap/tools/map.jl:141-151): one
 * line per read and top-k hit, "<header without '>'> <+|-> <score> <window
 * start - 1> <record name>\n", the score as Julia's string(::Float32).
 * vals / locs: (nb, k) host arrays (locs 1-based column ids, 1..ncols);
 * heads: nb headers, each followed by '\n'; strand / starts (1-based) /
 * col_rec: per-column index tables; rec_names: the record names (first
 * header token without '>'), each followed by '\n'.  nthreads host threads.
 * A location of -1 (the rows of an allocation-free search whose device-side
 * wait gave up) returns R2M_ETIMEOUT.  Free the text with r2m_text_free. */
int r2m_format_table(const float *vals, const int32_t *locs, int64_t nb, int k, const char *heads,
                     size_t heads_len, const uint8_t *strand, const int64_t *starts, const int32_t *col_rec,
                     int64_t ncols, const char *rec_names, size_t rec_names_len, int nthreads, r2m_text **out);
const char *r2m_text_data(const r2m_text *t, size_t *len);
void r2m_text_free(r2m_text *t);
/* Julia's string(::Float32) of x into out (cap >= 32, NUL-terminated);
 * returns its length, or a negative error code. */
int r2m_format_f32(float x, char *out, size_t cap);

/* ------------------------------------------------------- host-ring engine */

typedef struct r2m_compact r2m_compact;

/* Replaces CompactEngine (RotorMap/search/engine_compact.jl:256-289): the
 * index h_B (N, rdim) e4m3 stays in HOST memory and is streamed through a
 * ring of `depth` device slots of about chunk_cols columns on its own H2D
 * stream.  The first resident_chunks chunks instead get device slots of
 * their own, filled once (an index somewhat larger than the device keeps
 * most of itself resident and streams only the rest).  d_scaleB (scaled
 * scores) is a device vector of N column scales.  pin != 0 page-locks h_B
 * for the engine's lifetime (read-only registration; left pageable when the
 * system refuses).  The host memory must stay valid and unchanged while the
 * engine lives. */
int r2m_compact_create(const uint8_t *h_B, const float *d_scaleB, int rdim, int64_t N, int k, int rows_cap,
                       int score_mode, int64_t chunk_cols, int depth, int resident_chunks, int pin,
                       const r2m_tuning *tune, r2m_compact **out);
int r2m_compact_destroy(r2m_compact *c);
int64_t r2m_compact_chunks(const r2m_compact *c);
int64_t r2m_compact_resident_chunks(const r2m_compact *c);
int r2m_compact_is_pinned(const r2m_compact *c);
/* Replaces batch_gemm_topk_compact! (RotorMap/search/engine_compact.jl:
 * 300-343): the same results as r2m_batch_gemm_topk over the whole index
 * (values, locations and tie order, bit for bit).  Enqueues on `stream`
 * (chunk copies on the engine's H2D stream, ordered by events) and returns;
 * with a pageable h_B each chunk copy holds the host until the slot it
 * refills is free. */
int r2m_compact_batch_gemm_topk(r2m_compact *c, const uint8_t *d_A, const float *d_scaleA, int nb,
                                float *d_vals, int32_t *d_locs, r2m_stream_t stream);

/* ------------------------------------------------------------ host FASTA */

typedef struct r2m_reads r2m_reads;

/* Replaces fasta_reads (RotorMap/fasta/reader.jl:321-350) with _LUT3/_emit3!
 * semantics (reader.jl:21-28,120-198): every record's sequence is packed to
 * forward 2-bit words, trimmed to its first k bases; records with fewer
 * than k bases are skipped; headers are kept verbatim with the '>'.
 * Records are returned in file order.  `data` need not be NUL-terminated. */
int r2m_fasta_reads(const char *data, size_t len, int k, int nthreads,
                    r2m_reads **out);
int64_t r2m_reads_count(const r2m_reads *r);
/* r2m_reads_count(r) * cld(k,16) words, fragment-major. */
const uint32_t *r2m_reads_words(const r2m_reads *r);
/* Header i (not NUL-terminated); its byte length in *len. */
const char *r2m_reads_header(const r2m_reads *r, int64_t i, size_t *len);
/* Bulk header access for hosts that convert many headers at once: every
 * header followed by one '\n' (headers never contain '\n'), total byte
 * length in *total_len, and the r2m_reads_count(r) + 1 byte offsets where
 * each header starts in that blob. */
const char *r2m_reads_header_blob(const r2m_reads *r, size_t *total_len);
const size_t *r2m_reads_header_offsets(const r2m_reads *r);
void r2m_reads_free(r2m_reads *r);

/* ----------------------------------------------------------- host genome */

typedef struct r2m_genome r2m_genome;

/* Reference-genome FASTA -> packed records for the index builder: the
 * record walk of build_index_matrix (RotorMap/index/build.jl:291-324) and
 * the record table of RotorMap/test/harness.jl:52-91 (header to the first
 * '\n' at or after the record start, one trailing '\r' removed; sequence
 * bytes up to the next record start, '\n'/'\r' skipped, A/C/G/T either
 * case -> 0..3, anything else -> 2).  Every record's bases are 2-bit packed
 * from a word boundary and followed by one zero guard word.  nthreads host
 * threads. */
int r2m_fasta_genome(const char *data, size_t len, int nthreads, r2m_genome **out);
int64_t r2m_genome_count(const r2m_genome *g);
const uint32_t *r2m_genome_words(const r2m_genome *g, size_t *nwords);
const int64_t *r2m_genome_word_off(const r2m_genome *g);  /* per record */
const int64_t *r2m_genome_nbases(const r2m_genome *g);    /* per record */
/* every header followed by one '\n' (total bytes in *total_len) */
const char *r2m_genome_header_blob(const r2m_genome *g, size_t *total_len);
void r2m_genome_free(r2m_genome *g);

/* ---------------------------------------------------------- device FASTA */

typedef struct r2m_dreads r2m_dreads;

/* Device counterpart of r2m_fasta_reads (RotorMap/fasta/reader.jl:321-350):
 * d_data is `len` FASTA bytes in device memory.  Same kept records, in file
 * order, with the same words; headers come back as byte spans into d_data
 * (headers are [spans[2i], spans[2i+1]) ).  Runs on `stream` and
 * synchronises it twice (record count, kept count).  Free with
 * r2m_dreads_free. */
int r2m_fasta_reads_device(const void *d_data, size_t len, int k, r2m_stream_t stream, r2m_dreads **out);
int64_t r2m_dreads_count(const r2m_dreads *r);
/* 1 when a record whose header line is not closed ended the parse (that
 * record and everything after it dropped), else 0 -- a caller that feeds a
 * file in pieces cut at record starts stops after such a piece. */
int r2m_dreads_stopped(const r2m_dreads *r);
/* device, r2m_dreads_count(r) x cld(k,16) words */
const uint32_t *r2m_dreads_words(const r2m_dreads *r);
/* device, r2m_dreads_count(r) x 2 int64 header byte spans */
const int64_t *r2m_dreads_spans(const r2m_dreads *r);
/* device, every kept header followed by one '\n' (total bytes in *total_len) */
const uint8_t *r2m_dreads_header_blob(const r2m_dreads *r, size_t *total_len);
void r2m_dreads_free(r2m_dreads *r);

/* ---------------------------------------------------------- serving form */

/* The serving form: a continuous-batching request loop over one fused
 * engine, on the library's own streams and one loop thread.  It replaces the
 * per-file driver loop of run_map (RotorMap/tools/map.jl:100-184, which maps
 * one read file at a time through rope_topk_stream_compact in synchronous
 * batches) for hosts that map many requests at once: requests of any size
 * arrive from any thread; each is admitted, in arrival order, when its
 * device state (words + result lists, r2m_server_request_bytes) fits both
 * the byte budget and the device memory free at that moment less
 * `hbm_reserve`; every GPU batch is cut from all admitted requests (a
 * request that arrives while others run joins the next batch).  A read's
 * result does not depend on the batch it lands in.  Cancelling a queued
 * request drops it; cancelling an admitted one stops its remaining rows and
 * frees it once its rows in flight are done, leaving other requests
 * untouched.  A failed CUDA call fails every unfinished request with that
 * first error and closes the server (first error wins, as the reference's
 * err_out, RotorMap/encode/stream.jl:95-110). */
typedef struct r2m_server r2m_server;

enum { R2M_REQ_QUEUED = 0, R2M_REQ_ACTIVE = 1, R2M_REQ_DONE = 2, R2M_REQ_CANCELLED = 3, R2M_REQ_FAILED = 4 };

typedef struct {
  int64_t batches, rows, max_rows;          /* GPU batches launched, rows in them, tallest */
  int64_t requests_done, requests_cancelled, requests_failed;
  int64_t in_use_bytes, peak_in_use_bytes;  /* admitted requests' device state */
  int64_t queued, active;                   /* requests waiting / admitted now */
} r2m_server_stats;

/* eng: a fused engine (its rows_cap is the batch height, its score mode the
 * quantisation: scaled e4m3 rows for R2M_SCORE_SCALED, else the reference's
 * e4m3); (k, s, m, c, normalize): the encoder, matching the engine's row
 * width.  hbm_budget 0 = no byte budget (free memory alone); max_inflight:
 * GPU batches queued ahead (0 = 2).  The engine must outlive the server and
 * must not be used by others meanwhile. */
int r2m_server_create(r2m_engine *eng, int k, int s, int m, int c, int normalize, int64_t hbm_budget,
                      int64_t hbm_reserve, int max_inflight, r2m_server **out);
/* Submit n reads (h_words: n * cld(k,16) forward 2-bit words).  Results go
 * to the caller's h_vals / h_locs (n, k) when the request is done; all three
 * buffers must stay valid until then (page-locked buffers are copied
 * asynchronously, pageable ones synchronously by the loop thread).
 * t_arrival: CLOCK_MONOTONIC seconds of the arrival (<= 0: now).  A request
 * larger than the byte budget returns R2M_ENOMEM. */
int r2m_server_submit(r2m_server *srv, const uint32_t *h_words, int64_t n, float *h_vals, int32_t *h_locs,
                      double t_arrival, int64_t *id);
/* Submit FASTA bytes (parsed now by r2m_fasta_reads with the reference's
 * trim / skip rules; the reads' headers: r2m_server_reads).  Input that does
 * not start with a '>' header, or keeps no read of k bases, returns R2M_EIO.
 * Results: r2m_server_copy_result. */
int r2m_server_submit_fasta(r2m_server *srv, const char *data, size_t len, int nthreads, double t_arrival,
                            int64_t *id, int64_t *n_reads);
int r2m_server_cancel(r2m_server *srv, int64_t id);
/* Block until the request has finished (timeout_s < 0: no limit; R2M_ETIMEOUT
 * when it runs out); *state = its R2M_REQ_* state. */
int r2m_server_wait(r2m_server *srv, int64_t id, double timeout_s, int *state);
/* State, read count and CLOCK_MONOTONIC times of a request. */
int r2m_server_request(r2m_server *srv, int64_t id, int *state, int64_t *n, double *t_arrival,
                       double *t_admit, double *t_done);
const char *r2m_server_request_error(r2m_server *srv, int64_t id);
/* Copy a done request's results (needed for FASTA requests; a no-op copy
 * for the caller's own buffers). */
int r2m_server_copy_result(r2m_server *srv, int64_t id, float *h_vals, int32_t *h_locs);
const r2m_reads *r2m_server_reads(r2m_server *srv, int64_t id);
/* Forget a finished request (its id becomes unknown). */
int r2m_server_release(r2m_server *srv, int64_t id);
int r2m_server_get_stats(r2m_server *srv, r2m_server_stats *out);
int64_t r2m_server_request_bytes(const r2m_server *srv, int64_t n);
/* Stop the loop: finish every request first (cancel_pending = 0) or cancel
 * the unfinished ones; frees the server.  Returns the first loop failure. */
int r2m_server_destroy(r2m_server *srv, int cancel_pending);

/* ------------------------------------------- reference index file (.bin) */

/* The reference's index file is a Julia `Serialization` stream of one
 * NamedTuple (save / load, RotorMap/common/dna.jl:23-34; the fields of
 * _index_data_nt, RotorMap/index/build.jl:755-772).  These entry points read
 * and write the subset of that format such a NamedTuple uses: Int64, Bool and
 * String fields, arrays of bits types (UInt8, Int32, Int64, Float16, Float32,
 * Float64, DLFP8Types.Float8_E4M3FN) and Vector{String}. */
typedef struct r2m_jlbin r2m_jlbin;

enum { R2M_JL_OTHER = 0, R2M_JL_INT = 1, R2M_JL_BOOL = 2, R2M_JL_STRING = 3, R2M_JL_ARRAY = 4,
       R2M_JL_STRVEC = 5 };
enum { R2M_JL_U8 = 1, R2M_JL_I32 = 2, R2M_JL_I64 = 3, R2M_JL_F16 = 4, R2M_JL_F32 = 5, R2M_JL_F64 = 6,
       R2M_JL_E4M3 = 7 };

/* One NamedTuple field.  Arrays are Julia-shaped: dims[0] is the fastest
 * (column-major) dimension, so embeds8 (rdim, N) holds N columns of rdim
 * bytes back to back.  A Vector{String} (R2M_JL_STRVEC) is given as its
 * distinct strings (blob + nuniq + 1 offsets uniq_off) and, in data, one
 * int32 index into them per element. */
typedef struct {
  const char *name;     /* field name, NUL-terminated */
  int kind;             /* R2M_JL_* kind */
  int elty;             /* R2M_JL_ARRAY element type */
  int64_t ival;         /* R2M_JL_INT value, R2M_JL_BOOL 0/1 */
  const char *str;      /* R2M_JL_STRING bytes (not NUL-terminated) */
  int64_t str_len;
  int ndims;            /* arrays: 1 or 2 */
  int64_t dims[2];
  const void *data;     /* array elements; STRVEC: int32 per element */
  int64_t offset;       /* read side: byte offset of `data` in the file (-1 if none) */
  const char *blob;     /* STRVEC distinct strings, concatenated */
  const int64_t *uniq_off; /* STRVEC: nuniq + 1 offsets into blob */
  int64_t nuniq;
} r2m_jl_field;

/* Replaces `load` of an index .bin (RotorMap/common/dna.jl:30-34, called by
 * load_index, RotorMap/index/load.jl:49-73): memory-maps the file and parses
 * the NamedTuple; array payloads point into the mapping and stay valid until
 * r2m_jlbin_close.  R2M_EIO names the first byte the reader does not accept.
 * r2m_jlbin_parse reads a stream already in memory (kept by the caller). */
int r2m_jlbin_open(const char *path, r2m_jlbin **out);
int r2m_jlbin_parse(const void *data, size_t len, r2m_jlbin **out);
int r2m_jlbin_version(const r2m_jlbin *b);  /* the stream's format version byte */
int r2m_jlbin_nfields(const r2m_jlbin *b);
int r2m_jlbin_field(const r2m_jlbin *b, int i, r2m_jl_field *out);
void r2m_jlbin_close(r2m_jlbin *b);
/* Replaces `save` of an index (RotorMap/common/dna.jl:23-27, called by
 * run_save, RotorMap/index/build.jl:781-795): writes the NamedTuple of
 * `fields` in order as the stream Julia's `deserialize` reads back (Int64,
 * Bool, String, arrays, Vector{String} with repeated strings longer than 7
 * bytes written once and referenced after). */
int r2m_jlbin_write(const char *path, const r2m_jl_field *fields, int nfields);

#ifdef __cplusplus
}
#endif

#endif /* R2M_H */
