// gemm_topk.cu -- the read x index similarity search: a persistent tcgen05
// fp8 GEMM whose epilogue is a streaming per-row top-k, plus the merge of
// the per-split partial lists and the engine object behind the C ABI.
//
// Replaces the reference's chunk loop batch_gemm_topk!
// (RotorMap/search/engine_fp8.jl:399-437): cuBLASLt fp8 GEMM into an fp16 C
// chunk in HBM (gemm/fp8_lt.jl:128-168) followed by seg_rowtopk_merge_kernel!
// (gemm/topk_kernels.jl:213-329).  Here the score tile lives only in TMEM.
//
// Kernel structure (one CTA per SM, 192 threads):
//   warp 0      TMA producer: A tile (128 reads x 128 B of K) and B tile
//               (256 index columns x 128 B) per stage, 128-byte swizzle,
//               4-stage mbarrier ring, no multicast.
//   warp 1      TMEM owner + MMA issuer: tcgen05.mma kind::f8f6f4,
//               M=128 N=256 K=32, fp32 accumulators double-buffered in TMEM
//               (2 x 256 of the 512 columns).
//   warps 2..5  epilogue: one thread per read row (TMEM lane); tcgen05.ld of
//               32 columns at a time (the next chunk in flight while one is
//               scored), score transform (fp16 rounding / column scale),
//               chunk max vs the row's threshold, and insertion into a
//               register reservoir of the top KT (score desc, column asc).
// Work unit = (read tile of 128 rows, column split); each unit streams its
// split's column tiles and leaves a sorted partial list per row; a second
// kernel merges the splits.  Every mbarrier wait is bounded; a wait that
// gives up raises a shared abort flag, records a code in the device error
// word and the CTA drains its in-flight work before freeing TMEM.
#include <float.h>
#include <limits.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace r2m {

constexpr int BM = 128;           // read rows per tile (TMEM lanes)
constexpr int BN = 256;           // index columns per tile (TMEM fp32 columns)
constexpr int BK = 128;           // K bytes per stage (one 128-byte swizzle row)
constexpr int STAGES = 4;
constexpr int A_STAGE = BM * BK;  // 16 KiB
constexpr int B_STAGE = BN * BK;  // 32 KiB
constexpr int TMEM_COLS = 512;
constexpr long long WAIT_LIMIT = 4000000000LL;  // clock cycles (~2 s)
constexpr int MAX_SPLITS = 128;
// Epilogue forms of both kernels: 4 * H epilogue warps.  With H = 2 two warps
// share each TMEM lane quarter, each draining one half (128 columns) of
// every tile into its own reservoir, so a (read tile, column split) unit
// leaves two partial lists per row.  That halves the per-warp latency chain
// of a tile and the reservoir warm-up at every unit start.  The CTA-pair
// kernel always takes it (k <= 32): its epilogue must drain a tile in the
// time its MMAs take one, and with 4 warps it held the MMAs back (headline
// launch, same box: 1,553 ms per launch with 4 epilogue warps, 1,530 ms with
// 8).  The single-CTA kernel takes it for short units only: on long units
// the extra warps cost clock under the board's power cap.  The host picks H
// per launch (epi_halves_for).  KT = 64 always uses H = 1 (its reservoir
// needs the registers).
__host__ __device__ constexpr int epi_threads(int H) { return 64 + 128 * H; }
constexpr int SCRATCH_F = 17;  // floats per epilogue thread (16-value slow-path passes)
// 256-column tiles per work unit at or below which the 8-warp epilogue pays
constexpr int SHORT_UNIT_TILES = 8192;

struct GemmArgs {
  int nb;
  int num_m_tiles;
  long long N;
  int n_tiles;
  int splits;
  int num_kb;
  int score_mode;
  int mpad;  // num_m_tiles * BM (partial-list row stride)
  const float *scaleB;
  float *part_vals;
  int *part_cols;
  uint32_t *err;
  long long *pace;  // CTA-pair kernel: per-pair progress (null = no pacing)
  int pace_window;  // column tiles a pair may run ahead of the slowest one
};

__device__ __forceinline__ int split_lo(int s, int n_tiles, int splits) {
  return (int)(((long long)s * n_tiles) / splits);
}

__device__ __forceinline__ float round_f16(float x) { return __half2float(__float2half_rn(x)); }

// The best KT (value, column) pairs of one row, kept sorted in registers:
// larger value first, equal values -> smaller column first.  `thr` is the
// worst kept value.  Insertion is branch-free: the new entry's rank is a sum
// of independent compares and every slot picks (old, shifted, new) with two
// selects, so there is no dependent chain through the list.
template <int KT>
struct Reservoir {
  float v[KT];
  int c[KT];
  float thr;

  __device__ __forceinline__ void reset() {
#pragma unroll
    for (int i = 0; i < KT; ++i) {
      v[i] = -INFINITY;
      c[i] = INT_MAX;
    }
    thr = -INFINITY;
  }
  // Called only with x > thr and a column larger than every kept column (the
  // scan runs in increasing column order), so the rank is #{v[i] >= x}.
  __device__ __forceinline__ void insert(float x, int col) {
    int p = 0;
#pragma unroll
    for (int i = 0; i < KT; ++i) p += (v[i] >= x) ? 1 : 0;
#pragma unroll
    for (int i = KT - 1; i > 0; --i) {
      const bool shift = i > p, here = i == p;
      v[i] = shift ? v[i - 1] : (here ? x : v[i]);
      c[i] = shift ? c[i - 1] : (here ? col : c[i]);
    }
    if (p == 0) {
      v[0] = x;
      c[0] = col;
    }
    thr = v[KT - 1];
  }
  __device__ __forceinline__ void sort_desc() {}
};

// Column scales of one 32-column chunk: broadcast loads (every lane of the
// warp reads the same 128 bytes).  Past the index end they read as 1; those
// columns are masked to -inf before scoring.
__device__ __forceinline__ void load_scales(float4 (&s)[8], const float *scaleB, long long c0, long long N,
                                            bool tail) {
  if (!tail) {
    const float4 *p = reinterpret_cast<const float4 *>(scaleB + c0);
#pragma unroll
    for (int q = 0; q < 8; ++q) s[q] = __ldg(p + q);
  } else {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long c = c0 + 4 * q;
      s[q].x = c < N ? __ldg(scaleB + c) : 1.f;
      s[q].y = c + 1 < N ? __ldg(scaleB + c + 1) : 1.f;
      s[q].z = c + 2 < N ? __ldg(scaleB + c + 2) : 1.f;
      s[q].w = c + 3 < N ? __ldg(scaleB + c + 3) : 1.f;
    }
  }
}

__device__ __forceinline__ void apply_scales(float (&v)[32], const float4 (&s)[8]) {
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    v[4 * q] *= s[q].x;
    v[4 * q + 1] *= s[q].y;
    v[4 * q + 2] *= s[q].z;
    v[4 * q + 3] *= s[q].w;
  }
}

// Score one 32-column chunk of this thread's row (columns c0 .. c0+31): the
// chunk max (a depth-5 tree over 8 partial maxima) against the row's threshold decides whether the
// chunk goes through the insert path, staged 16 values at a time in `scratch`.
template <int KT>
__device__ __forceinline__ void score_chunk(Reservoir<KT> &R, float (&v)[32], long long c0, long long N, bool tail,
                                            bool f16, float *scratch) {
  if (tail) {
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (c0 + j >= N) v[j] = -INFINITY;
  }
  float m[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) m[j] = fmaxf(fmaxf(v[j], v[j + 8]), fmaxf(v[j + 16], v[j + 24]));
#pragma unroll
  for (int w = 4; w >= 1; w >>= 1)
#pragma unroll
    for (int j = 0; j < w; ++j) m[j] = fmaxf(m[j], m[j + w]);
  float mx = m[0];
  if (f16) mx = round_f16(mx);
  if (mx > R.thr) {
#pragma unroll
    for (int p = 0; p < 2; ++p) {
#pragma unroll
      for (int j = 0; j < 16; ++j) scratch[j] = v[16 * p + j];
#pragma unroll 1
      for (int j = 0; j < 16; ++j) {
        float x = scratch[j];
        if (f16) x = round_f16(x);
        if (x > R.thr) R.insert(x, (int)(c0 + 16 * p + j));
      }
    }
  }
}

// Drain this warp's CH chunks of one accumulator tile (TMEM address `taddr`
// = its lane quarter and first chunk; columns c_first .. c_first + 32 CH - 1)
// into the row's reservoir.  Software-pipelined: the TMEM load and the column
// scales of chunk i + 1 are in flight while chunk i is scored.  Every load is
// waited for before returning, so the caller may release the accumulator.
template <int KT, int CH>
__device__ __forceinline__ void drain_tile(Reservoir<KT> &R, uint32_t taddr, long long c_first, long long N,
                                           const float *scaleB, bool scaled, bool f16, float *scratch) {
  static_assert(CH % 2 == 0, "chunks are drained in pairs");
  const bool tail = c_first + 32LL * CH > N;
  float va[32], vb[32];
  float4 s[8];
  __syncwarp();
  tmem_ld32(taddr, va);
  if (scaled) load_scales(s, scaleB, c_first, N, tail);
#pragma unroll 1
  for (int i = 0; i < CH; i += 2) {
    const long long c0 = c_first + 32LL * i;
    __syncwarp();
    tmem_wait_ld_tied(va);
    if (scaled) apply_scales(va, s);
    tmem_ld32(taddr + (uint32_t)(i + 1) * 32u, vb);
    if (scaled) load_scales(s, scaleB, c0 + 32, N, tail);
    score_chunk(R, va, c0, N, tail, f16, scratch);
    __syncwarp();
    tmem_wait_ld_tied(vb);
    if (scaled) apply_scales(vb, s);
    if (i + 2 < CH) {
      tmem_ld32(taddr + (uint32_t)(i + 2) * 32u, va);
      if (scaled) load_scales(s, scaleB, c0 + 64, N, tail);
    }
    score_chunk(R, vb, c0 + 32, N, tail, f16, scratch);
  }
}

// The same, one chunk at a time: for the 8-warp form with a 32-entry
// reservoir, whose 168-register budget has no room for a second chunk.
template <int KT, int CH>
__device__ __forceinline__ void drain_tile_serial(Reservoir<KT> &R, uint32_t taddr, long long c_first, long long N,
                                                  const float *scaleB, bool scaled, bool f16, float *scratch) {
  const bool tail = c_first + 32LL * CH > N;
#pragma unroll 1
  for (int i = 0; i < CH; ++i) {
    const long long c0 = c_first + 32LL * i;
    float v[32];
    float4 s[8];
    __syncwarp();
    if (scaled) load_scales(s, scaleB, c0, N, tail);
    tmem_ld32(taddr + (uint32_t)i * 32u, v);
    tmem_wait_ld_tied(v);
    if (scaled) apply_scales(v, s);
    score_chunk(R, v, c0, N, tail, f16, scratch);
  }
}

template <int KT, int H>
__device__ __forceinline__ void drain_acc(Reservoir<KT> &R, uint32_t taddr, long long c_first, long long N,
                                      const float *scaleB, bool scaled, bool f16, float *scratch) {
  constexpr int CH = BN / 32 / H;
  if constexpr (H == 1 || KT < 32)
    drain_tile<KT, CH>(R, taddr, c_first, N, scaleB, scaled, f16, scratch);
  else
    drain_tile_serial<KT, CH>(R, taddr, c_first, N, scaleB, scaled, f16, scratch);
}

template <int KT, int H>
__global__ void __launch_bounds__(epi_threads(H), 1)
    k_gemm_topk(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem =
      reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *sA = smem;
  uint8_t *sB = smem + STAGES * A_STAGE;
  uint64_t *full = reinterpret_cast<uint64_t *>(sB + STAGES * B_STAGE);
  uint64_t *empty = full + STAGES;
  uint64_t *acc_full = empty + STAGES;
  uint64_t *acc_empty = acc_full + 2;
  uint64_t *drain = acc_empty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  float *scratch_all = reinterpret_cast<float *>(tmem_slot + 4);  // epilogue threads x SCRATCH_F floats

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 4 * H);  // epilogue warps
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const int num_units = g.num_m_tiles * g.splits;

  if (warp == 0) {
    // ------------------------------------------------ TMA producer
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      long long issued = 0;
      bool ok = true;
      for (int u = blockIdx.x; ok && u < num_units; u += gridDim.x) {
        const int mt = u % g.num_m_tiles, sp = u / g.num_m_tiles;
        const int t0 = split_lo(sp, g.n_tiles, g.splits), t1 = split_lo(sp + 1, g.n_tiles, g.splits);
        for (int t = t0; ok && t < t1; ++t) {
          for (int kb = 0; kb < g.num_kb; ++kb) {
            if (!mbar_wait_bounded(&empty[stage], phase ^ 1u, abort_flag, WAIT_LIMIT)) {
              if (!*abort_flag) atomicExch(g.err, kErrTimeoutEmpty);
              *abort_flag = 1;
              ok = false;
              break;
            }
            mbar_arrive_expect_tx(&full[stage], A_STAGE + B_STAGE);
            tma_load_2d(sA + stage * A_STAGE, &tmA, &full[stage], kb * BK, mt * BM);
            tma_load_2d(sB + stage * B_STAGE, &tmB, &full[stage], kb * BK, t * BN);
            ++issued;
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
        }
      }
      if (!ok) {
        // let the copies already issued land before the CTA can exit
        int nlast = issued < STAGES ? (int)issued : STAGES;
        for (int j = 1; j <= nlast; ++j) {
          int s = stage - j;
          uint32_t ph = phase;
          if (s < 0) {
            s += STAGES;
            ph ^= 1u;
          }
          long long t0 = clock64();
          while (!mbar_try_wait(&full[s], ph) && clock64() - t0 < WAIT_LIMIT) {
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t idesc = idesc_e4m3_f32(BM, BN);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (int u = blockIdx.x; ok && u < num_units; u += gridDim.x) {
        const int sp = u / g.num_m_tiles;
        const int t0 = split_lo(sp, g.n_tiles, g.splits), t1 = split_lo(sp + 1, g.n_tiles, g.splits);
        for (int t = t0; ok && t < t1; ++t) {
          if (!mbar_wait_bounded(&acc_empty[acc], acc_phase ^ 1u, abort_flag, WAIT_LIMIT)) {
            if (!*abort_flag) atomicExch(g.err, kErrTimeoutAccEmpty);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
          for (int kb = 0; kb < g.num_kb; ++kb) {
            if (!mbar_wait_bounded(&full[stage], phase, abort_flag, WAIT_LIMIT)) {
              if (!*abort_flag) atomicExch(g.err, kErrTimeoutFull);
              *abort_flag = 1;
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA + stage * A_STAGE);
            const uint32_t b0 = smem_u32(sB + stage * B_STAGE);
#pragma unroll
            for (int kk = 0; kk < BK / 32; ++kk) {
              mma_f8(d_tmem, smem_desc_sw128(a0 + kk * 32), smem_desc_sw128(b0 + kk * 32), idesc,
                     (kb | kk) != 0 ? 1u : 0u);
            }
            mma_commit(&empty[stage]);
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
          if (!ok) break;
          mma_commit(&acc_full[acc]);
          acc ^= 1;
          if (acc == 0) acc_phase ^= 1u;
        }
      }
      // every MMA issued by this thread has completed once `drain` flips
      mma_commit(drain);
      long long t0 = clock64();
      while (!mbar_try_wait(drain, 0) && clock64() - t0 < WAIT_LIMIT) {
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------ epilogue (top-k)
    constexpr int CH = BN / 32 / H;  // 32-column chunks per warp and tile
    const int quarter = warp & 3;    // TMEM lanes [32*quarter, 32*quarter+32)
    const int half = (warp - 2) >> 2;  // tile chunks [CH half, CH half + CH)
    const int row_in_tile = quarter * 32 + lane;
    float *scratch = scratch_all + (threadIdx.x - 64) * SCRATCH_F;
    const bool f16 = g.score_mode == R2M_SCORE_F16;
    const bool scaled = g.score_mode == R2M_SCORE_SCALED;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    Reservoir<KT> R;
    for (int u = blockIdx.x; ok && u < num_units; u += gridDim.x) {
      const int mt = u % g.num_m_tiles, sp = u / g.num_m_tiles;
      const int t0 = split_lo(sp, g.n_tiles, g.splits), t1 = split_lo(sp + 1, g.n_tiles, g.splits);
      R.reset();
      for (int t = t0; t < t1; ++t) {
        bool w = mbar_wait_bounded(&acc_full[acc], acc_phase, abort_flag, WAIT_LIMIT);
        if (__any_sync(FULL, !w)) {
          if (lane == 0 && !*abort_flag) atomicExch(g.err, kErrTimeoutAccFull);
          *abort_flag = 1;
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN + half * CH * 32);
        drain_acc<KT, H>(R, taddr, (long long)t * BN + half * CH * 32, g.N, g.scaleB, scaled, f16, scratch);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[acc]);
        acc ^= 1;
        if (acc == 0) acc_phase ^= 1u;
      }
      if (!ok) break;
      R.sort_desc();
      const int row = mt * BM + row_in_tile;
      if (row < g.nb) {
        const size_t list = (size_t)sp * H + half;
        float *pv = g.part_vals + (list * g.mpad + row) * KT;
        int *pc = g.part_cols + (list * g.mpad + row) * KT;
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          pv[j] = R.v[j];
          pc[j] = R.c[j];
        }
      }
    }
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, TMEM_COLS);
  }
}

// ------------------------------------------------------------------
// 2-SM variant: a CTA pair (cluster of 2) computes a 256-read x 256-column
// tile with tcgen05.mma.cta_group::2 (M = 256, N = 256, K = 32).  Each CTA
// loads its own 128 read rows and its own 128 of the 256 index columns per
// K chunk (32 KiB instead of 48 KiB per CTA), so a CTA pulls 2/3 of the
// single-CTA kernel's operand bytes per FLOP.  The leader CTA (rank 0)
// issues the MMAs; both CTAs' TMA loads complete on the leader's stage
// barrier; the leader's commits release both CTAs' stages and signal both
// CTAs' accumulators; each CTA's epilogue drains its own 128 TMEM lanes (all
// 256 columns) and arrives on the leader's accumulator-empty barrier.  No
// load uses multicast.
//
// A stage holds two 128-byte K chunks (8 MMAs), and one commit releases it in
// both CTAs (the commit's arrive goes to the barrier at the same offset in
// each CTA of the mask).  The one issuing thread is what bounds this kernel:
// per stage it waits on the stage barrier, forms descriptors, issues the
// MMAs and commits.  With one chunk and two commits per stage that took ~730
// SM clocks against 512 of tensor work (clock64 probes on the headline
// launch, 65,536 reads x 16.8M columns), so the tensor pipe idled ~30% of the
// time.  Same-box A/B, identical results: 1,697 ms per launch -> 1,553 ms
// with two chunks per stage, one commit and precomputed descriptors; three
// chunks per stage (two stages in flight) 1,800 ms; one commit to the leader
// passed on to the peer by the leader's producer (the peer's loads then
// start later) 1,983 ms.
constexpr int HALF_TILE = 128 * BK;            // 16 KiB: one 128-byte K chunk of 128 rows
constexpr int KCH = 2;                         // K chunks per stage
constexpr int STAGES2 = 3;                     // stages in flight (3 x 64 KiB per CTA)
constexpr int STAGE2_BYTES = KCH * HALF_TILE;  // per operand and CTA

// Pair pacing.  Every pair streams the index in column order, and the pairs
// of one wave (units p, p + npairs, ... run side by side) read the same index
// tiles, so a tile comes from DRAM once and from L2 for the other pairs --
// while the pairs stay within an L2's worth of tiles of each other.  Left
// alone they drift apart over a long unit, and then every pair streams the
// index from DRAM itself.  So each pair's producer publishes its position
// (column tiles issued since the launch; -1 = not started, LLONG_MAX = done)
// every PACE_EVERY tiles and, while it is more than `window` tiles ahead of
// the slowest started pair, sleeps -- for at most PACE_CHECKS short naps.
// Pacing only ever delays a pair a little: it never waits for a pair that is
// not running, nor for one more than PACE_LOST windows behind (a pair that
// started late, e.g. on a GPU shared with other work, is outside any shared
// L2 range and cannot be waited out), and it cannot stall the launch.
// Same-box sweep on 65,536 reads x 16.8M columns (mean of two launches):
// no pacing 1,761 ms; window 16 checked every 16 tiles 1,667 ms; windows of
// 32 / 64 / 128 tiles 1,693 / 1,717 / 1,732 ms; tighter windows or checks
// every 8 or 4 tiles 1,698-1,837 ms (the naps and reads start to cost).
constexpr int PACE_EVERY = 16;
constexpr int PACE_CHECKS = 16;
constexpr int PACE_WINDOW = 16;  // tiles of 256 columns: 8 MiB of a 2048-byte index
constexpr int PACE_LOST = 8;     // windows behind which a pair is no longer waited for

__device__ __forceinline__ void pace_pair(long long *pace, int pair, int npairs, long long pos, int window) {
  volatile long long *p = pace;
  p[pair] = pos;
  for (int it = 0; it < PACE_CHECKS; ++it) {
    const long long lost = pos - (long long)PACE_LOST * window;
    long long mn = LLONG_MAX;
    for (int q = 0; q < npairs; ++q) {
      const long long v = p[q];
      if (v >= 0 && v >= lost && v < mn) mn = v;
    }
    if (pos - mn <= window) return;
    __nanosleep(1000);
  }
}
// CTA-pair kernel: TMA warp, MMA warp and 4 * H epilogue warps (epilogue
// forms above).
template <int KT, int H>
__global__ void __launch_bounds__(epi_threads(H), 1)
    k_gemm_topk2(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem =
      reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *sA = smem;
  uint8_t *sB = smem + STAGES2 * STAGE2_BYTES;
  uint64_t *full = reinterpret_cast<uint64_t *>(sB + STAGES2 * STAGE2_BYTES);
  uint64_t *empty = full + STAGES2;
  uint64_t *acc_full = empty + STAGES2;
  uint64_t *acc_empty = acc_full + 2;
  uint64_t *drain = acc_empty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  float *scratch_all = reinterpret_cast<float *>(tmem_slot + 4);  // epilogue threads x SCRATCH_F floats

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES2; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&acc_full[a], 1);
      mbar_init(&acc_empty[a], 2 * 4 * H);  // epilogue warps x 2 CTAs (leader's copy is used)
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_slot, TMEM_COLS);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // both CTAs' barriers are initialised before any remote arrive
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int num_units = g.num_m_tiles * g.splits;

  if (warp == 0) {
    // ------------------------------------------------ TMA producer (both CTAs)
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      long long issued = 0;
      long long pos = 0;  // column tiles this pair issued in earlier units
      const bool pacing = leader && g.pace != nullptr;
      bool ok = true;
      for (int u = pair; ok && u < num_units; u += npairs) {
        const int mt = u % g.num_m_tiles, sp = u / g.num_m_tiles;
        const int t0 = split_lo(sp, g.n_tiles, g.splits), t1 = split_lo(sp + 1, g.n_tiles, g.splits);
        for (int t = t0; ok && t < t1; ++t) {
          if (pacing && (t - t0) % PACE_EVERY == 0) pace_pair(g.pace, pair, npairs, pos + (t - t0), g.pace_window);
          for (int kb = 0; kb < g.num_kb; kb += KCH) {
            if (!mbar_wait_bounded(&empty[stage], phase ^ 1u, abort_flag, WAIT_LIMIT)) {
              if (!*abort_flag) atomicExch(g.err, kErrTimeoutEmpty);
              *abort_flag = 1;
              ok = false;
              break;
            }
            const uint32_t fbar = mapa_shared(smem_u32(&full[stage]), 0);
            const int nch = g.num_kb - kb < KCH ? g.num_kb - kb : KCH;
            if (leader) mbar_arrive_expect_tx(&full[stage], 4 * HALF_TILE * nch);
            for (int c = 0; c < nch; ++c) {
              tma_load_2d_pair(sA + stage * STAGE2_BYTES + c * HALF_TILE, &tmA, fbar, (kb + c) * BK,
                               mt * 256 + (int)rank * 128);
              tma_load_2d_pair(sB + stage * STAGE2_BYTES + c * HALF_TILE, &tmB, fbar, (kb + c) * BK,
                               t * BN + (int)rank * 128);
            }
            ++issued;
            if (++stage == STAGES2) {
              stage = 0;
              phase ^= 1u;
            }
          }
        }
        pos += t1 - t0;
      }
      if (pacing) reinterpret_cast<volatile long long *>(g.pace)[pair] = LLONG_MAX;  // holds no one back
      if (!ok && leader) {
        int nlast = issued < STAGES2 ? (int)issued : STAGES2;
        for (int j = 1; j <= nlast; ++j) {
          int s = stage - j;
          uint32_t ph = phase;
          if (s < 0) {
            s += STAGES2;
            ph ^= 1u;
          }
          long long c0 = clock64();
          while (!mbar_try_wait(&full[s], ph) && clock64() - c0 < WAIT_LIMIT) {
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer (leader CTA)
    if (lane == 0 && leader) {
      const uint32_t idesc = idesc_e4m3_f32(256, BN);
      // descriptors of stage 0; a stage / chunk / K step offset adds its
      // 16-byte units to the start-address field
      const uint64_t dA0 = smem_desc_sw128(smem_u32(sA)), dB0 = smem_desc_sw128(smem_u32(sB));
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (int u = pair; ok && u < num_units; u += npairs) {
        const int sp = u / g.num_m_tiles;
        const int t0 = split_lo(sp, g.n_tiles, g.splits), t1 = split_lo(sp + 1, g.n_tiles, g.splits);
        for (int t = t0; ok && t < t1; ++t) {
          if (!mbar_wait_bounded(&acc_empty[acc], acc_phase ^ 1u, abort_flag, WAIT_LIMIT)) {
            if (!*abort_flag) atomicExch(g.err, kErrTimeoutAccEmpty);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
          for (int kb = 0; kb < g.num_kb; kb += KCH) {
            if (!mbar_wait_bounded(&full[stage], phase, abort_flag, WAIT_LIMIT)) {
              if (!*abort_flag) atomicExch(g.err, kErrTimeoutFull);
              *abort_flag = 1;
              ok = false;
              break;
            }
            tc_fence_after();
            const int nch = g.num_kb - kb < KCH ? g.num_kb - kb : KCH;
            const uint64_t so = (uint64_t)((stage * STAGE2_BYTES) >> 4);
#pragma unroll
            for (int c = 0; c < KCH; ++c) {
              if (c < nch) {
#pragma unroll
                for (int kk = 0; kk < BK / 32; ++kk) {
                  const uint64_t o = so + (uint64_t)((c * HALF_TILE + kk * 32) >> 4);
                  mma_f8_pair(d_tmem, dA0 + o, dB0 + o, idesc, ((kb + c) | kk) != 0 ? 1u : 0u);
                }
              }
            }
            mma_commit_pair_mask(smem_u32(&empty[stage]), (uint16_t)3);  // both CTAs' stage
            if (++stage == STAGES2) {
              stage = 0;
              phase ^= 1u;
            }
          }
          if (!ok) break;
          const uint32_t fb = smem_u32(&acc_full[acc]);
          mma_commit_pair(mapa_shared(fb, 0));
          mma_commit_pair(mapa_shared(fb, 1));
          acc ^= 1;
          if (acc == 0) acc_phase ^= 1u;
        }
      }
      mma_commit_pair(mapa_shared(smem_u32(drain), 0));
      long long c0 = clock64();
      while (!mbar_try_wait(drain, 0) && clock64() - c0 < WAIT_LIMIT) {
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------ epilogue (both CTAs)
    constexpr int CH = BN / 32 / H;        // 32-column chunks per warp and tile
    const int quarter = warp & 3;          // TMEM lanes this warp may read
    const int half = (warp - 2) >> 2;      // tile chunks [CH half, CH half + CH)
    const int row_in_tile = quarter * 32 + lane;
    float *scratch = scratch_all + (threadIdx.x - 64) * SCRATCH_F;
    const bool f16 = g.score_mode == R2M_SCORE_F16;
    const bool scaled = g.score_mode == R2M_SCORE_SCALED;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    Reservoir<KT> R;
    for (int u = pair; ok && u < num_units; u += npairs) {
      const int mt = u % g.num_m_tiles, sp = u / g.num_m_tiles;
      const int t0 = split_lo(sp, g.n_tiles, g.splits), t1 = split_lo(sp + 1, g.n_tiles, g.splits);
      R.reset();
      for (int t = t0; t < t1; ++t) {
        bool w = mbar_wait_bounded(&acc_full[acc], acc_phase, abort_flag, WAIT_LIMIT);
        if (__any_sync(FULL, !w)) {
          if (lane == 0 && !*abort_flag) atomicExch(g.err, kErrTimeoutAccFull);
          *abort_flag = 1;
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN + half * CH * 32);
        drain_acc<KT, H>(R, taddr, (long long)t * BN + half * CH * 32, g.N, g.scaleB, scaled, f16, scratch);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(mapa_shared(smem_u32(&acc_empty[acc]), 0));
        acc ^= 1;
        if (acc == 0) acc_phase ^= 1u;
      }
      if (!ok) break;
      const int row = mt * 256 + (int)rank * 128 + row_in_tile;
      if (row < g.nb) {
        const size_t list = (size_t)sp * H + half;
        float *pv = g.part_vals + (list * g.mpad + row) * KT;
        int *pc = g.part_cols + (list * g.mpad + row) * KT;
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          pv[j] = R.v[j];
          pc[j] = R.c[j];
        }
      }
    }
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync();  // the leader's MMAs touch the peer's smem and TMEM until here
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, TMEM_COLS);
  }
}

// Merge the per-split sorted lists of every row into its final top-k:
// one warp per row, k rounds of a warp arg-max over the list heads.
__global__ void k_merge_splits(const float *__restrict__ pv, const int *__restrict__ pc, int splits,
                               int mpad, int KT, int nb, int k, int score_mode,
                               const float *__restrict__ scaleA, float *out_v, int *out_l) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= nb) return;
  const unsigned FULL = 0xFFFFFFFFu;
  constexpr int PER = MAX_SPLITS / 32;
  int head[PER];
  float hv[PER];
  int hc[PER];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    int s = lane + 32 * q;
    head[q] = 0;
    if (s < splits) {
      size_t b = ((size_t)s * mpad + row) * KT;
      hv[q] = pv[b];
      hc[q] = pc[b];
    } else {
      hv[q] = -INFINITY;
      hc[q] = INT_MAX;
    }
  }
  const float sa = (score_mode == R2M_SCORE_SCALED) ? scaleA[row] : 1.0f;
  for (int r = 0; r < k; ++r) {
    float bv = hv[0];
    int bc = hc[0], bq = 0;
#pragma unroll
    for (int q = 1; q < PER; ++q) {
      bool better = (hv[q] > bv) || (hv[q] == bv && hc[q] < bc);
      bv = better ? hv[q] : bv;
      bc = better ? hc[q] : bc;
      bq = better ? q : bq;
    }
    float wv = bv;
    int wc = bc, wl = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      float ov = __shfl_xor_sync(FULL, wv, o);
      int oc = __shfl_xor_sync(FULL, wc, o);
      int ol = __shfl_xor_sync(FULL, wl, o);
      bool better = (ov > wv) || (ov == wv && oc < wc) || (ov == wv && oc == wc && ol < wl);
      wv = better ? ov : wv;
      wc = better ? oc : wc;
      wl = better ? ol : wl;
    }
    if (lane == 0) {
      bool empty = (wv == -INFINITY) || wc == INT_MAX;
      out_v[(size_t)row * k + r] = empty ? -INFINITY : wv * sa;
      out_l[(size_t)row * k + r] = empty ? 0 : wc + 1;
    }
    if (lane == wl) {
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        if (q == bq) {
          int s = lane + 32 * q;
          int h = ++head[q];
          if (h < KT) {
            size_t b = ((size_t)s * mpad + row) * KT + h;
            hv[q] = pv[b];
            hc[q] = pc[b];
          } else {
            hv[q] = -INFINITY;
            hc[q] = INT_MAX;
          }
        }
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------ host

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int get_encode_fn(EncodeTiledFn *fn) {
  static std::mutex mu;
  static EncodeTiledFn cached = nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!cached) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
      return fail(R2M_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
    cached = reinterpret_cast<EncodeTiledFn>(p);
  }
  *fn = cached;
  return R2M_OK;
}

// 2-D uint8 tensor of `rows` x `cols` bytes (row stride = cols), box
// `box_rows` x 128 bytes, 128-byte swizzle, zero fill outside.
static int make_map(CUtensorMap *map, const void *base, long long rows, int cols, int box_rows) {
  EncodeTiledFn fn = nullptr;
  int rc = get_encode_fn(&fn);
  if (rc) return rc;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box,
                  estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(R2M_ECUDA, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
  return R2M_OK;
}

static int pick_kt(int k) {
  if (k <= 8) return 8;
  if (k <= 16) return 16;
  if (k <= 20) return 20;
  if (k <= 32) return 32;
  return 64;
}

static size_t gemm_smem_bytes(int H) {
  return 1024 + (size_t)STAGES * (A_STAGE + B_STAGE) + (2 * STAGES + 5) * 8 + 16 +
         (size_t)(epi_threads(H) - 64) * SCRATCH_F * sizeof(float);
}

// Column splits for a given number of read tiles.  The single-CTA kernel,
// or fewer read tiles than half the CTA pairs: enough units to keep every
// CTA busy, chosen to minimise the last-wave imbalance.  The CTA-pair kernel
// with more read tiles runs power-bound, where a wave with a few idle pairs
// loses little (the busy ones clock higher) but every doubling of the splits
// costs about 9% at equal wave use (measured against 3,297,890 columns,
// 16,384-65,536 reads: one split beat the imbalance-minimising choice by 8-18%
// below 65,536 reads); so there the splits maximise
// units / (waves x pairs) x 0.91^log2(splits) over 1..8.
static int choose_splits(int m_tiles, int n_tiles, int ctas, int forced, int max_splits = MAX_SPLITS,
                         bool pair = false) {
  if (forced > 0) {
    int s = forced;
    if (s > n_tiles) s = n_tiles;
    if (s > max_splits) s = max_splits;
    return s < 1 ? 1 : s;
  }
  int cap = n_tiles < max_splits ? n_tiles : max_splits;
  if (cap < 1) cap = 1;
  if (pair && 2 * m_tiles >= ctas) {
    int best = 1;
    double best_score = -1.0;
    for (int s = 1; s <= 8 && s <= cap; ++s) {
      const long long units = (long long)m_tiles * s;
      const long long waves = (units + ctas - 1) / ctas;
      const double score = (double)units / (double)(waves * ctas) * std::pow(0.91, std::log2((double)s));
      if (score > best_score + 1e-9) {
        best_score = score;
        best = s;
      }
    }
    return best;
  }
  int smin = (4 * ctas + m_tiles - 1) / m_tiles;
  if (smin < 1) smin = 1;
  if (smin > cap) smin = cap;
  int best = smin;
  double best_eff = -1.0;
  for (int s = smin; s <= cap && s <= 2 * smin; ++s) {
    long long units = (long long)m_tiles * s;
    long long waves = (units + ctas - 1) / ctas;
    double eff = (double)units / (double)(waves * ctas);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = s;
    }
  }
  return best;
}

template <int KT, int H>
static int launch_gemm(const CUtensorMap &mA, const CUtensorMap &mB, const GemmArgs &g, int ctas,
                       cudaStream_t st) {
  size_t smem = gemm_smem_bytes(H);
  // a function attribute is per device: set it on every launch (cheap)
  R2M_CUDA(cudaFuncSetAttribute(k_gemm_topk<KT, H>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_gemm_topk<KT, H><<<ctas, epi_threads(H), smem, st>>>(mA, mB, g);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}

static size_t gemm2_smem_bytes(int H) {
  return 1024 + (size_t)STAGES2 * 2 * STAGE2_BYTES + (2 * STAGES2 + 5) * 8 + 16 +
         (size_t)(epi_threads(H) - 64) * SCRATCH_F * sizeof(float);
}

// Epilogue halves of a launch of kernel `kind`: the CTA-pair kernel always
// takes 2 when the reservoir allows (k <= 32), the single-CTA kernel for
// short units only.
static int epi_halves_for(int kind, int KT, int n_tiles, int splits) {
  if (KT > 32) return 1;
  if (kind == 2) return 2;
  return (n_tiles + splits - 1) / splits <= SHORT_UNIT_TILES ? 2 : 1;
}

template <int KT, int H>
static int launch_gemm2(const CUtensorMap &mA, const CUtensorMap &mB, const GemmArgs &g, int pairs,
                        cudaStream_t st) {
  size_t smem = gemm2_smem_bytes(H);
  R2M_CUDA(cudaFuncSetAttribute(k_gemm_topk2<KT, H>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * pairs, 1, 1);
  cfg.blockDim = dim3(epi_threads(H), 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  R2M_CUDA(cudaLaunchKernelEx(&cfg, k_gemm_topk2<KT, H>, mA, mB, g));
  return R2M_OK;
}

// Reservoir size of an engine: the smallest of 8/16/20/32/64 that holds k,
// or tuning.reserved[4] when that is one of them and holds k.
static int kt_for(int k, const r2m_tuning *tune) {
  const int r = tune ? tune->reserved[4] : 0;
  if ((r == 8 || r == 16 || r == 20 || r == 32 || r == 64) && r >= k) return r;
  return pick_kt(k);
}

// Load every fused-kernel instance once per device (and set its shared-
// memory limit) so that no kernel is first loaded while a stream is being
// captured into a graph.
static int preload_kernels() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  R2M_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64 || done[dev]) return R2M_OK;
#define R2M_PRELOAD1(KT, H)                                                                    \
  R2M_CUDA(cudaFuncSetAttribute(k_gemm_topk<KT, H>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                (int)gemm_smem_bytes(H)))
#define R2M_PRELOAD2(KT, H)                                                                     \
  R2M_CUDA(cudaFuncSetAttribute(k_gemm_topk2<KT, H>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                (int)gemm2_smem_bytes(H)))
  R2M_PRELOAD1(8, 1); R2M_PRELOAD1(16, 1); R2M_PRELOAD1(20, 1); R2M_PRELOAD1(32, 1); R2M_PRELOAD1(64, 1);
  R2M_PRELOAD1(8, 2); R2M_PRELOAD1(16, 2); R2M_PRELOAD1(20, 2); R2M_PRELOAD1(32, 2);
  R2M_PRELOAD2(8, 1); R2M_PRELOAD2(16, 1); R2M_PRELOAD2(20, 1); R2M_PRELOAD2(32, 1); R2M_PRELOAD2(64, 1);
  R2M_PRELOAD2(8, 2); R2M_PRELOAD2(16, 2); R2M_PRELOAD2(20, 2); R2M_PRELOAD2(32, 2);
#undef R2M_PRELOAD1
#undef R2M_PRELOAD2
  cudaFuncAttributes fa;
  R2M_CUDA(cudaFuncGetAttributes(&fa, k_merge_splits));
  done[dev] = true;
  return R2M_OK;
}

// Which kernel a batch of nb reads runs on: 1 = one CTA per 128-read tile,
// 2 = CTA pairs per 256-read tile.  mode 0 (auto) uses pairs above 128 reads.
static int kernel_kind(int mode, int nb) {
  if (mode == 1) return 1;
  if (mode == 2) return 2;
  return nb > BM ? 2 : 1;
}

// Launch the fused kernel of `kind` (1 single-CTA, 2 CTA pairs) with
// `halves` epilogue halves for the reservoir size KT.
static int dispatch_gemm(int kind, int halves, int KT, const CUtensorMap &mA, const CUtensorMap &mB,
                         const CUtensorMap &mB128, const GemmArgs &g, int ctas, cudaStream_t st) {
  if (kind == 2) {
    if (halves == 2) {
      switch (KT) {
        case 8: return launch_gemm2<8, 2>(mA, mB128, g, ctas, st);
        case 16: return launch_gemm2<16, 2>(mA, mB128, g, ctas, st);
        case 20: return launch_gemm2<20, 2>(mA, mB128, g, ctas, st);
        default: return launch_gemm2<32, 2>(mA, mB128, g, ctas, st);
      }
    }
    switch (KT) {
      case 8: return launch_gemm2<8, 1>(mA, mB128, g, ctas, st);
      case 16: return launch_gemm2<16, 1>(mA, mB128, g, ctas, st);
      case 20: return launch_gemm2<20, 1>(mA, mB128, g, ctas, st);
      case 32: return launch_gemm2<32, 1>(mA, mB128, g, ctas, st);
      default: return launch_gemm2<64, 1>(mA, mB128, g, ctas, st);
    }
  }
  if (halves == 2) {
    switch (KT) {
      case 8: return launch_gemm<8, 2>(mA, mB, g, ctas, st);
      case 16: return launch_gemm<16, 2>(mA, mB, g, ctas, st);
      case 20: return launch_gemm<20, 2>(mA, mB, g, ctas, st);
      default: return launch_gemm<32, 2>(mA, mB, g, ctas, st);
    }
  }
  switch (KT) {
    case 8: return launch_gemm<8, 1>(mA, mB, g, ctas, st);
    case 16: return launch_gemm<16, 1>(mA, mB, g, ctas, st);
    case 20: return launch_gemm<20, 1>(mA, mB, g, ctas, st);
    case 32: return launch_gemm<32, 1>(mA, mB, g, ctas, st);
    default: return launch_gemm<64, 1>(mA, mB, g, ctas, st);
  }
}

// Progress slots for pair pacing (one per CTA pair of a launch).
constexpr int kPaceSlots = 1024;

// Pacing window of the CTA-pair kernel from tuning.reserved[3]: 0 = the
// default, > 0 = that many column tiles, < 0 = no pacing.
static int pace_window_for(const r2m_tuning *tune) {
  const int r = tune ? tune->reserved[3] : 0;
  return r < 0 ? 0 : r == 0 ? PACE_WINDOW : r;
}

// Split lists the workspace must hold for any batch height up to rows_cap.
static size_t lists_needed(int rows_cap, int n_tiles, int ctas, int forced, int mode, int KT) {
  size_t lists = 0;
  for (int nb = BM; nb < rows_cap + BM; nb += BM) {
    int h = nb < rows_cap ? nb : rows_cap;
    int kind = kernel_kind(mode, h);
    int tile = kind == 2 ? 256 : BM;
    int mt = (h + tile - 1) / tile;
    int c = kind == 2 ? (ctas / 2 > 0 ? ctas / 2 : 1) : ctas;
    // either kernel may leave two partial lists per row and split
    (void)kind;
    const int H = KT <= 32 ? 2 : 1;
    size_t l = (size_t)choose_splits(mt, n_tiles, c, forced, MAX_SPLITS / H, kind == 2) * H * mt * tile;
    if (l > lists) lists = l;
  }
  return lists;
}

}  // namespace r2m

using namespace r2m;

struct r2m_engine {
  const uint8_t *B;
  const float *scaleB;
  int rdim;
  long long N;
  long long N_cap;  // columns at creation (the workspace is sized for them)
  int k, KT;
  int rows_cap;
  int score_mode;
  int ctas;
  int forced_splits;
  int n_tiles;
  CUtensorMap mapB;
  CUtensorMap mapB128;  // 128-row box for the CTA-pair kernel
  int mode;             // 0 auto, 1 single-CTA kernel, 2 CTA-pair kernel
  int epi;              // CTA-pair epilogue: 0 auto, 1 four warps, 2 eight warps
  float *part_vals;
  int *part_cols;
  size_t part_lists;  // capacity in lists (rows x splits)
  uint32_t *err;
  long long *pace;    // per-pair progress of the CTA-pair kernel (kPaceSlots)
  int pace_window;    // 0 = no pacing
  bool timing;        // record events around the two kernels of each call
  cudaEvent_t ev[3];
  int last_splits;
};

extern "C" int r2m_engine_create(const uint8_t *d_B, const float *d_scaleB, int rdim, int64_t N, int k,
                                 int rows_cap, int score_mode, const r2m_tuning *tune,
                                 r2m_engine **out) {
  R2M_REQUIRE(out != nullptr, "out is null");
  *out = nullptr;
  R2M_REQUIRE(d_B != nullptr, "B is null");
  R2M_REQUIRE(rdim >= 16 && rdim % 16 == 0, "rdim must be a positive multiple of 16");
  R2M_REQUIRE(N >= 1 && N <= (1LL << 31) - 1 - BN, "N out of range");
  R2M_REQUIRE(k >= 1 && k <= 64 && k <= N, "need 1 <= k <= min(N, 64)");
  R2M_REQUIRE(rows_cap >= 1, "rows_cap must be >= 1");
  R2M_REQUIRE(score_mode >= R2M_SCORE_F16 && score_mode <= R2M_SCORE_SCALED, "bad score_mode");
  R2M_REQUIRE(score_mode != R2M_SCORE_SCALED || d_scaleB, "scaled scores need scaleB");
  R2M_REQUIRE((reinterpret_cast<uintptr_t>(d_B) & 15) == 0, "B must be 16-byte aligned");
  R2M_REQUIRE(score_mode != R2M_SCORE_SCALED || (reinterpret_cast<uintptr_t>(d_scaleB) & 15) == 0,
              "scaleB must be 16-byte aligned");
  int rc = r2m_device_check();
  if (!rc) rc = preload_kernels();
  if (rc) return rc;
  r2m_engine *e = new r2m_engine();
  e->B = d_B;
  e->scaleB = d_scaleB;
  e->rdim = rdim;
  e->N = N;
  e->N_cap = N;
  e->k = k;
  e->KT = kt_for(k, tune);
  e->rows_cap = rows_cap;
  e->score_mode = score_mode;
  e->ctas = (tune && tune->ctas > 0) ? tune->ctas : sm_count();
  e->forced_splits = (tune && tune->splits > 0) ? tune->splits : 0;
  e->timing = tune && tune->reserved[0] != 0;
  e->mode = tune ? tune->reserved[1] : 0;
  if (e->mode < 0 || e->mode > 2) e->mode = 0;
  e->epi = tune ? tune->reserved[2] : 0;
  if (e->epi < 0 || e->epi > 2) e->epi = 0;
  e->pace_window = pace_window_for(tune);
  e->last_splits = 0;
  if (e->timing) {
    for (int i = 0; i < 3; ++i) {
      cudaError_t ce = cudaEventCreate(&e->ev[i]);
      if (ce != cudaSuccess) {
        delete e;
        return cuda_fail(ce, "cudaEventCreate");
      }
    }
  }
  e->n_tiles = (int)((N + BN - 1) / BN);
  rc = make_map(&e->mapB, d_B, N, rdim, BN);
  if (!rc) rc = make_map(&e->mapB128, d_B, N, rdim, 128);
  if (rc) {
    delete e;
    return rc;
  }
  // workspace: the largest (read tiles x splits) any batch height can ask for
  size_t lists = lists_needed(rows_cap, e->n_tiles, e->ctas, e->forced_splits, e->mode, e->KT);
  e->part_lists = lists;
  cudaError_t ce = cudaMalloc(&e->part_vals, lists * e->KT * sizeof(float));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->part_cols, lists * e->KT * sizeof(int));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->pace, kPaceSlots * sizeof(long long));
  if (ce != cudaSuccess) {
    cudaFree(e->part_vals);
    cudaFree(e->part_cols);
    delete e;
    return fail(R2M_ENOMEM, "engine workspace allocation failed");
  }
  rc = device_error_word(&e->err);
  if (rc) {
    cudaFree(e->part_vals);
    cudaFree(e->part_cols);
    cudaFree(e->pace);
    delete e;
    return rc;
  }
  *out = e;
  return R2M_OK;
}

extern "C" int r2m_engine_destroy(r2m_engine *eng) {
  if (!eng) return R2M_OK;
  cudaFree(eng->part_vals);
  cudaFree(eng->part_cols);
  cudaFree(eng->pace);
  if (eng->timing)
    for (int i = 0; i < 3; ++i) cudaEventDestroy(eng->ev[i]);
  delete eng;
  return R2M_OK;
}

extern "C" int r2m_engine_set_tuning(r2m_engine *eng, const r2m_tuning *tune) {
  R2M_REQUIRE(eng != nullptr && tune != nullptr, "null pointer");
  const int ctas = tune->ctas > 0 ? tune->ctas : sm_count();
  const int forced = tune->splits > 0 ? tune->splits : 0;
  const int mode = (tune->reserved[1] >= 0 && tune->reserved[1] <= 2) ? tune->reserved[1] : 0;
  const int KT = kt_for(eng->k, tune);
  size_t lists = lists_needed(eng->rows_cap, eng->n_tiles, ctas, forced, mode, KT);
  if (lists * KT > eng->part_lists * eng->KT) {  // grow the split workspace
    float *pv = nullptr;
    int *pc = nullptr;
    cudaError_t ce = cudaMalloc(&pv, lists * KT * sizeof(float));
    if (ce == cudaSuccess) ce = cudaMalloc(&pc, lists * KT * sizeof(int));
    if (ce != cudaSuccess) {
      cudaFree(pv);
      return fail(R2M_ENOMEM, "engine workspace allocation failed");
    }
    R2M_CUDA(cudaDeviceSynchronize());
    cudaFree(eng->part_vals);
    cudaFree(eng->part_cols);
    eng->part_vals = pv;
    eng->part_cols = pc;
    eng->part_lists = lists;
  } else {
    eng->part_lists = eng->part_lists * eng->KT / KT;  // the same bytes hold more, shorter lists
  }
  eng->KT = KT;
  eng->ctas = ctas;
  eng->forced_splits = forced;
  eng->mode = mode;
  eng->epi = (tune->reserved[2] >= 0 && tune->reserved[2] <= 2) ? tune->reserved[2] : 0;
  eng->pace_window = pace_window_for(tune);
  return R2M_OK;
}

namespace r2m {
// Point the engine at another B (and scaleB) of at most the columns it was
// created for: the split workspace stays valid, the tensor maps are encoded
// again on the host.  The maps reach the kernels as launch parameters, so
// launches already queued keep the previous B.
int engine_rebind(r2m_engine *eng, const uint8_t *d_B, const float *d_scaleB, int64_t N) {
  R2M_REQUIRE(eng != nullptr && d_B != nullptr, "null pointer");
  R2M_REQUIRE(N >= eng->k && N <= eng->N_cap, "rebind: N must be in k..N at creation");
  R2M_REQUIRE((reinterpret_cast<uintptr_t>(d_B) & 15) == 0, "B must be 16-byte aligned");
  R2M_REQUIRE(eng->score_mode != R2M_SCORE_SCALED || (d_scaleB && (reinterpret_cast<uintptr_t>(d_scaleB) & 15) == 0),
              "scaled scores need a 16-byte aligned scaleB");
  CUtensorMap m, m128;
  int rc = make_map(&m, d_B, N, eng->rdim, BN);
  if (!rc) rc = make_map(&m128, d_B, N, eng->rdim, 128);
  if (rc) return rc;
  eng->B = d_B;
  eng->scaleB = d_scaleB;
  eng->N = N;
  eng->n_tiles = (int)((N + BN - 1) / BN);
  eng->mapB = m;
  eng->mapB128 = m128;
  return R2M_OK;
}
}  // namespace r2m

extern "C" int r2m_engine_info(const r2m_engine *eng, int *k, int *rdim, int *score_mode, int *rows_cap,
                               int64_t *N) {
  R2M_REQUIRE(eng != nullptr, "engine is null");
  if (k) *k = eng->k;
  if (rdim) *rdim = eng->rdim;
  if (score_mode) *score_mode = eng->score_mode;
  if (rows_cap) *rows_cap = eng->rows_cap;
  if (N) *N = eng->N;
  return R2M_OK;
}

extern "C" int64_t r2m_engine_workspace_bytes(const r2m_engine *eng) {
  if (!eng) return 0;
  return (int64_t)(eng->part_lists * eng->KT * (sizeof(float) + sizeof(int)));
}

extern "C" int r2m_batch_gemm_topk(r2m_engine *eng, const uint8_t *d_A, const float *d_scaleA, int nb,
                                   float *d_vals, int32_t *d_locs, r2m_stream_t stream) {
  R2M_REQUIRE(eng != nullptr, "engine is null");
  R2M_REQUIRE(nb >= 0 && nb <= eng->rows_cap, "nb must be in 0..rows_cap");
  if (nb == 0) return R2M_OK;
  R2M_REQUIRE(d_A && d_vals && d_locs, "null pointer");
  R2M_REQUIRE((reinterpret_cast<uintptr_t>(d_A) & 15) == 0, "A must be 16-byte aligned");
  R2M_REQUIRE(eng->score_mode != R2M_SCORE_SCALED || d_scaleA, "scaled scores need scaleA");
  cudaStream_t st = as_stream(stream);
  CUtensorMap mapA;
  int rc = make_map(&mapA, d_A, nb, eng->rdim, BM);
  if (rc) return rc;
  const int kind = kernel_kind(eng->mode, nb);
  const int tile = kind == 2 ? 256 : BM;
  const int ctas_eff = kind == 2 ? (eng->ctas / 2 > 0 ? eng->ctas / 2 : 1) : eng->ctas;
  GemmArgs g;
  g.nb = nb;
  g.num_m_tiles = (nb + tile - 1) / tile;
  g.N = eng->N;
  g.n_tiles = eng->n_tiles;
  const int hmax = eng->KT <= 32 ? 2 : 1;
  g.splits = choose_splits(g.num_m_tiles, eng->n_tiles, ctas_eff, eng->forced_splits, MAX_SPLITS / hmax, kind == 2);
  const int halves =
      eng->epi == 1 ? 1 : eng->epi == 2 ? hmax : epi_halves_for(kind, eng->KT, eng->n_tiles, g.splits);
  const int lists_per_row = halves * g.splits;  // partial lists each row leaves
  g.num_kb = (eng->rdim + BK - 1) / BK;
  g.score_mode = eng->score_mode;
  g.mpad = g.num_m_tiles * tile;
  g.scaleB = eng->scaleB;
  g.part_vals = eng->part_vals;
  g.part_cols = eng->part_cols;
  g.err = eng->err;
  if ((size_t)lists_per_row * g.mpad > eng->part_lists) return fail(R2M_ESTATE, "engine workspace too small");
  long long units = (long long)g.num_m_tiles * g.splits;
  int ctas = (int)(units < ctas_eff ? units : ctas_eff);
  eng->last_splits = g.splits;
  g.pace = nullptr;
  g.pace_window = 0;
  if (kind == 2 && eng->pace_window > 0 && ctas > 1 && ctas <= kPaceSlots) {
    // every pair starts as "not started" (-1)
    R2M_CUDA(cudaMemsetAsync(eng->pace, 0xFF, (size_t)ctas * sizeof(long long), st));
    g.pace = eng->pace;
    g.pace_window = eng->pace_window;
  }
  if (eng->timing) R2M_CUDA(cudaEventRecord(eng->ev[0], st));
  rc = dispatch_gemm(kind, halves, eng->KT, mapA, eng->mapB, eng->mapB128, g, ctas, st);
  if (rc) return rc;
  if (eng->timing) R2M_CUDA(cudaEventRecord(eng->ev[1], st));
  const int warps = 8;
  k_merge_splits<<<(nb + warps - 1) / warps, 32 * warps, 0, st>>>(
      eng->part_vals, eng->part_cols, lists_per_row, g.mpad, eng->KT, nb, eng->k, eng->score_mode, d_scaleA,
      d_vals, d_locs);
  R2M_CUDA(cudaGetLastError());
  if (eng->timing) R2M_CUDA(cudaEventRecord(eng->ev[2], st));
  return R2M_OK;
}

extern "C" int r2m_engine_kernel_ms(r2m_engine *eng, float *gemm_ms, float *merge_ms, int *splits) {
  R2M_REQUIRE(eng != nullptr, "engine is null");
  R2M_REQUIRE(eng->timing, "engine was created without kernel timing (tuning.reserved[0] = 1)");
  R2M_CUDA(cudaEventSynchronize(eng->ev[2]));
  float a = 0.f, b = 0.f;
  R2M_CUDA(cudaEventElapsedTime(&a, eng->ev[0], eng->ev[1]));
  R2M_CUDA(cudaEventElapsedTime(&b, eng->ev[1], eng->ev[2]));
  if (gemm_ms) *gemm_ms = a;
  if (merge_ms) *merge_ms = b;
  if (splits) *splits = eng->last_splits;
  return R2M_OK;
}

// ------------------------------------------------------------------
// Allocation-free search.
//
// Some callers cannot allocate device memory at the point where they map a
// batch: a serving loop where a cudaMalloc would synchronize the device and
// stall other streams, or a host whose memory pool (CUDA.jl's, PyTorch's
// caching allocator) already owns the free device memory, so a side
// allocation can fail.  This entry point needs no engine: the pacing slots
// and the per-split partial top-k lists live in the file-scope array below,
// whose device address is looked up with cudaGetSymbolAddress by the first
// call on each device (so that first call should come before any stream
// capture) and again whenever the device's current context is a different
// one (after a cudaDeviceReset the module, and with it the array, is loaded
// anew).  Every GPU that loads this library holds the array
// (kNoAllocScratchBytes) until the process exits; all calls share it, so
// calls that overlap on the GPU race.  The schedule is the engine's
// automatic one (the CTA-pair kernel above 128 reads, paced; the epilogue
// form and the column splits the engine would pick), with the splits cut to
// what the array holds.
namespace r2m {

constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 32 MiB
constexpr size_t kNoAllocPaceBytes = kPaceSlots * sizeof(long long);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ __align__(256) uint32_t g_noalloc_err;

static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[64];
static uint32_t *g_noalloc_err_ptr[64];
static unsigned long long g_noalloc_ctx[64];  // id of the context the addresses belong to

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Process-unique id of the current context (0 when the driver cannot tell).
static unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
  }
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device addresses of the scratch array and error word on the current device
// (looked up on the first call per device and per context).
static int noalloc_setup(unsigned char **scratch, uint32_t **err) {
  int dev = 0;
  R2M_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(R2M_ESTATE, "device ordinal out of range");
  const unsigned long long ctx = current_ctx_id();
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (g_noalloc_ptr[dev] == nullptr || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
    void *p = nullptr, *q = nullptr;
    R2M_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    R2M_CUDA(cudaGetSymbolAddress(&q, g_noalloc_err));
    g_noalloc_ptr[dev] = static_cast<unsigned char *>(p);
    g_noalloc_err_ptr[dev] = static_cast<uint32_t *>(q);
    g_noalloc_ctx[dev] = current_ctx_id();  // the lookup made the device's context current
  }
  *scratch = g_noalloc_ptr[dev];
  *err = g_noalloc_err_ptr[dev];
  return R2M_OK;
}

// A bounded wait that gave up leaves partial lists unwritten: mark every
// output row invalid (NaN values, location -1) so the caller sees it.
__global__ void k_noalloc_poison(const uint32_t *err, float *vals, int *locs, long long count) {
  if (*err == 0) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    vals[i] = __int_as_float(0x7fc00000);
    locs[i] = -1;
  }
}

}  // namespace r2m

extern "C" int r2m_batch_gemm_topk_noalloc(const uint8_t *d_B, const float *d_scaleB, int rdim, int64_t N,
                                           const uint8_t *d_A, const float *d_scaleA, int nb, int k,
                                           int score_mode, float *d_vals, int32_t *d_locs,
                                           r2m_stream_t stream) {
  R2M_REQUIRE(d_B != nullptr, "B is null");
  R2M_REQUIRE(rdim >= 16 && rdim % 16 == 0, "rdim must be a positive multiple of 16");
  R2M_REQUIRE(N >= 1 && N <= (1LL << 31) - 1 - BN, "N out of range");
  R2M_REQUIRE(k >= 1 && k <= 64 && k <= N, "need 1 <= k <= min(N, 64)");
  R2M_REQUIRE(nb >= 0, "nb must be >= 0");
  R2M_REQUIRE(score_mode >= R2M_SCORE_F16 && score_mode <= R2M_SCORE_SCALED, "bad score_mode");
  if (nb == 0) return R2M_OK;
  R2M_REQUIRE(d_A && d_vals && d_locs, "null pointer");
  R2M_REQUIRE(score_mode != R2M_SCORE_SCALED || (d_scaleA && d_scaleB), "scaled scores need scaleA and scaleB");
  R2M_REQUIRE((reinterpret_cast<uintptr_t>(d_B) & 15) == 0 && (reinterpret_cast<uintptr_t>(d_A) & 15) == 0,
              "A and B must be 16-byte aligned");
  R2M_REQUIRE(score_mode != R2M_SCORE_SCALED || (reinterpret_cast<uintptr_t>(d_scaleB) & 15) == 0,
              "scaleB must be 16-byte aligned");
  const int KT = pick_kt(k);
  const int kind = kernel_kind(0, nb);
  const int tile = kind == 2 ? 256 : BM;
  const int m_tiles = (nb + tile - 1) / tile;
  const size_t list_bytes = (size_t)KT * (sizeof(float) + sizeof(int));
  const size_t max_lists = (kNoAllocScratchBytes - kNoAllocPaceBytes) / list_bytes;
  const size_t mpad = (size_t)m_tiles * tile;
  if (mpad > max_lists)
    return fail(R2M_EINVAL, "nb = " + std::to_string(nb) + " exceeds the allocation-free scratch (" +
                                std::to_string(kNoAllocScratchBytes >> 20) + " MiB holds at most " +
                                std::to_string(max_lists / 256 * 256) + " rows at k = " + std::to_string(k) +
                                "); split the batch or use r2m_batch_gemm_topk");
  unsigned char *scratch = nullptr;
  uint32_t *err = nullptr;
  int rc = noalloc_setup(&scratch, &err);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  CUtensorMap mapA, mapB, mapB128;
  if ((rc = make_map(&mapB, d_B, N, rdim, BN))) return rc;
  if ((rc = make_map(&mapB128, d_B, N, rdim, 128))) return rc;
  if ((rc = make_map(&mapA, d_A, nb, rdim, BM))) return rc;
  const int n_tiles = (int)((N + BN - 1) / BN);
  const int sms = sm_count();
  const int ctas_eff = kind == 2 ? (sms / 2 > 0 ? sms / 2 : 1) : sms;
  const int hmax = KT <= 32 ? 2 : 1;
  // the engine's automatic schedule, with the splits cut to the scratch
  int splits = choose_splits(m_tiles, n_tiles, ctas_eff, 0, MAX_SPLITS / hmax, kind == 2);
  int halves = epi_halves_for(kind, KT, n_tiles, splits);
  while (splits > 1 && (size_t)halves * splits * mpad > max_lists) {
    --splits;
    halves = epi_halves_for(kind, KT, n_tiles, splits);
  }
  if ((size_t)halves * splits * mpad > max_lists) halves = 1;
  GemmArgs g;
  g.nb = nb;
  g.num_m_tiles = m_tiles;
  g.N = N;
  g.n_tiles = n_tiles;
  g.splits = splits;
  g.num_kb = (rdim + BK - 1) / BK;
  g.score_mode = score_mode;
  g.mpad = (int)mpad;
  g.scaleB = d_scaleB;
  long long *pace = reinterpret_cast<long long *>(scratch);
  unsigned char *lists = scratch + kNoAllocPaceBytes;
  const size_t nlists = (size_t)halves * splits * mpad;
  g.part_vals = reinterpret_cast<float *>(lists);
  g.part_cols = reinterpret_cast<int *>(lists + nlists * KT * sizeof(float));
  g.err = err;
  const long long units = (long long)m_tiles * splits;
  const int ctas = (int)(units < ctas_eff ? units : ctas_eff);
  g.pace = nullptr;
  g.pace_window = 0;
  // the error word must start at zero; the partial lists are fully
  // rewritten by the kernel before the merge reads them
  R2M_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
  if (kind == 2 && ctas > 1 && ctas <= kPaceSlots) {
    R2M_CUDA(cudaMemsetAsync(pace, 0xFF, (size_t)ctas * sizeof(long long), st));  // "not started"
    g.pace = pace;
    g.pace_window = PACE_WINDOW;
  }
  rc = dispatch_gemm(kind, halves, KT, mapA, mapB, mapB128, g, ctas, st);
  if (rc) return rc;
  const int warps = 8;
  k_merge_splits<<<(nb + warps - 1) / warps, 32 * warps, 0, st>>>(g.part_vals, g.part_cols, halves * splits,
                                                                   g.mpad, KT, nb, k, score_mode, d_scaleA,
                                                                   d_vals, d_locs);
  R2M_CUDA(cudaGetLastError());
  k_noalloc_poison<<<64, 256, 0, st>>>(err, d_vals, d_locs, (long long)nb * k);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}

// The give-up path of the allocation-free search, driven without a fault:
// the kernels' bounded wait, with a short limit, on an mbarrier nothing
// arrives on, records its code in this path's error word; the poison pass
// then marks the caller's rows as the search would.
extern "C" int r2m_selftest_noalloc_timeout(int64_t limit_cycles, int nb, int k, float *d_vals,
                                            int32_t *d_locs, r2m_stream_t stream) {
  R2M_REQUIRE(limit_cycles >= 0 && limit_cycles <= (int64_t)4000000000LL, "limit_cycles must be in 0..4e9");
  R2M_REQUIRE(nb >= 0 && k >= 1, "need nb >= 0 and k >= 1");
  if (nb == 0) return R2M_OK;
  R2M_REQUIRE(d_vals && d_locs, "null pointer");
  unsigned char *scratch = nullptr;
  uint32_t *err = nullptr;
  int rc = noalloc_setup(&scratch, &err);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  R2M_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
  rc = launch_selftest_wait((long long)limit_cycles, 0, err, st);
  if (rc) return rc;
  k_noalloc_poison<<<64, 256, 0, st>>>(err, d_vals, d_locs, (long long)nb * k);
  R2M_CUDA(cudaGetLastError());
  return R2M_OK;
}
