// FP64 SYRK emulated on the INT8 tensor cores (Ozaki scheme), the B200 form
// of the reference's tc_ozimmu_syrk (BLAS/tc_ozimmu_syrk.cu:3-143), whose
// name implies ozIMMU, the Ozaki-scheme INT8 DGEMM of Ootomo, Ozaki & Yokota
// ("DGEMM on integer matrix multiplication unit", IJHPCA 2024; Ozaki et al.,
// "Error-free transformations of matrix multiplication by using fast routines
// of matrix multiplication", Numer. Algorithms 2012).
//
// Slicing (exact, deterministic): for row i, e_i = max_p exponent(a_ip) with
// |a_ip| < 2^e_i; x = a_ip * 2^-e_i; for s = 1..S: y = 128 x, q_s = trunc(y)
// (|q_s| <= 127), x = y - q_s. Then a_ip = 2^e_i (sum_s q_s 2^-7s + r),
// |r| < 2^-7S, every step exact in FP64.
//
// Product: C_ij = 2^(e_i+e_j) sum_L 2^-7L P_L(i,j), P_L = sum_{s+t=L} Q_s Q_t^T,
// keeping levels L = 2..S+1. Each P_L is computed EXACTLY on tcgen05.mma
// kind::i8 with INT32 accumulation in TMEM (|P_L| <= (L-1) * k * 127^2 <
// 2^31 for k <= 8192 and S <= 14 — checked on the host), then folded into
// FP64 C: C += alpha 2^(e_i+e_j-7L) P_L (one FP64 rounding per level), by a
// kernel of its own after the GEMM (which stores the level sums) or, when
// their workspace does not fit, by the GEMM's epilogue. Slices are stored
// K-major, one int8 plane per slice, so a single 3-D tensor map (k, row,
// slice) feeds every pair.
#include <algorithm>
#include <climits>
#include <cmath>
#include <mutex>
#include <cstring>
#include <cstdio>
#include <vector>

#include "tb_internal.h"
#include "tb_ptx.cuh"

namespace tb {
namespace {

constexpr int kOzBM = 128, kOzBN = 256, kOzBK = 128;  // BK in int8 elements (128 B rows)
constexpr int kOzStages = 4;
constexpr int kOzABytes = kOzBM * kOzBK, kOzBBytes = kOzBN * kOzBK;
constexpr int kOzStageBytes = kOzABytes + kOzBBytes;
constexpr int kOzSmem = kOzStages * kOzStageBytes + 1024 + 256;
constexpr int kOzMaxSlices = 14;
constexpr int kOzLeaf = 512;  // largest TRSM diagonal block inverted explicitly

// kind::i8 instruction descriptor: c_format S32 (2), a/b_format signed int8 (1),
// both K-major, N >> 3 at [17,23), M >> 4 at [24,29).
constexpr uint32_t kOzIdesc =
    (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kOzBN >> 3) << 17) | ((uint32_t)(kOzBM >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                            int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void tmem_ld32_s32(uint32_t taddr, int* v) {
  float f[32];
  tmem_ld32(taddr, f);
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __float_as_int(f[i]);
}

// ---------------------------------------------------------------- slicing
// An operand is a rows x k matrix whose row i is one K-vector:
//   by rows (cols == 0): element (i, p) = X[i + p * ldx] (rows of a column-major matrix)
//   by cols (cols == 1): element (i, p) = X[p + i * ldx] (columns of a column-major matrix)
// mask 1 keeps only p + koff <= i, mask 2 only p + koff >= i (a triangular
// operand whose K range starts at koff); masked elements read as zero.
__device__ __forceinline__ bool oz_keep(int mask, long long i, long long p, long long koff) {
  return mask == 0 || (mask == 1 ? p + koff <= i : p + koff >= i);
}

__device__ __forceinline__ int oz_frexp_max(int m, double v) {
  if (v != 0.0) {
    int ex;
    frexp(v, &ex);
    m = ex > m ? ex : m;
  }
  return m;
}

// e[i] = max(e[i], max_p exponent(x_ip)) with |x_ip| < 2^e; e[] pre-set very
// negative (all-zero rows keep it and are sliced with exponent 0).
__global__ void __launch_bounds__(256) oz_exp_rows_kernel(long long rows, long long k, const double* __restrict__ X,
                                                          long long ldx, int mask, long long koff,
                                                          int* __restrict__ e) {
  const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
  if (i >= rows) return;
  int m = INT_MIN / 2;
  for (long long p = blockIdx.y; p < k; p += gridDim.y)
    if (oz_keep(mask, i, p, koff)) m = oz_frexp_max(m, X[i + p * ldx]);
  atomicMax(&e[i], m);
}

// One warp per operand row (a column of X, contiguous in memory).
__global__ void __launch_bounds__(256) oz_exp_cols_kernel(long long rows, long long k, const double* __restrict__ X,
                                                          long long ldx, int mask, long long koff,
                                                          int* __restrict__ e) {
  const long long i = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= rows) return;
  int m = INT_MIN / 2;
  for (long long p = lane; p < k; p += 32)
    if (oz_keep(mask, i, p, koff)) m = oz_frexp_max(m, X[p + i * ldx]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int t = __shfl_xor_sync(0xffffffffu, m, o);
    m = t > m ? t : m;
  }
  if (lane == 0) atomicMax(&e[i], m);
}

// Dynamic range of the operand rows, for the automatic slice count: per row
// i, with e_i its largest exponent (|x| < 2^e_i) and r_i its root mean
// square, d_i = e_i - log2(r_i) is how many bits the row's largest entries
// sit above its typical one. The largest d_i over the rows is written (in
// 1/256 bit units) to *out with atomicMax. The sum of squares is kept scaled
// by 2^-2m for the running maximum exponent m, so no value overflows.
__device__ __forceinline__ void oz_stat_add(int& m, double& ssq, double v) {
  if (v == 0.0) return;
  int ex;
  frexp(v, &ex);
  if (ex > m) {
    ssq = ldexp(ssq, 2 * (m - ex));
    m = ex;
  }
  const double y = ldexp(v, -m);
  ssq = fma(y, y, ssq);
}
__device__ __forceinline__ void oz_stat_merge(int& m, double& ssq, int m2, double s2) {
  if (s2 == 0.0) return;
  if (ssq == 0.0) {
    m = m2;
    ssq = s2;
    return;
  }
  if (m2 > m) {
    ssq = ldexp(ssq, 2 * (m - m2)) + s2;
    m = m2;
  } else {
    ssq += ldexp(s2, 2 * (m2 - m));
  }
}
__device__ __forceinline__ void oz_stat_publish(double ssq, long long cnt, int* out) {
  if (ssq <= 0.0 || cnt <= 0) return;
  const double d = -0.5 * log2(ssq / (double)cnt);  // e_i - log2(rms_i) >= 0
  atomicMax(out, (int)ceil(d * 256.0));
}
// 16 rows per block (rows of a column-major matrix): half-warp h of warp w
// reads the 16 rows at column phase c = 2w + h, columns p = c, c + 16, ...
// (each half-warp load is 128 contiguous bytes), eight loads in flight per
// thread; the 16 phases' partial (m, ssq, count) of a row are merged in
// phase order, so the result is deterministic.
__global__ void __launch_bounds__(256) oz_spread_rows_kernel(long long rows, long long k, const double* __restrict__ X,
                                                             long long ldx, int mask, long long koff, int* out) {
  __shared__ int sm[16][16];
  __shared__ double ss[16][16];
  __shared__ long long sc[16][16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = lane & 15, c = 2 * warp + (lane >> 4);
  const long long i = (long long)blockIdx.x * 16 + r;
  int m = INT_MIN / 4;
  double ssq = 0.0;
  long long cnt = 0;
  if (i < rows) {
    long long p = c;
    for (; p + 7 * 16 < k; p += 8 * 16) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = __ldcs(X + i + (p + 16 * u) * ldx);
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (oz_keep(mask, i, p + 16 * u, koff)) {
          oz_stat_add(m, ssq, v[u]);
          ++cnt;
        }
    }
    for (; p < k; p += 16)
      if (oz_keep(mask, i, p, koff)) {
        oz_stat_add(m, ssq, X[i + p * ldx]);
        ++cnt;
      }
  }
  sm[c][r] = m;
  ss[c][r] = ssq;
  sc[c][r] = cnt;
  __syncthreads();
  if (threadIdx.x < 16 && i < rows) {
    m = sm[0][r];
    ssq = ss[0][r];
    cnt = sc[0][r];
    for (int q = 1; q < 16; ++q) {
      oz_stat_merge(m, ssq, sm[q][r], ss[q][r]);
      cnt += sc[q][r];
    }
    oz_stat_publish(ssq, cnt, out);
  }
}
// One warp per row (a column of X, contiguous in memory).
__global__ void __launch_bounds__(256) oz_spread_cols_kernel(long long rows, long long k, const double* __restrict__ X,
                                                             long long ldx, int mask, long long koff, int* out) {
  const long long i = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= rows) return;
  int m = INT_MIN / 4;
  double ssq = 0.0;
  long long cnt = 0;
  long long p = lane;
  for (; p + 3 * 32 < k; p += 4 * 32) {
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = __ldcs(X + p + 32 * u + i * ldx);
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (oz_keep(mask, i, p + 32 * u, koff)) {
        oz_stat_add(m, ssq, v[u]);
        ++cnt;
      }
  }
  for (; p < k; p += 32)
    if (oz_keep(mask, i, p, koff)) {
      oz_stat_add(m, ssq, X[p + i * ldx]);
      ++cnt;
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int m2 = __shfl_xor_sync(0xffffffffu, m, o);
    const double s2 = __shfl_xor_sync(0xffffffffu, ssq, o);
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    oz_stat_merge(m, ssq, m2, s2);
  }
  if (lane == 0) oz_stat_publish(ssq, cnt, out);
}

// Slices 16 consecutive K values of one row (already scaled by 2^-e) into S
// int8 planes: one 16-byte vector per slice at Q[s * plane + i * ldq + col].
__device__ __forceinline__ void oz_emit16(double* x, int S, int8_t* __restrict__ Q, long long plane, long long off) {
  for (int s = 0; s < S; ++s) {
    uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const double y = x[j] * 128.0;
      const double q = trunc(y);
      x[j] = y - q;
      w[j >> 2] |= ((uint32_t)(uint8_t)(int8_t)(int)q) << (8 * (j & 3));
    }
    *reinterpret_cast<uint4*>(Q + s * plane + off) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// By-rows operand: 32 rows x 128 K values per block, transposed through
// shared memory so global reads are coalesced along the rows. Columns
// [k, kw) of the planes are written as zeros (kw a multiple of 16).
__global__ void __launch_bounds__(256) oz_slice_rows_kernel(long long rows, long long k, const double* __restrict__ X,
                                                            long long ldx, int mask, long long koff,
                                                            const int* __restrict__ e, int S, int8_t* __restrict__ Q,
                                                            long long ldq, long long plane, long long qoff,
                                                            long long kw) {
  __shared__ double tile[128][33];
  const long long r0 = (long long)blockIdx.x * 32, p0 = (long long)blockIdx.y * 128;
  const int t = threadIdx.x;
  for (int idx = t; idx < 32 * 128; idx += 256) {
    const int r = idx & 31, c = idx >> 5;
    const long long gi = r0 + r, gp = p0 + c;
    tile[c][r] = (gi < rows && gp < k && oz_keep(mask, gi, gp, koff)) ? X[gi + gp * ldx] : 0.0;
  }
  __syncthreads();
  const int r = t >> 3, c0 = (t & 7) * 16;
  const long long gi = r0 + r, gp = p0 + c0;
  if (gi >= rows || gp >= kw) return;
  const int ex = e[gi] < -1000 ? 0 : e[gi];
  double x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = ldexp(tile[c0 + j][r], -ex);
  oz_emit16(x, S, Q, plane, gi * ldq + qoff + gp);
}

// By-cols operand: each thread reads 16 consecutive K values of one row.
__global__ void __launch_bounds__(256) oz_slice_cols_kernel(long long rows, long long k, const double* __restrict__ X,
                                                            long long ldx, int mask, long long koff,
                                                            const int* __restrict__ e, int S, int8_t* __restrict__ Q,
                                                            long long ldq, long long plane, long long qoff,
                                                            long long kw) {
  const int t = threadIdx.x;
  const long long gi = (long long)blockIdx.x * 32 + (t >> 3), gp = (long long)blockIdx.y * 128 + (t & 7) * 16;
  if (gi >= rows || gp >= kw) return;
  const int ex = e[gi] < -1000 ? 0 : e[gi];
  double x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const long long p = gp + j;
    x[j] = (p < k && oz_keep(mask, gi, p, koff)) ? ldexp(X[p + gi * ldx], -ex) : 0.0;
  }
  oz_emit16(x, S, Q, plane, gi * ldq + qoff + gp);
}

// ---------------------------------------------------------------- products
// C (M x N, column-major FP64) = alpha * sum_L 2^(eA_i + eB_j - 7L) P_L + beta * C
// with P_L = sum_{s+t=L} QA_s QB_t^T over the tile's K-blocks [kb0, kb1).
// tile = {m0, n0, kb0 | kOzAccumulate?, kb1}; kOzAccumulate: beta is taken
// as 1 for this tile (a later K chunk of a product whose first chunk
// already applied beta).
constexpr int kOzAccumulate = 1 << 30;
constexpr int kOzRawAll = 1;

struct OzArgs {
  CUtensorMap mapA;  // QA planes, box {128, 128, 1}
  CUtensorMap mapB;  // QB planes, box {128, 256, 1}
  const int4* tiles;
  int num_tiles;
  int S;
  int kb_shift, kb_mod;  // B's K-block = kb + kb_shift (mod kb_mod when kb_mod > 0)
  int M, N;
  int tri;  // 1: only C(i, j) with j <= i is written; 2: only j >= i
  double* C;
  long long ldc;
  double alpha, beta;
  const int* eA;
  const int* eB;
  // 0: fold every level into C; kOzRawAll: write every level's INT32 sums to
  // raw_out + (L - 2) raw_plane (oz_fold_kernel folds them afterwards); >= 2:
  // write only P_raw_level to raw_out (a checking aid)
  int raw_level;
  int* raw_out;
  long long ld_raw, raw_plane;
  int* err;
};

__device__ __forceinline__ int level_pairs_begin(int L, int S) { return L - S > 1 ? L - S : 1; }
__device__ __forceinline__ int level_pairs_end(int L, int S) { return L - 1 < S ? L - 1 : S; }

// 2^e for an integer e: built from the IEEE-754 exponent field when 2^e is a
// normal double (the fold's scales always are in practice), else ldexp.
__device__ __forceinline__ double pow2i(int e) {
  if (e >= -1022 && e <= 1023) return __longlong_as_double((long long)(e + 1023) << 52);
  return ldexp(1.0, e);
}

// The fold epilogue's scalars, copied into registers: the stores go through
// generic pointers the compiler cannot tell apart from the parameter memory,
// so fields read in the store loops would be re-read from it after every
// store.
struct OzEpi {
  double* C;
  int* raw_out;
  long long ldc, ld_raw, raw_plane;
  const int* eA;
  const int* eB;
  double alpha;
  int N, M, tri, raw_level;
};

__device__ __forceinline__ OzEpi oz_epi(const OzArgs& a) {
  return OzEpi{a.C, a.raw_out, a.ldc, a.ld_raw, a.raw_plane, a.eA, a.eB, a.alpha, a.N, a.M, a.tri, a.raw_level};
}

// A row's slicing exponent (all-zero rows keep a very negative one and were
// sliced with exponent 0).
__device__ __forceinline__ int oz_row_exp(const int* e, long long i) { return e[i] < -1000 ? 0 : e[i]; }

// Empty product (K range outside the operands' support): C(gi, n0 + j) =
// beta C(gi, n0 + j) for the tile's written columns (oz_fold_kernel does it
// when the levels are folded there).
__device__ __forceinline__ void oz_scale_row(const OzEpi& ep, long long gi, long long n0, double beta) {
  if (beta == 1.0 || ep.raw_level != 0) return;
  for (int j = 0; j < kOzBN; ++j) {
    const long long gj = n0 + j;
    if (gj < ep.N && (ep.tri == 0 || (ep.tri == 1 ? gj <= gi : gj >= gi))) {
      double* c = ep.C + gi + gj * ep.ldc;
      *c = beta == 0.0 ? 0.0 : beta * *c;
    }
  }
}

// Level L's INT32 sums v of row gi at columns g0 + [0, 32): each folded into
// C with one rounding, C = alpha 2^(ei + ej - 7L) v + (L == 2 ? beta C : C),
// or written as they are (every level, or only the requested one).
__device__ __forceinline__ void oz_fold32(const OzEpi& ep, const int* v, long long gi, long long g0, int ei, int L,
                                          double beta) {
  // the columns g0 + [lo, hi) of this row that are written: one range per
  // row instead of a 64-bit triangle test per element
  long long hl = (long long)ep.N - g0, ll = 0;
  if (ep.tri == 1) hl = min(hl, gi - g0 + 1);  // gj <= gi
  if (ep.tri == 2) ll = gi - g0;               // gj >= gi
  const int hi = (int)max(0LL, min(32LL, hl)), lo = (int)max(0LL, min(32LL, ll));
  if (ep.raw_level != 0) {
    if (ep.raw_level != kOzRawAll && L != ep.raw_level) return;
    int* const out = ep.raw_out + (ep.raw_level == kOzRawAll ? (long long)(L - 2) * ep.raw_plane : 0LL);
#pragma unroll
    for (int j = 0; j < 32; ++j)
      if (j >= lo && j < hi) out[gi + (g0 + j) * ep.ld_raw] = v[j];
    return;
  }
  double old[32];
  bool keep[32];
  int ejs[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    keep[j] = j >= lo && j < hi;
    old[j] = 0.0;
    ejs[j] = 0;
    if (keep[j]) {
      if (L > 2 || beta != 0.0) old[j] = ep.C[gi + (g0 + j) * ep.ldc];
      ejs[j] = oz_row_exp(ep.eB, g0 + j);
    }
  }
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (!keep[j]) continue;
    const double scale = ep.alpha * pow2i(ei + ejs[j] - 7 * L);
    const double base = (L == 2) ? beta * old[j] : old[j];
    ep.C[gi + (g0 + j) * ep.ldc] = fma(scale, (double)v[j], base);
  }
}

__global__ void __launch_bounds__(192, 1) oz_gemm_kernel(const __grid_constant__ OzArgs args) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kOzStages * kOzStageBytes);
  uint64_t* empty = full + kOzStages;
  uint64_t* tfull = empty + kOzStages;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = args.S;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kOzStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_map(&args.mapA);
    tma_prefetch_map(&args.mapB);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      uint32_t issued_mask = 0, phase_mask = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
        const int4 tile = args.tiles[t];
        const int kb0 = tile.z & (kOzAccumulate - 1), kb1 = tile.w;
        for (int L = 2; L <= S + 1 && ok; ++L)
          for (int s = level_pairs_begin(L, S); s <= level_pairs_end(L, S) && ok; ++s)
            for (int kb = kb0; kb < kb1; ++kb) {
              if (!mbar_wait(&empty[st], ph ^ 1u, abort_flag, args.err, kDevErrTimeoutProducer)) {
                ok = false;
                break;
              }
              int kbb = kb + args.kb_shift;
              if (args.kb_mod > 0 && kbb >= args.kb_mod) kbb -= args.kb_mod;
              mbar_arrive_expect_tx(&full[st], kOzStageBytes);
              uint8_t* dst = smem + st * kOzStageBytes;
              tma_load_3d(dst, &args.mapA, &full[st], kb * kOzBK, tile.x, s - 1);
              tma_load_3d(dst + kOzABytes, &args.mapB, &full[st], kbb * kOzBK, tile.y, L - s - 1);
              issued_mask |= 1u << st;
              phase_mask = (phase_mask & ~(1u << st)) | (ph << st);
              if (++st == kOzStages) {
                st = 0;
                ph ^= 1u;
              }
            }
      }
      if (!ok) {
        for (int i = 0; i < kOzStages; ++i) {
          if (!((issued_mask >> i) & 1u)) continue;
          const uint64_t t0 = globaltimer_ns();
          while (!mbar_try_wait(&full[i], (phase_mask >> i) & 1u))
            if (globaltimer_ns() - t0 > 1000000000ull) break;
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      int it = 0;
      bool ok = true, any = false;
      for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
        const int4 tile = args.tiles[t];
        const int kb0 = tile.z & (kOzAccumulate - 1), kb1 = tile.w;
        if (kb1 <= kb0) continue;  // empty product: no accumulator round trip
        for (int L = 2; L <= S + 1 && ok; ++L, ++it) {
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          if (!mbar_wait(&tempty[buf], tph ^ 1u, abort_flag, args.err, kDevErrTimeoutMma)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem_base + (uint32_t)(buf * kOzBN);
          bool first = true;
          for (int s = level_pairs_begin(L, S); s <= level_pairs_end(L, S) && ok; ++s)
            for (int kb = kb0; kb < kb1; ++kb) {
              if (!mbar_wait(&full[st], ph, abort_flag, args.err, kDevErrTimeoutMma)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const uint32_t a = smem_u32(smem + st * kOzStageBytes), b = a + kOzABytes;
#pragma unroll
              for (int kk = 0; kk < kOzBK / 32; ++kk) {
                umma_i8(d, sdesc_sw128(a + kk * 32, 16, 1024), sdesc_sw128(b + kk * 32, 16, 1024), kOzIdesc,
                        first ? 0u : 1u);
                first = false;
              }
              any = true;
              tc_commit(&empty[st]);
              if (++st == kOzStages) {
                st = 0;
                ph ^= 1u;
              }
            }
          if (!ok) break;
          tc_commit(&tfull[buf]);
        }
      }
      if (!ok && any) {
        tc_commit(drain);
        const uint64_t t0 = globaltimer_ns();
        while (!mbar_try_wait(drain, 0))
          if (globaltimer_ns() - t0 > 1000000000ull) break;
      }
    }
    __syncwarp();
  } else {
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    const OzEpi ep = oz_epi(args);
    int it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
      const int4 tile = args.tiles[t];
      const double beta = (tile.z & kOzAccumulate) ? 1.0 : args.beta;
      const long long gi = (long long)tile.x + row;
      const bool row_ok = gi < ep.M;
      const int ei = row_ok ? oz_row_exp(ep.eA, gi) : 0;
      if (tile.w <= (tile.z & (kOzAccumulate - 1))) {
        if (row_ok) oz_scale_row(ep, gi, tile.y, beta);
        continue;
      }
      for (int L = 2; L <= S + 1; ++L, ++it) {
        const int buf = it & 1;
        const uint32_t tph = (uint32_t)(it >> 1) & 1u;
        if (!mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * kOzBN);
#pragma unroll 1
        for (int c0 = 0; c0 < kOzBN; c0 += 32) {
          int v[32];
          tmem_ld32_s32(tacc + c0, v);
          if (row_ok) oz_fold32(ep, v, gi, (long long)tile.y + c0, ei, L, beta);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[buf]);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem_base, 512);
}

// ---------------------------------------------------------------- CTA pairs
// The same product on 256 x 256 tiles, each run by a cluster of two CTAs on
// two SMs (tcgen05 cta_group::2): CTA r loads rows tile.x + 128 r of the A
// planes and rows tile.y + 128 r of the B planes into its own shared memory;
// the leader (r = 0) issues the 256-row MMA, which reads both CTAs' halves,
// and each CTA's TMEM receives its 128 accumulator rows, which its own
// epilogue stores or folds. Per SM one 128-deep K block moves 32 KB from L2 instead of
// the single-CTA tile's 48 KB for the same MMA work. The level sums are the
// same exact integers and the fold the same arithmetic, so the results are
// bit-identical to the single-CTA kernel's.
//   full[s]   leader only: both CTAs' loads complete_tx on it, the leader's
//             producer arms it with both CTAs' bytes;
//   empty[s]  both CTAs: the leader's commit multicasts to the pair;
//   tfull[b]  both CTAs: the leader's commit multicasts to the pair;
//   tempty[b] leader only: the 8 epilogue warps of the pair arrive remotely.
// Every wait is bounded; a cluster barrier before TMEM is freed keeps either
// CTA from leaving while the pair's MMAs or remote arrivals may still touch it.
constexpr int kOzPairStages = 6;
constexpr int kOzPairStageBytes = 2 * kOzABytes;  // 128 rows of A and 128 rows of B planes
constexpr int kOzPairSmem = kOzPairStages * kOzPairStageBytes + 1024 + 256;
static_assert(kOzPairSmem <= 232448, "shared memory budget");
constexpr uint32_t kOzPairIdesc =
    (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kOzBN >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);

__device__ __forceinline__ void umma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 3-D tiled load into this CTA's shared memory whose completion is counted on
// the pair leader's mbarrier (`leader_bar`, a shared::cluster address). No
// multicast: every CTA fetches only its own half.
__device__ __forceinline__ void tma_load_3d_pair(void* smem_dst, const CUtensorMap* map, uint32_t leader_bar, int x,
                                                 int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
      "%5}], [%2];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(leader_bar), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(192, 1) oz_pair_kernel(const __grid_constant__ OzArgs args) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kOzPairStages * kOzPairStageBytes);
  uint64_t* empty = full + kOzPairStages;
  uint64_t* tfull = empty + kOzPairStages;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = args.S;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kOzPairStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 8);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_map(&args.mapA);
    tma_prefetch_map(&args.mapB);
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_slot, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // the peer's barriers exist before any remote arrival
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t full_leader = mapa_shared(smem_u32(full), 0);
  const uint32_t tempty_leader = mapa_shared(smem_u32(tempty), 0);

  if (warp == 0) {
    // ------------------------------------------------------------ producers (both CTAs)
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      uint32_t issued_mask = 0, phase_mask = 0;
      bool ok = true;
      for (int t = pair; t < args.num_tiles && ok; t += npairs) {
        const int4 tile = args.tiles[t];
        const int kb0 = tile.z & (kOzAccumulate - 1), kb1 = tile.w;
        for (int L = 2; L <= S + 1 && ok; ++L)
          for (int s = level_pairs_begin(L, S); s <= level_pairs_end(L, S) && ok; ++s)
            for (int kb = kb0; kb < kb1; ++kb) {
              if (!mbar_wait(&empty[st], ph ^ 1u, abort_flag, args.err, kDevErrTimeoutProducer)) {
                ok = false;
                break;
              }
              int kbb = kb + args.kb_shift;
              if (args.kb_mod > 0 && kbb >= args.kb_mod) kbb -= args.kb_mod;
              if (leader) mbar_arrive_expect_tx(&full[st], 2 * kOzPairStageBytes);
              uint8_t* dst = smem + st * kOzPairStageBytes;
              const uint32_t bar = full_leader + 8u * (uint32_t)st;
              tma_load_3d_pair(dst, &args.mapA, bar, kb * kOzBK, tile.x + 128 * (int)rank, s - 1);
              tma_load_3d_pair(dst + kOzABytes, &args.mapB, bar, kbb * kOzBK, tile.y + 128 * (int)rank, L - s - 1);
              issued_mask |= 1u << st;
              phase_mask = (phase_mask & ~(1u << st)) | (ph << st);
              if (++st == kOzPairStages) {
                st = 0;
                ph ^= 1u;
              }
            }
      }
      if (!ok) {
        // Abort path: the leader sees its loads land on its own barriers; the
        // peer's loads report to the leader, so the peer waits a bounded time.
        if (leader) {
          for (int i = 0; i < kOzPairStages; ++i) {
            if (!((issued_mask >> i) & 1u)) continue;
            const uint64_t t0 = globaltimer_ns();
            while (!mbar_try_wait(&full[i], (phase_mask >> i) & 1u))
              if (globaltimer_ns() - t0 > 1000000000ull) break;
          }
        } else {
          const uint64_t t0 = globaltimer_ns();
          while (globaltimer_ns() - t0 < 2000000ull) {
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer (leader)
    if (leader && lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      int it = 0;
      bool ok = true, any = false;
      for (int t = pair; t < args.num_tiles && ok; t += npairs) {
        const int4 tile = args.tiles[t];
        const int kb0 = tile.z & (kOzAccumulate - 1), kb1 = tile.w;
        if (kb1 <= kb0) continue;  // empty product: no accumulator round trip
        for (int L = 2; L <= S + 1 && ok; ++L, ++it) {
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          if (!mbar_wait(&tempty[buf], tph ^ 1u, abort_flag, args.err, kDevErrTimeoutMma)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem_base + (uint32_t)(buf * kOzBN);
          bool first = true;
          for (int s = level_pairs_begin(L, S); s <= level_pairs_end(L, S) && ok; ++s)
            for (int kb = kb0; kb < kb1; ++kb) {
              if (!mbar_wait(&full[st], ph, abort_flag, args.err, kDevErrTimeoutMma)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const uint32_t a = smem_u32(smem + st * kOzPairStageBytes), b = a + kOzABytes;
#pragma unroll
              for (int kk = 0; kk < kOzBK / 32; ++kk) {
                umma_i8_pair(d, sdesc_sw128(a + kk * 32, 16, 1024), sdesc_sw128(b + kk * 32, 16, 1024), kOzPairIdesc,
                             first ? 0u : 1u);
                first = false;
              }
              any = true;
              tc_commit_pair(&empty[st], 3);
              if (++st == kOzPairStages) {
                st = 0;
                ph ^= 1u;
              }
            }
          if (!ok) break;
          tc_commit_pair(&tfull[buf], 3);
        }
      }
      if (!ok && any) {
        tc_commit_pair(drain, 1);
        const uint64_t t0 = globaltimer_ns();
        while (!mbar_try_wait(drain, 0)) {
          if (globaltimer_ns() - t0 > 1000000000ull) {
            if (args.err) atomicCAS(args.err, 0, kDevErrTimeoutTeardown);
            break;
          }
        }
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue (both CTAs)
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    const OzEpi ep = oz_epi(args);
    int it = 0;
    bool ok = true;
    for (int t = pair; t < args.num_tiles && ok; t += npairs) {
      const int4 tile = args.tiles[t];
      const double beta = (tile.z & kOzAccumulate) ? 1.0 : args.beta;
      const long long gi = (long long)tile.x + 128 * (int)rank + row;
      const bool row_ok = gi < ep.M;
      const int ei = row_ok ? oz_row_exp(ep.eA, gi) : 0;
      if (tile.w <= (tile.z & (kOzAccumulate - 1))) {
        if (row_ok) oz_scale_row(ep, gi, tile.y, beta);
        continue;
      }
      for (int L = 2; L <= S + 1; ++L, ++it) {
        const int buf = it & 1;
        const uint32_t tph = (uint32_t)(it >> 1) & 1u;
        if (!mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * kOzBN);
#pragma unroll 1
        for (int c0 = 0; c0 < kOzBN; c0 += 32) {
          int v[32];
          tmem_ld32_s32(tacc + c0, v);
          if (c0 == kOzBN - 32) {  // this CTA's half of the accumulator is read: tell the leader
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(tempty_leader + 8u * (uint32_t)buf);
          }
          if (row_ok) oz_fold32(ep, v, gi, (long long)tile.y + c0, ei, L, beta);
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // the pair's MMAs, remote arrivals and TMEM reads are over
  tc_fence_after();
  if (warp == 1) tmem_dealloc_pair(tmem_base, 512);
}

// ---------------------------------------------------------------- level fold
// FP64 instructions issued while an SM's tensor core runs tcgen05 MMAs wait
// until the MMAs pause: folded in the GEMM's epilogue, a level's fold ended
// only when the next level's MMAs did, and the MMA issuer then waited 30-70
// us per level for its accumulator (measured with %globaltimer stamps). So
// large products write every level's exact INT32 sums to a workspace and this
// kernel folds them afterwards with the same arithmetic, in the same order,
// as the epilogue fold (results are bit-identical):
//   c = beta (beta != 0 ? C : 0); c = fma(alpha 2^(ei + ej - 7L), P_L, c),
//   L = 2 .. S + 1.
// One block per 32-column slab of a tile of the GEMM's tile list (tile_rows
// rows; eight slabs per tile, so even a one-wave GEMM gives every SM several
// blocks); a thread takes one row. The slab's level sums stream through
// shared memory: per column, S contiguous runs of the tile's rows (one per
// level) are fetched by bulk copies into a ring of kOzFoldStages stages, so
// up to kOzFoldStages * S * tile_rows * 4 bytes per block are in flight
// without holding them in registers, and the threads fold column q while the
// copies of the next columns land. The workspace's leading dimension is a
// multiple of 32 rows, so the runs never leave it (rows at or past M are
// fetched and not used). Every wait is bounded.
constexpr int kOzFoldSlab = 32;
constexpr int kOzFoldStages = 4;
__host__ __device__ constexpr int oz_fold_smem(int S, int tile_rows) { return kOzFoldStages * S * tile_rows * 4; }

__global__ void __launch_bounds__(256) oz_fold_kernel(const int4* __restrict__ tiles, int tile_rows, int M, int N,
                                                      int tri, int S, double alpha, double beta, double* C,
                                                      long long ldc, const int* __restrict__ eA,
                                                      const int* __restrict__ eB, const int* __restrict__ raw,
                                                      long long ld_raw, long long plane, int* err) {
  extern __shared__ __align__(128) int fold_buf[];
  __shared__ uint64_t bars[kOzFoldStages];
  __shared__ int abort_flag;
  const int4 tile = tiles[blockIdx.x / (kOzBN / kOzFoldSlab)];
  const int c0 = (int)(blockIdx.x % (kOzBN / kOzFoldSlab)) * kOzFoldSlab;
  const double b = (tile.z & kOzAccumulate) ? 1.0 : beta;
  const bool empty = tile.w <= (tile.z & (kOzAccumulate - 1));
  const int tid = threadIdx.x;
  if (empty) {
    for (int r = tid; r < tile_rows; r += blockDim.x) {
      const long long i = (long long)tile.x + r;
      if (i >= M) break;
      for (int c = c0; c < c0 + kOzFoldSlab; ++c) {
        const long long j = (long long)tile.y + c;
        if (j >= N || (tri == 1 && j > i)) break;  // columns only grow
        if (tri == 2 && j < i) continue;
        double* const cp = C + i + j * ldc;
        if (b != 1.0) *cp = b == 0.0 ? 0.0 : b * *cp;
      }
    }
    return;
  }
  // the slab's columns with work: [cb, ce)
  long long ce = std::min<long long>(c0 + kOzFoldSlab, (long long)N - tile.y);
  if (tri == 1) ce = std::min<long long>(ce, (long long)tile.x + tile_rows - tile.y);  // some row i >= j
  long long cb = c0;
  if (tri == 2) cb = std::max<long long>(cb, (long long)tile.x - tile.y);  // some row i <= j
  const int ncols = (int)(ce - cb);
  if (ncols <= 0) return;
  const int run = (int)std::min<long long>(tile_rows, ld_raw - tile.x);  // rows fetched per level (multiple of 32)
  const uint32_t run_bytes = (uint32_t)run * 4u;
  if (tid == 0) {
    for (int s = 0; s < kOzFoldStages; ++s) mbar_init(&bars[s], 1);
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int q) {  // column cb + q into stage q % kOzFoldStages (thread 0)
    const int s = q % kOzFoldStages;
    const long long j = (long long)tile.y + cb + q;
    mbar_arrive_expect_tx(&bars[s], run_bytes * (uint32_t)S);
    for (int l = 0; l < S; ++l)
      bulk_load(fold_buf + (s * S + l) * tile_rows, raw + tile.x + j * ld_raw + l * plane, run_bytes, &bars[s]);
  };
  if (tid == 0)
    for (int q = 0; q < kOzFoldStages && q < ncols; ++q) issue(q);
  const long long i = (long long)tile.x + tid;
  const bool row_ok = tid < tile_rows && i < M;
  const int ei = row_ok ? oz_row_exp(eA, i) : 0;
  int q = 0;
  for (; q < ncols; ++q) {
    const int s = q % kOzFoldStages;
    const bool ok = mbar_wait(&bars[s], (uint32_t)(q / kOzFoldStages) & 1u, &abort_flag, err, kDevErrTimeoutEpilogue);
    if (__syncthreads_or(!ok)) break;
    const long long j = (long long)tile.y + cb + q;
    if (row_ok && !(tri == 1 && j > i) && !(tri == 2 && j < i)) {
      const int ej = oz_row_exp(eB, j);
      double* const cp = C + i + j * ldc;
      const int* const v = fold_buf + s * S * tile_rows + tid;
      double acc = b * (b != 0.0 ? *cp : 0.0);
      for (int l = 0; l < S; ++l) acc = fma(alpha * pow2i(ei + ej - 7 * (l + 2)), (double)v[l * tile_rows], acc);
      *cp = acc;
    }
    __syncthreads();  // stage s is read
    if (tid == 0 && q + kOzFoldStages < ncols) issue(q + kOzFoldStages);
  }
  if (q < ncols && tid == 0) {
    // a wait gave up: let the copies already issued land before the block
    // leaves (bounded)
    const uint64_t t0 = globaltimer_ns();
    for (int r = q; r < ncols && r < q + kOzFoldStages; ++r)
      while (!mbar_try_wait(&bars[r % kOzFoldStages], (uint32_t)(r / kOzFoldStages) & 1u))
        if (globaltimer_ns() - t0 > 1000000000ull) break;
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode3() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

tb_status make_q_map(CUtensorMap* map, int8_t* Q, long long ldq, long long n, int S, int box_rows) {
  EncodeTiledFn enc = encode3();
  if (!enc) return TB_ERROR_CUDA;
  cuuint64_t dims[3] = {(cuuint64_t)ldq, (cuuint64_t)n, (cuuint64_t)S};
  cuuint64_t strides[2] = {(cuuint64_t)ldq, (cuuint64_t)(ldq * n)};
  cuuint32_t box[3] = {(cuuint32_t)kOzBK, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, Q, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("ozaki: cuTensorMapEncodeTiled failed (%d)", (int)r);
    return TB_ERROR_CUDA;
  }
  return TB_SUCCESS;
}

// ---------------------------------------------------------------- host side
// Largest K chunk whose level sums stay exact in INT32:
// (pairs per level <= S) * K * 127^2 < 2^31.
long long oz_kmax(int S) { return ((2147483647LL / ((long long)S * 127 * 127)) / kOzBK) * kOzBK; }

struct OzOperand {
  const double* X = nullptr;
  long long ld = 0;
  long long rows = 0, k = 0;
  bool by_cols = false;
  int mask = 0;
  long long koff = 0;
  // the K sub-range [k0, k0 + kc) of the operand, as an operand of its own
  OzOperand chunk(long long k0, long long kc) const {
    OzOperand o = *this;
    o.X = by_cols ? X + k0 : X + k0 * ld;
    o.k = kc;
    o.koff = koff + k0;
    return o;
  }
};

// Planes of one operand: S int8 planes [rows][ldq] and row exponents.
struct OzPlanes {
  int8_t* Q = nullptr;
  long long ldq = 0, rows = 0;
  int* e = nullptr;
};

tb_status oz_exponents(const OzOperand& o, int* e, cudaStream_t st) {
  if (o.rows == 0 || o.k == 0) return TB_SUCCESS;
  if (o.by_cols) {
    oz_exp_cols_kernel<<<(unsigned)((o.rows + 7) / 8), 256, 0, st>>>(o.rows, o.k, o.X, o.ld, o.mask, o.koff, e);
  } else {
    dim3 g((unsigned)((o.rows + 255) / 256), (unsigned)(o.k < 64 ? o.k : 64));
    oz_exp_rows_kernel<<<g, 256, 0, st>>>(o.rows, o.k, o.X, o.ld, o.mask, o.koff, e);
  }
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

// Writes columns [qoff, qoff + kw) of the planes (zeros beyond o.k).
tb_status oz_slice(const OzOperand& o, const int* e, int S, const OzPlanes& q, long long qoff, long long kw,
                   cudaStream_t st) {
  if (o.rows == 0 || kw == 0) return TB_SUCCESS;
  dim3 g((unsigned)((o.rows + 31) / 32), (unsigned)((kw + 127) / 128));
  if (o.by_cols)
    oz_slice_cols_kernel<<<g, 256, 0, st>>>(o.rows, o.k, o.X, o.ld, o.mask, o.koff, e, S, q.Q, q.ldq, q.ldq * q.rows,
                                            qoff, kw);
  else
    oz_slice_rows_kernel<<<g, 256, 0, st>>>(o.rows, o.k, o.X, o.ld, o.mask, o.koff, e, S, q.Q, q.ldq, q.ldq * q.rows,
                                            qoff, kw);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

// Exponents + slices of one operand into fresh planes.
tb_status oz_prepare(const OzOperand& o, int S, const OzPlanes& q, cudaStream_t st) {
  TB_CUDA_TRY(cudaMemsetAsync(q.e, 0x80, sizeof(int) * (size_t)(o.rows > 0 ? o.rows : 1), st));
  TB_TRY(oz_exponents(o, q.e, st));
  return oz_slice(o, q.e, S, q, 0, q.ldq, st);
}

size_t oz_planes_bytes(long long rows, long long ldq, int S) {
  return (size_t)round_up((long long)S * rows * ldq, 256) + (size_t)round_up(rows * 4 + 4, 256);
}

// Carves planes for `rows` x ldq out of ws (advancing it).
OzPlanes oz_carve(char*& ws, long long rows, long long ldq, int S) {
  OzPlanes q;
  q.rows = rows;
  q.ldq = ldq;
  q.Q = reinterpret_cast<int8_t*>(ws);
  ws += round_up((long long)S * rows * ldq, 256);
  q.e = reinterpret_cast<int*>(ws);
  ws += round_up(rows * 4 + 4, 256);
  return q;
}

// Per-tile K range of a product chunk [k0, k1) of an operand pair whose
// product vanishes outside [kbeg(m0, n0), kend(m0, n0)).
enum class KRange {
  kFull,       // [0, K)
  kRowsLower,  // A lower triangular by rows:      [0, m0 + BM)
  kRowsUpper,  // A upper triangular by rows:      [m0, K)
  kColsLower,  // B operand lower triangular:      [0, n0 + BN)
};

// tiles: 0 all tiles of M x N, 1 those meeting the lower triangle, 2 the upper.
std::vector<int4> oz_plan(int M, int N, int tiles, KRange kr, long long K, long long k0, long long k1,
                          bool first_chunk) {
  std::vector<int4> plan = tiles == 1   ? plan_lower(M, kOzBN, 0, 0)
                           : tiles == 2 ? plan_upper(M, kOzBN, 0, 0)
                                        : plan_rect(M, N, kOzBN, 0, 0);
  std::vector<int4> out;
  out.reserve(plan.size());
  for (int4 t : plan) {
    long long b = 0, e = K;
    if (kr == KRange::kRowsLower) e = std::min<long long>(K, (long long)t.x + kOzBM);
    if (kr == KRange::kRowsUpper) b = t.x;
    if (kr == KRange::kColsLower) e = std::min<long long>(K, (long long)t.y + kOzBN);
    // tiles whose whole range lies in an earlier chunk were written there
    b = std::max(b, k0);
    e = std::min(e, k1);
    if (e <= b) {
      if (!first_chunk) continue;
      t.z = t.w = 0;  // empty product: the kernel only applies beta to the tile
    } else {
      // every tile is written by the first chunk; later chunks accumulate
      t.z = (int)((b - k0) / kOzBK) | (first_chunk ? 0 : kOzAccumulate);
      t.w = (int)((e - k0 + kOzBK - 1) / kOzBK);
    }
    out.push_back(t);
  }
  return out;
}

// Products of at least 256 x 256 run on CTA pairs; TB_OZ_PAIR=0 in the
// environment keeps them on single CTAs (read once; the two give
// bit-identical results, so this only compares their speed).
bool oz_pair_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("TB_OZ_PAIR");
    on = (e && e[0] == '0') ? 0 : 1;
  }
  return on == 1;
}

// Products fold their levels after the GEMM (oz_fold_kernel) when the INT32
// level sums fit in kOzLevelBytesMax of workspace; TB_OZ_FOLD=fused in the
// environment folds them in the GEMM's epilogue instead (read once; the two
// give bit-identical results).
constexpr double kOzLevelBytesMax = 32.0 * (1ull << 30);
bool oz_split_fold_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("TB_OZ_FOLD");
    on = (e && strcmp(e, "fused") == 0) ? 0 : 1;
  }
  return on == 1;
}

// Vertically adjacent 128-row tiles of a plan merged into 256-row pair tiles.
// A pair tile's K range spans both halves' ranges: a half's product outside
// its own range multiplies plane values that are zero there (the slicing
// masks triangular operands; leaf inverses store zeros above the diagonal),
// and an empty half adds no range (its rows then fold zero products, which
// leaves beta C).
std::vector<int4> oz_pair_plan(const std::vector<int4>& plan, int M, int N) {
  const long long rb = ((long long)M + 255) / 256, cb = ((long long)N + kOzBN - 1) / kOzBN;
  std::vector<int> where((size_t)(rb * cb), -1);
  std::vector<int4> out;
  out.reserve(plan.size());
  for (const int4& t : plan) {
    int& w = where[(size_t)((long long)(t.x >> 8) * cb + t.y / kOzBN)];
    if (w < 0) {
      w = (int)out.size();
      out.push_back(make_int4((t.x >> 8) << 8, t.y, t.z, t.w));
      continue;
    }
    int4& m = out[w];
    const int tz = t.z & (kOzAccumulate - 1), mz = m.z & (kOzAccumulate - 1);
    if (t.w <= tz) continue;  // empty half
    if (m.w <= mz) {          // only the other half's range so far: empty
      m.z = t.z;
      m.w = t.w;
      continue;
    }
    m.z = (tz < mz ? tz : mz) | (t.z & kOzAccumulate);
    m.w = t.w > m.w ? t.w : m.w;
  }
  return out;
}

tb_status oz_launch(const OzPlanes& a, const OzPlanes& b, int kb_shift, int kb_mod, const std::vector<int4>& plan,
                    int M, int N, int tri, double alpha, double* C, long long ldc, double beta, int S, double flops,
                    int raw_level, int* raw_out, long long ld_raw, cudaStream_t st) {
  if (plan.empty()) return TB_SUCCESS;
  const bool pair = M >= 256 && N >= 256 && oz_pair_enabled();
  // fold after the GEMM (oz_fold_kernel) when the levels' workspace fits
  const long long ld_r = round_up((long long)M, 32), plane = ld_r * (long long)N;
  int* levels = nullptr;
  // (at most kOzLevelBytesMax, and no more than half of the device memory
  // still free unless the pool slot already holds it: an application sharing
  // the GPU keeps its headroom, and the fused fold needs no workspace)
  const double level_bytes = (double)S * plane * 4.0;
  if (raw_level == 0 && oz_split_fold_enabled() && level_bytes <= kOzLevelBytesMax &&
      (level_bytes <= (double)pool_capacity(2) || level_bytes <= 0.5 * (double)free_device_bytes()))
    levels = static_cast<int*>(pool_get((size_t)S * (size_t)plane * 4, 2));
  OzArgs g;
  memset(&g, 0, sizeof(g));
  TB_TRY(make_q_map(&g.mapA, a.Q, a.ldq, a.rows, S, kOzBM));
  TB_TRY(make_q_map(&g.mapB, b.Q, b.ldq, b.rows, S, pair ? 128 : kOzBN));
  const std::vector<int4> pair_plan = pair ? oz_pair_plan(plan, M, N) : std::vector<int4>();
  const std::vector<int4>& tiles = pair ? pair_plan : plan;
  g.tiles = upload_tiles(tiles, st);
  if (!g.tiles) return TB_ERROR_ALLOC;
  g.num_tiles = (int)tiles.size();
  g.S = S;
  g.kb_shift = kb_shift;
  g.kb_mod = kb_mod;
  g.M = M;
  g.N = N;
  g.tri = tri;
  g.C = C;
  g.ldc = ldc;
  g.alpha = alpha;
  g.beta = beta;
  g.eA = a.e;
  g.eB = b.e;
  g.raw_level = levels ? kOzRawAll : raw_level;
  g.raw_out = levels ? levels : raw_out;
  g.ld_raw = levels ? ld_r : ld_raw;
  g.raw_plane = plane;
  g.err = device_error_word();
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr[dev]) {
    TB_CUDA_TRY(cudaFuncSetAttribute(oz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzSmem));
    TB_CUDA_TRY(cudaFuncSetAttribute(oz_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzPairSmem));
    TB_CUDA_TRY(cudaFuncSetAttribute(oz_fold_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     oz_fold_smem(kOzMaxSlices, 256)));
    attr[dev] = true;
  }
  void* tok = prof_begin(st, kProfOzaki);
  if (pair) {
    const int pairs_max = sm_count() / 2;
    const int pairs = g.num_tiles < pairs_max ? g.num_tiles : pairs_max;
    oz_pair_kernel<<<2 * pairs, 192, kOzPairSmem, st>>>(g);
  } else {
    const int grid = g.num_tiles < sm_count() ? g.num_tiles : sm_count();
    oz_gemm_kernel<<<grid, 192, kOzSmem, st>>>(g);
  }
  TB_CUDA_TRY(cudaGetLastError());
  if (levels) {
    note_launch();
    const int tile_rows = pair ? 256 : kOzBM;
    oz_fold_kernel<<<g.num_tiles * (kOzBN / kOzFoldSlab), 256, oz_fold_smem(S, tile_rows), st>>>(
        g.tiles, tile_rows, M, N, tri, S, alpha, beta, C, ldc, g.eA, g.eB, levels, ld_r, plane, g.err);
    TB_CUDA_TRY(cudaGetLastError());
  }
  prof_end(tok, st, flops);
  note_launch();
  return TB_SUCCESS;
}

// Automatic slice count. Truncating row i after S slices of 7 bits leaves
// an error below 2^(e_i - 7S) per entry; relative to the row's root mean
// square that is 2^(d_i - 7S), which the dot products carry into C at about
// the same relative size. S is the smallest count with 7S >= 50 + max_i d_i
// (2^-50 ~ 9e-16 of headroom under the 1e-14 target), at least 8 (the 53
// bits of the significand) and at most kOzMaxSlices.
constexpr int kOzAutoBits = 50;

int oz_slices_for_spread(double spread_bits) {
  int S = (int)std::ceil((kOzAutoBits + spread_bits) / 7.0);
  return std::max(8, std::min(kOzMaxSlices, S));
}

// Largest row spread of the operands (bits), one small device word per device.
tb_status oz_max_spread(const std::vector<OzOperand>& ops, cudaStream_t st, double* spread) {
  static int* word[64] = {};
  static std::mutex mu;
  int dev = 0;
  TB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return TB_ERROR_NOT_SUPPORTED;
  int* w = nullptr;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!word[dev] && dev_malloc(reinterpret_cast<void**>(&word[dev]), 256) != cudaSuccess) {
      cudaGetLastError();
      word[dev] = nullptr;
      return TB_ERROR_ALLOC;
    }
    w = word[dev];
  }
  TB_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(int), st));
  for (const OzOperand& o : ops) {
    if (o.rows == 0 || o.k == 0) continue;
    if (o.by_cols)
      oz_spread_cols_kernel<<<(unsigned)((o.rows + 7) / 8), 256, 0, st>>>(o.rows, o.k, o.X, o.ld, o.mask, o.koff, w);
    else
      oz_spread_rows_kernel<<<(unsigned)((o.rows + 15) / 16), 256, 0, st>>>(o.rows, o.k, o.X, o.ld, o.mask, o.koff,
                                                                           w);
    TB_CUDA_TRY(cudaGetLastError());
    note_launch();
  }
  int h = 0;
  TB_CUDA_TRY(cudaMemcpyAsync(&h, w, sizeof(int), cudaMemcpyDeviceToHost, st));
  TB_CUDA_TRY(cudaStreamSynchronize(st));
  *spread = h / 256.0;
  return TB_SUCCESS;
}

tb_status check_slices(int S) {
  if (S < 1 || S > kOzMaxSlices) {
    set_last_error("ozaki: slices must be in [1, %d]", kOzMaxSlices);
    return TB_ERROR_INVALID_VALUE;
  }
  return TB_SUCCESS;
}

// Scratch of oz_gemm for operands of at most ra / rb rows and K.
size_t oz_gemm_ws(long long ra, long long rb, long long K, int S) {
  const long long ldq = round_up(std::min<long long>(std::max<long long>(K, 1), oz_kmax(S)), kOzBK);
  return oz_planes_bytes(ra, ldq, S) + oz_planes_bytes(rb, ldq, S);
}

// C (M x N) = alpha * a (M x K) * b (N x K)^T + beta * C in FP64 on the INT8
// tensor cores, in K chunks of at most oz_kmax(S). ws: oz_gemm_ws bytes.
tb_status oz_gemm(const OzOperand& a, const OzOperand& b, long long K, KRange kr, bool lower_tiles, double alpha,
                  double* C, long long ldc, double beta, int S, double flops, char* ws, cudaStream_t st) {
  const int M = (int)a.rows, N = (int)b.rows;
  if (M == 0 || N == 0) return TB_SUCCESS;
  const long long kc_max = oz_kmax(S);
  const long long ldq = round_up(std::min<long long>(std::max<long long>(K, 1), kc_max), kOzBK);
  OzPlanes qa = oz_carve(ws, M, ldq, S);
  OzPlanes qb = oz_carve(ws, N, ldq, S);
  const long long K1 = K > 0 ? K : 1;  // K == 0: one all-zero chunk applies beta
  for (long long k0 = 0; k0 < K1; k0 += kc_max) {
    const long long kc = std::min(kc_max, K1 - k0);
    const long long kreal = std::max(0LL, std::min(kc, K - k0));
    TB_TRY(oz_prepare(a.chunk(k0, kreal), S, qa, st));
    TB_TRY(oz_prepare(b.chunk(k0, kreal), S, qb, st));
    const std::vector<int4> plan = oz_plan(M, N, lower_tiles ? 1 : 0, kr, K1, k0, k0 + kc, k0 == 0);
    TB_TRY(oz_launch(qa, qb, 0, 0, plan, M, N, lower_tiles ? 1 : 0, alpha, C, ldc, beta, S,
                     flops * (double)kc / (double)K1, 0, nullptr, 0, st));
  }
  return TB_SUCCESS;
}

}  // namespace

// Slices A (n x k, column-major) into S int8 planes (K-major, row stride
// ldq; columns [k, kw) written as zeros) and row exponents e[n].
tb_status ozaki_slice(long long n, long long k, const double* A, long long lda, int S, int8_t* Q, long long ldq,
                      long long kw, int* e, cudaStream_t st) {
  OzOperand o;
  o.X = A;
  o.ld = lda;
  o.rows = n;
  o.k = k;
  OzPlanes q;
  q.Q = Q;
  q.ldq = ldq;
  q.rows = n;
  q.e = e;
  TB_CUDA_TRY(cudaMemsetAsync(e, 0x80, sizeof(int) * n, st));
  TB_TRY(oz_exponents(o, e, st));
  return oz_slice(o, e, S, q, 0, kw, st);
}

// FP64 SYRK: C(lower) = alpha A A^T + beta C, A n x k ('N') or k x n ('T').
tb_status ozaki_syrk_impl(bool trans, long n, long k, double alpha, const double* A, long lda, double beta, double* C,
                          long ldc, int S, int raw_level, int* raw_out, long ld_raw, cudaStream_t st,
                          bool upper = false) {
  const long rows_a = trans ? k : n;
  if (n < 0 || k < 0 || lda < (rows_a > 1 ? rows_a : 1) || ldc < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  if (n == 0) return TB_SUCCESS;
  OzOperand a;
  a.X = A;
  a.ld = lda;
  a.rows = n;
  a.k = k;
  a.by_cols = trans;
  if (S <= 0) {
    double spread = 0;
    TB_TRY(oz_max_spread({a}, st, &spread));
    S = oz_slices_for_spread(spread);
  }
  TB_TRY(check_slices(S));
  const long long kc_max = oz_kmax(S);
  if (raw_level >= 2 && k > kc_max) {
    set_last_error("ozaki: level products need k <= %lld with %d slices", kc_max, S);
    return TB_ERROR_NOT_SUPPORTED;
  }
  const long long K1 = k > 0 ? k : 1;
  const long long ldq = round_up(std::min<long long>(K1, kc_max), kOzBK);
  char* ws = static_cast<char*>(pool_get(oz_planes_bytes(n, ldq, S)));
  if (!ws) return TB_ERROR_ALLOC;
  OzPlanes q = oz_carve(ws, n, ldq, S);
  for (long long k0 = 0; k0 < K1; k0 += kc_max) {
    const long long kc = std::min(kc_max, K1 - k0);
    TB_TRY(oz_prepare(a.chunk(k0, std::max(0LL, std::min(kc, (long long)k - k0))), S, q, st));
    const std::vector<int4> plan = oz_plan((int)n, (int)n, upper ? 2 : 1, KRange::kFull, K1, k0, k0 + kc, k0 == 0);
    TB_TRY(oz_launch(q, q, 0, 0, plan, (int)n, (int)n, upper ? 2 : 1, alpha, C, ldc, beta, S,
                     (double)n * (double)(n + 1) * (double)kc, raw_level, raw_out, ld_raw, st));
  }
  return TB_SUCCESS;
}

// FP64 SYR2K: C(lower) = alpha (A B^T + B A^T) + beta C, A and B n x k.
// One product of [A | B] with [B | A]: both share the row exponents of
// [A | B] and one set of planes; the B operand reads the planes with its K
// halves swapped (kb_shift).
tb_status ozaki_syr2k_impl(long n, long k, double alpha, const double* A, long lda, const double* B, long ldb,
                           double beta, double* C, long ldc, int S, cudaStream_t st) {
  if (n < 0 || k < 0 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1) || ldc < (n > 1 ? n : 1))
    return TB_ERROR_INVALID_VALUE;
  if (n == 0) return TB_SUCCESS;
  if (S <= 0) {
    OzOperand a0, b0;
    a0.X = A;
    a0.ld = lda;
    a0.rows = n;
    a0.k = k;
    b0 = a0;
    b0.X = B;
    b0.ld = ldb;
    double spread = 0;
    TB_TRY(oz_max_spread({a0, b0}, st, &spread));
    S = oz_slices_for_spread(spread);
  }
  TB_TRY(check_slices(S));
  const long long kc_max = oz_kmax(S) / 2 / kOzBK * kOzBK;  // the concatenated K is twice the chunk
  const long long K1 = k > 0 ? k : 1;
  const long long kh = round_up(std::min<long long>(K1, kc_max), kOzBK);
  char* ws = static_cast<char*>(pool_get(oz_planes_bytes(n, 2 * kh, S)));
  if (!ws) return TB_ERROR_ALLOC;
  OzPlanes q = oz_carve(ws, n, 2 * kh, S);
  OzOperand a, b;
  a.X = A;
  a.ld = lda;
  a.rows = n;
  a.k = k;
  b = a;
  b.X = B;
  b.ld = ldb;
  for (long long k0 = 0; k0 < K1; k0 += kc_max) {
    const long long kc = std::min(kc_max, K1 - k0);
    const long long kreal = std::max(0LL, std::min(kc, (long long)k - k0));
    const OzOperand ac = a.chunk(k0, kreal), bc = b.chunk(k0, kreal);
    TB_CUDA_TRY(cudaMemsetAsync(q.e, 0x80, sizeof(int) * n, st));
    TB_TRY(oz_exponents(ac, q.e, st));
    TB_TRY(oz_exponents(bc, q.e, st));
    TB_TRY(oz_slice(ac, q.e, S, q, 0, kh, st));
    TB_TRY(oz_slice(bc, q.e, S, q, kh, kh, st));
    const std::vector<int4> plan = oz_plan((int)n, (int)n, 1, KRange::kFull, 2 * kh, 0, 2 * kh, k0 == 0);
    const int khb = (int)(kh / kOzBK);
    // later chunks accumulate: oz_plan marks them only when k0 > 0 via first_chunk
    TB_TRY(oz_launch(q, q, khb, 2 * khb, plan, (int)n, (int)n, 1, alpha, C, ldc, beta, S,
                     2.0 * (double)n * (double)(n + 1) * (double)kc, 0, nullptr, 0, st));
  }
  return TB_SUCCESS;
}

// FP64 TRMM (left, out of place): C = alpha op(A) B, A m x m lower ('L') or
// upper ('U') triangular (the other triangle is never read), B, C m x n.
tb_status ozaki_trmm_impl(bool upper, long m, long n, double alpha, const double* A, long lda, const double* B,
                          long ldb, double* C, long ldc, int S, cudaStream_t st) {
  if (m < 0 || n < 0 || lda < (m > 1 ? m : 1) || ldb < (m > 1 ? m : 1) || ldc < (m > 1 ? m : 1))
    return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  OzOperand a, b;
  a.X = A;
  a.ld = lda;
  a.rows = m;
  a.k = m;
  a.mask = upper ? 2 : 1;
  b.X = B;
  b.ld = ldb;
  b.rows = n;
  b.k = m;
  b.by_cols = true;
  if (S <= 0) {
    double spread = 0;
    TB_TRY(oz_max_spread({a, b}, st, &spread));
    S = oz_slices_for_spread(spread);
  }
  TB_TRY(check_slices(S));
  char* ws = static_cast<char*>(pool_get(oz_gemm_ws(m, n, m, S)));
  if (!ws) return TB_ERROR_ALLOC;
  return oz_gemm(a, b, m, upper ? KRange::kRowsUpper : KRange::kRowsLower, false, alpha, C, ldc, 0.0, S,
                 (double)m * m * n, ws, st);
}

// FP64 TRSM, A lower-triangular non-unit:
//   right: X A^T = B (the reference's tc_ozimmu_trsm), A n x n, B m x n
//   left : A X = B, A m x m
// The same recursion as the FP32 driver (halving at leaf boundaries). Leaves
// multiply by the FP64 inverse of the diagonal block (warp substitution on
// 32x32 blocks plus column chains, all FP64); leaf products and off-diagonal
// updates are Ozaki-scheme FP64 GEMMs on the INT8 tensor cores. Operands are
// sliced into planes before each product, so X can overwrite B in place.
namespace {
struct OzTrsm {
  bool right;
  long m, n, nt;
  const double* A;
  long lda;
  double* B;
  long ldb;
  int leaf;
  double* W;
  long long ldw, wstride;
  int S;
  char* ws;
  cudaStream_t st;
};

tb_status oz_trsm_leaf(OzTrsm& c, int bidx, long s, long e) {
  const long sz = e - s;
  OzOperand w;  // W_b by rows: row j holds W(j, :), lower triangular
  w.X = c.W + bidx * c.wstride;
  w.ld = c.ldw;
  w.rows = sz;
  w.k = sz;
  OzOperand x;
  if (c.right) {
    // B[:, s:e] = B[:, s:e] W^T: rows of B's block against rows of W
    x.X = c.B + s * c.ldb;
    x.ld = c.ldb;
    x.rows = c.m;
    x.k = sz;
    return oz_gemm(x, w, sz, KRange::kColsLower, false, 1.0, c.B + s * c.ldb, c.ldb, 0.0, c.S,
                   (double)c.m * sz * sz, c.ws, c.st);
  }
  // B[s:e, :] = W B[s:e, :]: rows of W against columns of B's block
  x.X = c.B + s;
  x.ld = c.ldb;
  x.rows = c.n;
  x.k = sz;
  x.by_cols = true;
  return oz_gemm(w, x, sz, KRange::kRowsLower, false, 1.0, c.B + s, c.ldb, 0.0, c.S, (double)c.n * sz * sz, c.ws,
                 c.st);
}

tb_status oz_trsm_update(OzTrsm& c, long s, long mid, long e) {
  const long kk = mid - s;
  OzOperand a21;  // A[mid:e, s:mid] by rows
  a21.X = c.A + mid + s * c.lda;
  a21.ld = c.lda;
  a21.rows = e - mid;
  a21.k = kk;
  OzOperand x;
  if (c.right) {
    // B[:, mid:e] -= B[:, s:mid] A[mid:e, s:mid]^T
    x.X = c.B + s * c.ldb;
    x.ld = c.ldb;
    x.rows = c.m;
    x.k = kk;
    return oz_gemm(x, a21, kk, KRange::kFull, false, -1.0, c.B + mid * c.ldb, c.ldb, 1.0, c.S,
                   2.0 * c.m * (e - mid) * kk, c.ws, c.st);
  }
  // B[mid:e, :] -= A[mid:e, s:mid] B[s:mid, :]
  x.X = c.B + s;
  x.ld = c.ldb;
  x.rows = c.n;
  x.k = kk;
  x.by_cols = true;
  return oz_gemm(a21, x, kk, KRange::kFull, false, -1.0, c.B + mid, c.ldb, 1.0, c.S, 2.0 * c.n * (e - mid) * kk,
                 c.ws, c.st);
}

tb_status oz_trsm_rec(OzTrsm& c, long s, long e) {
  if (e - s <= c.leaf) return oz_trsm_leaf(c, (int)(s / c.leaf), s, e);
  const long nleaves = (e - s + c.leaf - 1) / c.leaf;
  const long mid = s + ((nleaves + 1) / 2) * c.leaf;
  TB_TRY(oz_trsm_rec(c, s, mid));
  TB_TRY(oz_trsm_update(c, s, mid, e));
  return oz_trsm_rec(c, mid, e);
}
}  // namespace

tb_status ozaki_trsm_impl(bool right, long m, long n, const double* A, long lda, double* B, long ldb, long nb, int S,
                          cudaStream_t st) {
  if (m < 0 || n < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  const long nt = right ? n : m;
  if (lda < (nt > 1 ? nt : 1) || ldb < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  TB_TRY(check_slices(S));
  if (m == 0 || n == 0) return TB_SUCCESS;
  OzTrsm c;
  c.right = right;
  c.m = m;
  c.n = n;
  c.nt = nt;
  c.A = A;
  c.lda = lda;
  c.B = B;
  c.ldb = ldb;
  c.S = S;
  c.st = st;
  long leaf = round_up(std::min<long>(nb, kOzLeaf), 64);
  if (leaf > kOzLeaf) leaf = kOzLeaf;
  c.leaf = (int)leaf;
  std::vector<int2> leaves;
  for (long s = 0; s < nt; s += leaf) leaves.push_back(make_int2((int)s, (int)std::min<long>(leaf, nt - s)));
  const long nleaf = (long)leaves.size();
  c.ldw = leaf;
  c.wstride = leaf * leaf;
  const long other = right ? m : n;  // extent of B across the solve
  // largest product: other x (nt - leaf) by K <= nt / 2 + leaf
  const size_t g_bytes = oz_gemm_ws(std::max<long>(other, nt), std::max<long>(other, nt), nt / 2 + leaf, S);
  const size_t w_bytes = (size_t)round_up((long long)c.wstride * nleaf * 8, 256);
  const size_t d_bytes = (size_t)round_up((nt + 31) / 32 * 1024 * 8, 256);
  const size_t l_bytes = (size_t)round_up(nleaf * (long long)sizeof(int2), 256);
  char* ws = static_cast<char*>(pool_get(w_bytes + d_bytes + l_bytes + g_bytes));
  if (!ws) {
    set_last_error("ozaki trsm: cannot allocate %zu bytes of scratch", w_bytes + d_bytes + l_bytes + g_bytes);
    return TB_ERROR_ALLOC;
  }
  c.W = reinterpret_cast<double*>(ws);
  double* D = reinterpret_cast<double*>(ws + w_bytes);
  int2* dleaves = reinterpret_cast<int2*>(ws + w_bytes + d_bytes);
  c.ws = ws + w_bytes + d_bytes + l_bytes;
  TB_CUDA_TRY(cudaMemcpyAsync(dleaves, leaves.data(), nleaf * sizeof(int2), cudaMemcpyHostToDevice, st));
  TB_TRY(trsm_leaf_inverses_f64(nt, A, lda, dleaves, (int)nleaf, (int)leaf, D, c.W, c.ldw, c.wstride, st));
  return oz_trsm_rec(c, 0, nt);
}

}  // namespace tb

// ------------------------------------------------------------------ C ABI
namespace {
bool is(char c, char u) { return c == u || c == u + ('a' - 'A'); }
// TRSM: the products' operands (leaf inverses, X) exist only during the
// solve, so a non-positive count selects 10 there; the other routines pass
// it on and choose the count from their operands.
int trsm_slices(int s) { return s <= 0 ? 10 : s; }
}  // namespace

extern "C" tb_status tb_dsyrk_ozaki(char uplo, char trans, long n, long k, double alpha, const double* A, long lda,
                                    double beta, double* C, long ldc, int slices) {
  if (!is(uplo, 'L') && !is(uplo, 'U')) return TB_ERROR_INVALID_VALUE;
  if (!is(trans, 'N') && !is(trans, 'T')) return TB_ERROR_INVALID_VALUE;
  return tb::ozaki_syrk_impl(is(trans, 'T'), n, k, alpha, A, lda, beta, C, ldc, slices, 0,
                             nullptr, 0, tb::current_stream(), is(uplo, 'U'));
}

extern "C" tb_status tb_dsyr2k_ozaki(char uplo, char trans, long n, long k, double alpha, const double* A, long lda,
                                     const double* B, long ldb, double beta, double* C, long ldc, int slices) {
  if (!is(uplo, 'L') || !is(trans, 'N')) {
    tb::set_last_error("tb_dsyr2k_ozaki: only uplo='L', trans='N' are supported");
    return TB_ERROR_NOT_SUPPORTED;
  }
  return tb::ozaki_syr2k_impl(n, k, alpha, A, lda, B, ldb, beta, C, ldc, slices,
                              tb::current_stream());
}

extern "C" tb_status tb_dtrmm_ozaki(char uplo, long m, long n, double alpha, const double* A, long lda,
                                    const double* B, long ldb, double* C, long ldc, int slices) {
  if (!is(uplo, 'L') && !is(uplo, 'U')) return TB_ERROR_INVALID_VALUE;
  return tb::ozaki_trmm_impl(is(uplo, 'U'), m, n, alpha, A, lda, B, ldb, C, ldc, slices,
                             tb::current_stream());
}

extern "C" tb_status tb_dtrsm_ozaki(char side, long m, long n, const double* A, long lda, double* B, long ldb,
                                    long nb, int slices) {
  if (!is(side, 'R') && !is(side, 'L')) return TB_ERROR_INVALID_VALUE;
  return tb::ozaki_trsm_impl(is(side, 'R'), m, n, A, lda, B, ldb, nb, trsm_slices(slices),
                             tb::current_stream());
}

extern "C" tb_status tb_ozaki_level_product(long n, long k, const double* A, long lda, int slices, int level,
                                            int* P, long ldp) {
  if (level < 2 || level > slices + 1 || ldp < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  return tb::ozaki_syrk_impl(false, n, k, 1.0, A, lda, 0.0, nullptr, n > 1 ? n : 1, slices, level, P, ldp,
                             tb::current_stream());
}

extern "C" tb_status tb_ozaki_slice(long n, long k, const double* A, long lda, int slices, signed char* Q, long ldq,
                                    int* exponents) {
  if (n < 0 || k < 0 || lda < (n > 1 ? n : 1) || ldq < tb::round_up(k, 16) || ldq % 16 != 0)
    return TB_ERROR_INVALID_VALUE;
  if (slices < 1 || slices > 14) return TB_ERROR_INVALID_VALUE;
  if (n == 0 || k == 0) return TB_SUCCESS;
  return tb::ozaki_slice(n, k, A, lda, slices, reinterpret_cast<int8_t*>(Q), ldq, tb::round_up(k, 16), exponents,
                         tb::current_stream());
}

// ------------------------------------------------------------------ reference C++ API
#include "../../include/TensorBLAS.h"

namespace {
void report(const char* fn, tb_status s) {
  if (s != TB_SUCCESS) fprintf(stderr, "TensorBLAS %s: %s %s\n", fn, tb_status_string(s), tb_last_error());
}
}  // namespace

void tc_ozimmu_syrk(cublasHandle_t, long int n, long int k, double alpha, double* A, long int lda, double beta,
                    double* C, long int ldc, long int) {
  report("tc_ozimmu_syrk",
         tb::ozaki_syrk_impl(false, n, k, alpha, A, lda, beta, C, ldc, 0, 0, nullptr, 0, tb::current_stream()));
}

void tc_ozimmu_trsm(cublasHandle_t, long int m, long int n, double* A, long int lda, double* B, long int ldb,
                    long int nb) {
  report("tc_ozimmu_trsm", tb::ozaki_trsm_impl(true, m, n, A, lda, B, ldb, nb, 10, tb::current_stream()));
}

void tc_ozimmu_trmm(cublasHandle_t, long int m, long int n, double alpha, double* A, long int lda, double* B,
                    long int ldb, double* C, long int ldc, long int) {
  report("tc_ozimmu_trmm", tb::ozaki_trmm_impl(false, m, n, alpha, A, lda, B, ldb, C, ldc, 0, tb::current_stream()));
}

void tc_ozimmu_syr2k(cublasHandle_t, long int n, long int k, double alpha, double* A, long int lda, double* B,
                     long int ldb, double beta, double* C, long int ldc, long int) {
  report("tc_ozimmu_syr2k",
         tb::ozaki_syr2k_impl(n, k, alpha, A, lda, B, ldb, beta, C, ldc, 0, tb::current_stream()));
}
