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
// FP64 C by the epilogue: C += alpha 2^(e_i+e_j-7L) P_L (one FP64 rounding per
// level). Slices are stored K-major, one int8 plane per slice, so a single
// 3-D tensor map (k, row, slice) feeds every pair.
#include <climits>
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
// e[i] = max_p frexp-exponent(a_ip) (|a_ip| < 2^e[i]); e[] pre-set very negative.
__global__ void __launch_bounds__(256) oz_rowexp_kernel(long long n, long long k, const double* __restrict__ A,
                                                        long long lda, int* __restrict__ e) {
  const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  int m = INT_MIN / 2;
  for (long long p = blockIdx.y; p < k; p += gridDim.y) {
    const double v = A[i + p * lda];
    if (v != 0.0) {
      int ex;
      frexp(v, &ex);
      m = ex > m ? ex : m;
    }
  }
  atomicMax(&e[i], m);
}

// 32 rows x 128 columns per block: FP64 tile through shared memory, then
// each thread slices 16 consecutive columns of one row and writes them as one
// 16-byte int8 vector per slice (K-major planes Q[s][i][p], row stride ldq).
__global__ void __launch_bounds__(256) oz_slice_kernel(long long n, long long k, const double* __restrict__ A,
                                                       long long lda, const int* __restrict__ e, int S,
                                                       int8_t* __restrict__ Q, long long ldq, long long plane) {
  __shared__ double tile[128][33];
  const long long r0 = (long long)blockIdx.x * 32, p0 = (long long)blockIdx.y * 128;
  const int t = threadIdx.x;
  for (int idx = t; idx < 32 * 128; idx += 256) {
    const int r = idx & 31, c = idx >> 5;
    const long long gi = r0 + r, gp = p0 + c;
    tile[c][r] = (gi < n && gp < k) ? A[gi + gp * lda] : 0.0;
  }
  __syncthreads();
  const int r = t >> 3, c0 = (t & 7) * 16;
  const long long gi = r0 + r;
  if (gi >= n) return;
  const int ex = e[gi] < -1000 ? 0 : e[gi];
  double x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = ldexp(tile[c0 + j][r], -ex);
  for (int s = 0; s < S; ++s) {
    uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const double y = x[j] * 128.0;
      const double q = trunc(y);
      x[j] = y - q;
      w[j >> 2] |= ((uint32_t)(uint8_t)(int8_t)(int)q) << (8 * (j & 3));
    }
    const long long gp = p0 + c0;
    if (gp < k) *reinterpret_cast<uint4*>(Q + s * plane + gi * ldq + gp) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// ---------------------------------------------------------------- products
struct OzArgs {
  CUtensorMap mapA;  // Q planes, box {128, 128, 1}
  CUtensorMap mapB;  // Q planes, box {128, 256, 1}
  const int4* tiles;
  int num_tiles;
  int S, KB;  // slices, K-blocks of 128
  int n;
  double* C;
  long long ldc;
  double alpha, beta;
  const int* e;
  int raw_level;  // >= 2: write P_raw_level (int32) to raw_out instead of folding into C
  int* raw_out;
  long long ld_raw;
  int* err;
};

__device__ __forceinline__ int level_pairs_begin(int L, int S) { return L - S > 1 ? L - S : 1; }
__device__ __forceinline__ int level_pairs_end(int L, int S) { return L - 1 < S ? L - 1 : S; }

__global__ void __launch_bounds__(192, 1) oz_syrk_kernel(const __grid_constant__ OzArgs args) {
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
  const int S = args.S, KB = args.KB;

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
        for (int L = 2; L <= S + 1 && ok; ++L)
          for (int s = level_pairs_begin(L, S); s <= level_pairs_end(L, S) && ok; ++s)
            for (int kb = 0; kb < KB; ++kb) {
              if (!mbar_wait(&empty[st], ph ^ 1u, abort_flag, args.err, kDevErrTimeoutProducer)) {
                ok = false;
                break;
              }
              mbar_arrive_expect_tx(&full[st], kOzStageBytes);
              uint8_t* dst = smem + st * kOzStageBytes;
              tma_load_3d(dst, &args.mapA, &full[st], kb * kOzBK, tile.x, s - 1);
              tma_load_3d(dst + kOzABytes, &args.mapB, &full[st], kb * kOzBK, tile.y, L - s - 1);
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
            for (int kb = 0; kb < KB; ++kb) {
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
    int it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
      const int4 tile = args.tiles[t];
      const long long gi = (long long)tile.x + row;
      const bool row_ok = gi < args.n;
      const int ei = row_ok ? (args.e[gi] < -1000 ? 0 : args.e[gi]) : 0;
      for (int L = 2; L <= S + 1; ++L, ++it) {
        const int buf = it & 1;
        const uint32_t tph = (uint32_t)(it >> 1) & 1u;
        if (!mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * kOzBN);
        const bool fold = args.raw_level < 2;
#pragma unroll 1
        for (int c0 = 0; c0 < kOzBN; c0 += 32) {
          int v[32];
          tmem_ld32_s32(tacc + c0, v);
          if (!row_ok) continue;
          if (!fold) {
            if (L != args.raw_level) continue;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const long long gj = (long long)tile.y + c0 + j;
              if (gj < args.n && gj <= gi) args.raw_out[gi + gj * args.ld_raw] = v[j];
            }
            continue;
          }
          double old[32];
          bool keep[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const long long gj = (long long)tile.y + c0 + j;
            keep[j] = gj < args.n && gj <= gi;
            old[j] = 0.0;
            if (keep[j] && (L > 2 || args.beta != 0.0)) old[j] = args.C[gi + gj * args.ldc];
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (!keep[j]) continue;
            const long long gj = (long long)tile.y + c0 + j;
            const int ej = args.e[gj] < -1000 ? 0 : args.e[gj];
            const double scale = args.alpha * ldexp(1.0, ei + ej - 7 * L);
            const double base = (L == 2) ? args.beta * old[j] : old[j];
            args.C[gi + gj * args.ldc] = fma(scale, (double)v[j], base);
          }
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

}  // namespace

// Slices A (n x k, column-major) into S int8 planes (K-major, row stride ldq)
// and row exponents e[n].
tb_status ozaki_slice(long long n, long long k, const double* A, long long lda, int S, int8_t* Q, long long ldq,
                      int* e, cudaStream_t st) {
  TB_CUDA_TRY(cudaMemsetAsync(e, 0x80, sizeof(int) * n, st));
  TB_CUDA_TRY(cudaMemsetAsync(Q, 0, (size_t)S * n * ldq, st));  // K padding up to ldq reads as zero
  dim3 g1((unsigned)((n + 255) / 256), (unsigned)(k < 64 ? k : 64));
  oz_rowexp_kernel<<<g1, 256, 0, st>>>(n, k, A, lda, e);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  dim3 g2((unsigned)((n + 31) / 32), (unsigned)((k + 127) / 128));
  oz_slice_kernel<<<g2, 256, 0, st>>>(n, k, A, lda, e, S, Q, ldq, ldq * n);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

tb_status ozaki_syrk_impl(long n, long k, double alpha, const double* A, long lda, double beta, double* C, long ldc,
                          int S, int raw_level, int* raw_out, long ld_raw, cudaStream_t st) {
  if (n < 0 || k < 0 || lda < (n > 1 ? n : 1) || ldc < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  if (S < 1 || S > kOzMaxSlices) {
    set_last_error("ozaki: slices must be in [1, %d]", kOzMaxSlices);
    return TB_ERROR_INVALID_VALUE;
  }
  // exactness of the INT32 level sums: (pairs per level) * k * 127^2 < 2^31
  const double bound = (double)S * (double)k * 127.0 * 127.0;
  if (bound >= 2147483647.0) {
    set_last_error("ozaki: k = %ld too large for exact INT32 accumulation with %d slices", k, S);
    return TB_ERROR_NOT_SUPPORTED;
  }
  if (n == 0 || k == 0) return TB_SUCCESS;
  const long long ldq = round_up(k, 128);
  const size_t qbytes = (size_t)S * n * ldq;
  const size_t ebytes = (size_t)round_up(n * 4, 256);
  char* ws = static_cast<char*>(pool_get(qbytes + ebytes));
  if (!ws) return TB_ERROR_ALLOC;
  int* e = reinterpret_cast<int*>(ws);
  int8_t* Q = reinterpret_cast<int8_t*>(ws + ebytes);
  TB_TRY(ozaki_slice(n, k, A, lda, S, Q, ldq, e, st));
  OzArgs a;
  memset(&a, 0, sizeof(a));
  TB_TRY(make_q_map(&a.mapA, Q, ldq, n, S, kOzBM));
  TB_TRY(make_q_map(&a.mapB, Q, ldq, n, S, kOzBN));
  const std::vector<int4> plan = plan_lower((int)n, kOzBN, 0, 1);
  a.tiles = upload_tiles(plan, st);
  if (!a.tiles) return TB_ERROR_ALLOC;
  a.num_tiles = (int)plan.size();
  a.S = S;
  a.KB = (int)(ldq / kOzBK);
  a.n = (int)n;
  a.C = C;
  a.ldc = ldc;
  a.alpha = alpha;
  a.beta = beta;
  a.e = e;
  a.raw_level = raw_level;
  a.raw_out = raw_out;
  a.ld_raw = ld_raw;
  a.err = device_error_word();
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr[dev]) {
    TB_CUDA_TRY(cudaFuncSetAttribute(oz_syrk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzSmem));
    attr[dev] = true;
  }
  const int grid = a.num_tiles < sm_count() ? a.num_tiles : sm_count();
  void* tok = prof_begin(st);
  oz_syrk_kernel<<<grid, 192, kOzSmem, st>>>(a);
  TB_CUDA_TRY(cudaGetLastError());
  prof_end(tok, st, (double)n * (double)(n + 1) * (double)k);
  note_launch();
  return TB_SUCCESS;
}

}  // namespace tb

extern "C" tb_status tb_dsyrk_ozaki(char uplo, char trans, long n, long k, double alpha, const double* A, long lda,
                                    double beta, double* C, long ldc, int slices) {
  if (uplo != 'L' && uplo != 'l') {
    tb::set_last_error("tb_dsyrk_ozaki: only uplo='L' is supported");
    return TB_ERROR_NOT_SUPPORTED;
  }
  if (trans != 'N' && trans != 'n') {
    tb::set_last_error("tb_dsyrk_ozaki: only trans='N' is supported");
    return TB_ERROR_NOT_SUPPORTED;
  }
  return tb::ozaki_syrk_impl(n, k, alpha, A, lda, beta, C, ldc, slices <= 0 ? 10 : slices, 0, nullptr, 0,
                             tb::current_stream());
}

extern "C" tb_status tb_ozaki_level_product(long n, long k, const double* A, long lda, int slices, int level,
                                            int* P, long ldp) {
  if (level < 2 || level > slices + 1 || ldp < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  return tb::ozaki_syrk_impl(n, k, 1.0, A, lda, 0.0, nullptr, n > 1 ? n : 1, slices, level, P, ldp,
                             tb::current_stream());
}

extern "C" tb_status tb_ozaki_slice(long n, long k, const double* A, long lda, int slices, signed char* Q, long ldq,
                                    int* exponents) {
  if (n < 0 || k < 0 || lda < (n > 1 ? n : 1) || ldq < tb::round_up(k, 16) || ldq % 16 != 0)
    return TB_ERROR_INVALID_VALUE;
  if (slices < 1 || slices > 14) return TB_ERROR_INVALID_VALUE;
  if (n == 0 || k == 0) return TB_SUCCESS;
  return tb::ozaki_slice(n, k, A, lda, slices, reinterpret_cast<int8_t*>(Q), ldq, exponents, tb::current_stream());
}

// ------------------------------------------------------------------ reference C++ API
#include "../../include/TensorBLAS.h"

void tc_ozimmu_syrk(cublasHandle_t, long int n, long int k, double alpha, double* A, long int lda, double beta,
                    double* C, long int ldc, long int) {
  tb_status s = tb::ozaki_syrk_impl(n, k, alpha, A, lda, beta, C, ldc, 10, 0, nullptr, 0, tb::current_stream());
  if (s != TB_SUCCESS) fprintf(stderr, "TensorBLAS tc_ozimmu_syrk: %s %s\n", tb_status_string(s), tb_last_error());
}
