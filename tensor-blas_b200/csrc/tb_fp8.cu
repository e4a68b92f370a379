// FP8-e4m3 forms of SYRK / SYR2K / TRMM / SYMM / GEMM with per-128x128-block
// scaling (TB_PREC_FP8): the lowest-precision variant of the reference's
// tc_* family, for callers whose error budget allows ~1e-2.
//
// Each operand is quantised by block: for a 128-row x 128-deep block of the
// operand (rows = output rows for A, output columns for B; K = the
// contraction index), s = max|x| / 448 (e4m3's largest finite value) and
// q = e4m3(x / s) with saturation. The tcgen05 engine multiplies e4m3 x e4m3
// into FP32 in TMEM (kind::f8f6f4), one 128-deep K block per round, and the
// epilogue folds s_A(i, kb) * s_B(j, kb) * partial into FP32 registers, so
// every block keeps its own scale.
#include <cuda_fp8.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "tb_internal.h"

namespace tb {
namespace {

constexpr int kQB = 128;  // quantisation block (rows and K)

// Where element (i, p) of an operand (row i, contraction index p) lives.
struct Q8Src {
  const float* X;
  long long ld;
  int kind;  // 0: X[i + p*ld]; 1: X[p + i*ld]; 2: symmetric lower-stored; 3: symmetric upper-stored
  int mask;  // 0: all; 1: only p <= i (lower triangular); 2: only p >= i (upper triangular)
  int unit = 0;  // 1: the diagonal (i == p) reads as 1
};

__device__ __forceinline__ float q8_load(const Q8Src& s, long long i, long long p) {
  if (s.mask == 1 && p > i) return 0.f;
  if (s.mask == 2 && p < i) return 0.f;
  if (s.unit && i == p) return 1.f;
  switch (s.kind) {
    case 0:
      return s.X[i + p * s.ld];
    case 1:
      return s.X[p + i * s.ld];
    case 2:
      return i >= p ? s.X[i + p * s.ld] : s.X[p + i * s.ld];
    default:
      return i <= p ? s.X[i + p * s.ld] : s.X[p + i * s.ld];
  }
}

// How a 128 x 128 block at (r0, p0) can be read: 0 / 1 as a plain kind-0 /
// kind-1 block (every element inside the operand and unmasked, 16-byte
// aligned rows), 2 when the mask zeroes all of it, -1 otherwise (diagonal,
// partially masked or edge blocks take the scalar path).
__device__ __forceinline__ int q8_block_kind(const Q8Src& s, long long r0, long long p0, long long rows,
                                             long long K, bool vec) {
  if (!vec || r0 + kQB > rows || p0 + kQB > K) return -1;
  if (s.mask == 1) {  // keeps p <= i
    if (p0 > r0 + kQB - 1) return 2;
    if (p0 + kQB - 1 > r0) return -1;
  } else if (s.mask == 2) {  // keeps p >= i
    if (p0 + kQB - 1 < r0) return 2;
    if (p0 < r0 + kQB - 1) return -1;
  }
  if (s.unit && r0 < p0 + kQB && p0 < r0 + kQB) return -1;
  switch (s.kind) {
    case 0:
      return 0;
    case 1:
      return 1;
    case 2:  // lower-stored: i >= p reads X[i + p ld]
      return r0 >= p0 + kQB - 1 ? 0 : (r0 + kQB - 1 < p0 ? 1 : -1);
    default:  // upper-stored: i <= p reads X[i + p ld]
      return r0 + kQB - 1 <= p0 ? 0 : (r0 > p0 + kQB - 1 ? 1 : -1);
  }
}

__device__ __forceinline__ uint32_t q8_pack4(float a, float b, float c, float d, float scale) {
  const uint32_t qa = __nv_cvt_float_to_fp8(a / scale, __NV_SATFINITE, __NV_E4M3);
  const uint32_t qb = __nv_cvt_float_to_fp8(b / scale, __NV_SATFINITE, __NV_E4M3);
  const uint32_t qc = __nv_cvt_float_to_fp8(c / scale, __NV_SATFINITE, __NV_E4M3);
  const uint32_t qd = __nv_cvt_float_to_fp8(d / scale, __NV_SATFINITE, __NV_E4M3);
  return qa | (qb << 8) | (qc << 16) | (qd << 24);
}

// Block max|x| over the CTA's 256 threads.
__device__ __forceinline__ float q8_block_max(float amax, float* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
  __syncthreads();
  float m = red[0];
#pragma unroll
  for (int w = 1; w < 8; ++w) m = fmaxf(m, red[w]);
  return m;
}

// One 128 x 128 block per CTA (256 threads): s = max|x| / 448, then the
// e4m3 block K-major (128 bytes per row; K padding to the block edge is
// written as zeros). Interior blocks hold the whole block in registers
// (sixteen 16-byte loads per thread, all in flight together); a block read
// along i is transposed through a 16 KB byte tile whose 4-byte words are
// XOR-swizzled by row so that neither its writes nor its reads conflict.
// Other blocks read element by element, twice (max, then quantise).
__global__ void __launch_bounds__(256) q8_kernel(Q8Src src, long long rows, long long K, uint8_t* __restrict__ Q,
                                                 long long ldq, long long qoff, float* __restrict__ scales,
                                                 int scale_ld, int kb_off, int vec) {
  __shared__ __align__(16) uint32_t qs[kQB * 32];  // row r: 32 words, word w at r * 32 + (w ^ ((r >> 2) & 31))
  __shared__ float red[8];
  const long long r0 = (long long)blockIdx.x * kQB, p0 = (long long)blockIdx.y * kQB;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  float* const sc = scales + (long long)blockIdx.x * scale_ld + kb_off + blockIdx.y;
  const int kind = q8_block_kind(src, r0, p0, rows, K, vec != 0);
  if (kind == 2) {
    if (t == 0) *sc = 1.f;
    for (int job = t; job < kQB * (kQB / 16); job += 256) {
      const int r = job >> 3, c = (job & 7) * 16;
      *reinterpret_cast<uint4*>(Q + (r0 + r) * ldq + qoff + p0 + c) = make_uint4(0, 0, 0, 0);
    }
    return;
  }
  if (kind < 0) {
    float amax = 0.f;
    for (int idx = t; idx < kQB * kQB; idx += 256) {
      const int r = src.kind == 1 ? (idx >> 7) : (idx & 127);
      const int p = src.kind == 1 ? (idx & 127) : (idx >> 7);
      const long long gi = r0 + r, gp = p0 + p;
      if (gi < rows && gp < K) amax = fmaxf(amax, fabsf(q8_load(src, gi, gp)));
    }
    const float m = q8_block_max(amax, red);
    const float scale = m > 0.f ? m / 448.f : 1.f;
    if (t == 0) *sc = scale;
    for (int job = t; job < kQB * (kQB / 16); job += 256) {
      const int r = job >> 3, c = (job & 7) * 16;
      const long long gi = r0 + r;
      if (gi >= rows) continue;
      float x[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) x[j] = (p0 + c + j < K) ? q8_load(src, gi, p0 + c + j) : 0.f;
      *reinterpret_cast<uint4*>(Q + gi * ldq + qoff + p0 + c) =
          make_uint4(q8_pack4(x[0], x[1], x[2], x[3], scale), q8_pack4(x[4], x[5], x[6], x[7], scale),
                     q8_pack4(x[8], x[9], x[10], x[11], scale), q8_pack4(x[12], x[13], x[14], x[15], scale));
    }
    return;
  }
  const float* X = src.X;
  const long long ld = src.ld;
  float4 v[16];
  if (kind == 1) {
    // row r = w + 8 i, p = 4 lane .. 4 lane + 3
#pragma unroll
    for (int i = 0; i < 16; ++i)
      v[i] = __ldg(reinterpret_cast<const float4*>(X + (p0 + 4 * lane) + (r0 + w + 8 * i) * ld));
  } else {
    // p = 4 (w + 8 jj) + u, r = 4 lane .. 4 lane + 3
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
#pragma unroll
      for (int u = 0; u < 4; ++u)
        v[jj * 4 + u] =
            __ldg(reinterpret_cast<const float4*>(X + (r0 + 4 * lane) + (p0 + 4 * (w + 8 * jj) + u) * ld));
  }
  float amax = 0.f;
#pragma unroll
  for (int i = 0; i < 16; ++i)
    amax = fmaxf(fmaxf(amax, fmaxf(fabsf(v[i].x), fabsf(v[i].y))), fmaxf(fabsf(v[i].z), fabsf(v[i].w)));
  const float m = q8_block_max(amax, red);
  const float scale = m > 0.f ? m / 448.f : 1.f;
  if (t == 0) *sc = scale;
  if (kind == 1) {
#pragma unroll
    for (int i = 0; i < 16; ++i)
      *reinterpret_cast<uint32_t*>(Q + (r0 + w + 8 * i) * ldq + qoff + p0 + 4 * lane) =
          q8_pack4(v[i].x, v[i].y, v[i].z, v[i].w, scale);
    return;
  }
  // rows r = 4 lane + j; word s = w + 8 jj holds p = 4 s .. 4 s + 3
#pragma unroll
  for (int jj = 0; jj < 4; ++jj) {
    const int s = w + 8 * jj;
    const float4 a = v[jj * 4 + 0], b = v[jj * 4 + 1], c = v[jj * 4 + 2], d = v[jj * 4 + 3];
    qs[(4 * lane + 0) * 32 + (s ^ lane)] = q8_pack4(a.x, b.x, c.x, d.x, scale);
    qs[(4 * lane + 1) * 32 + (s ^ lane)] = q8_pack4(a.y, b.y, c.y, d.y, scale);
    qs[(4 * lane + 2) * 32 + (s ^ lane)] = q8_pack4(a.z, b.z, c.z, d.z, scale);
    qs[(4 * lane + 3) * 32 + (s ^ lane)] = q8_pack4(a.w, b.w, c.w, d.w, scale);
  }
  __syncthreads();
  // 16-byte pieces: lanes (c = lane & 7, g = lane >> 3) of warp-iteration
  // wi = 8 it + w take row r = 16 (wi >> 2) + 4 g + (wi & 3), bytes 16 c ..
#pragma unroll
  for (int it = 0; it < 4; ++it) {
    const int wi = 8 * it + w, c = lane & 7, g = lane >> 3;
    const int r = 16 * (wi >> 2) + 4 * g + (wi & 3);
    const int sw = (r >> 2) & 31;
    const uint32_t* row = qs + r * 32;
    *reinterpret_cast<uint4*>(Q + (r0 + r) * ldq + qoff + p0 + 16 * c) =
        make_uint4(row[(4 * c + 0) ^ sw], row[(4 * c + 1) ^ sw], row[(4 * c + 2) ^ sw], row[(4 * c + 3) ^ sw]);
  }
}

tb_status quantize(const Q8Src& src, long long rows, long long K, uint8_t* Q, long long ldq, long long qoff,
                   float* scales, int scale_ld, int kb_off, cudaStream_t st) {
  if (rows == 0 || K == 0) return TB_SUCCESS;
  const int vec = (reinterpret_cast<uintptr_t>(src.X) % 16 == 0 && src.ld % 4 == 0) ? 1 : 0;
  dim3 g((unsigned)((rows + kQB - 1) / kQB), (unsigned)((K + kQB - 1) / kQB));
  q8_kernel<<<g, 256, 0, st>>>(src, rows, K, Q, ldq, qoff, scales, scale_ld, kb_off, vec);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

// Quantised operand storage: rows x ldq bytes + scales [rows/128][scale_ld].
struct Q8Op {
  uint8_t* Q = nullptr;
  float* s = nullptr;
  long long rows = 0, ldq = 0;
  int scale_ld = 0;
};

size_t q8_bytes(long long rows, long long ldq) {
  return (size_t)round_up(rows * ldq, 256) + (size_t)round_up(((rows + kQB - 1) / kQB) * (ldq / kQB) * 4, 256);
}

Q8Op q8_carve(char*& ws, long long rows, long long ldq) {
  Q8Op o;
  o.rows = rows;
  o.ldq = ldq;
  o.scale_ld = (int)(ldq / kQB);
  o.Q = reinterpret_cast<uint8_t*>(ws);
  ws += round_up(rows * ldq, 256);
  o.s = reinterpret_cast<float*>(ws);
  ws += round_up(((rows + kQB - 1) / kQB) * (ldq / kQB) * 4, 256);
  return o;
}

tb_status q8_gemm(const Q8Op& a, const Q8Op& b, std::vector<int4>& plan, int M, int N, int tri, float alpha,
                  float beta, float* C, long long ldc, double flops, cudaStream_t st) {
  GemmCall c;
  c.fp8 = true;
  c.a_hi = {a.Q, a.rows, a.ldq, a.ldq, false};
  c.b_hi = {b.Q, b.rows, b.ldq, b.ldq, false};
  c.scale_a = a.s;
  c.scale_b = b.s;
  c.scale_ld = a.scale_ld;
  c.C = C;
  c.ldc = ldc;
  c.M = M;
  c.N = N;
  c.alpha = alpha;
  c.beta = beta;
  c.tri = tri;
  c.flops = flops;
  c.tiles = upload_tiles(plan, st);
  if (!c.tiles) return TB_ERROR_ALLOC;
  c.num_tiles = (int)plan.size();
  return gemm_launch(c, st);
}

char* q8_scratch(size_t bytes) {
  char* ws = static_cast<char*>(pool_get(bytes));
  if (!ws) set_last_error("fp8: cannot allocate %zu bytes of scratch", bytes);
  return ws;
}

}  // namespace

// C(lower) = alpha op(A) op(A)^T + beta C.
tb_status syrk_fp8(bool trans, long n, long k, float alpha, const float* A, long lda, float beta, float* C, long ldc,
                   cudaStream_t st, bool upper) {
  const long long ldq = round_up(k > 0 ? k : 1, kQB);
  char* ws = q8_scratch(q8_bytes(n, ldq));
  if (!ws) return TB_ERROR_ALLOC;
  Q8Op a = q8_carve(ws, n, ldq);
  TB_TRY(quantize({A, lda, trans ? 1 : 0, 0}, n, k, a.Q, ldq, 0, a.s, a.scale_ld, 0, st));
  std::vector<int4> plan = upper ? plan_upper((int)n, kGemmBNFp8, 0, (int)(ldq / kQB))
                                 : plan_lower((int)n, kGemmBNFp8, 0, (int)(ldq / kQB));
  return q8_gemm(a, a, plan, (int)n, (int)n, upper ? 2 : 1, alpha, beta, C, ldc, (double)n * (n + 1) * (double)k, st);
}

// C(lower) = alpha (A B^T + B A^T) + beta C, A and B n x k: [A | B] times [B | A]^T.
tb_status syr2k_fp8(long n, long k, float alpha, const float* A, long lda, const float* B, long ldb, float beta,
                    float* C, long ldc, cudaStream_t st) {
  const long long kh = round_up(k > 0 ? k : 1, kQB), ldq = 2 * kh;
  char* ws = q8_scratch(2 * q8_bytes(n, ldq));
  if (!ws) return TB_ERROR_ALLOC;
  Q8Op ab = q8_carve(ws, n, ldq), ba = q8_carve(ws, n, ldq);
  const int kbh = (int)(kh / kQB);
  TB_TRY(quantize({A, lda, 0, 0}, n, k, ab.Q, ldq, 0, ab.s, ab.scale_ld, 0, st));
  TB_TRY(quantize({B, ldb, 0, 0}, n, k, ab.Q, ldq, kh, ab.s, ab.scale_ld, kbh, st));
  TB_TRY(quantize({B, ldb, 0, 0}, n, k, ba.Q, ldq, 0, ba.s, ba.scale_ld, 0, st));
  TB_TRY(quantize({A, lda, 0, 0}, n, k, ba.Q, ldq, kh, ba.s, ba.scale_ld, kbh, st));
  std::vector<int4> plan = plan_lower((int)n, kGemmBNFp8, 0, 2 * kbh);
  return q8_gemm(ab, ba, plan, (int)n, (int)n, 1, alpha, beta, C, ldc, 2.0 * n * (n + 1) * (double)k, st);
}

// General TRMM (see trmm_ex_impl): C = alpha op(A) B (left) or alpha B op(A)
// (right), A triangular (other triangle unread), unit or stored diagonal.
tb_status trmm_fp8(bool right, bool upper, bool trans, bool unit, long m, long n, float alpha, const float* A,
                   long lda, const float* B, long ldb, float* C, long ldc, cudaStream_t st) {
  const long na = right ? n : m;
  const long long ldq = round_up(na, kQB);
  char* ws = q8_scratch(q8_bytes(m, ldq) + q8_bytes(n, ldq));
  if (!ws) return TB_ERROR_ALLOC;
  Q8Op a = q8_carve(ws, m, ldq), b = q8_carve(ws, n, ldq);
  const bool op_lower = upper == trans;
  const int u = unit ? 1 : 0;
  if (!right) {
    // rows i of op(A) (A by rows, or A^T = A by columns); B by columns
    TB_TRY(quantize({A, lda, trans ? 1 : 0, op_lower ? 1 : 2, u}, m, m, a.Q, ldq, 0, a.s, a.scale_ld, 0, st));
    TB_TRY(quantize({B, ldb, 1, 0, 0}, n, m, b.Q, ldq, 0, b.s, b.scale_ld, 0, st));
  } else {
    // rows i of B; rows j of op(A)^T: op(A)(p, j) = A[p + j lda] or A[j + p lda]
    TB_TRY(quantize({B, ldb, 0, 0, 0}, m, n, a.Q, ldq, 0, a.s, a.scale_ld, 0, st));
    TB_TRY(quantize({A, lda, trans ? 0 : 1, op_lower ? 2 : 1, u}, n, n, b.Q, ldq, 0, b.s, b.scale_ld, 0, st));
  }
  const int kb = (int)(ldq / kQB);
  std::vector<int4> plan = plan_rect((int)m, (int)n, kGemmBNFp8, 0, kb);
  for (int4& t : plan) {
    const long long o = right ? t.y : t.x;  // the tile's offset along A's order
    if (right != op_lower)
      t.w = (int)((std::min<long long>(o + kQB, na) + kQB - 1) / kQB);  // entries only up to the diagonal
    else
      t.z = (int)(o / kQB);  // entries only from the diagonal on
  }
  return q8_gemm(a, b, plan, (int)m, (int)n, 0, alpha, 0.f, C, ldc, (double)m * n * na, st);
}

// C = alpha A B + beta C, A m x m symmetric with triangle `lower` stored.
tb_status symm_fp8(bool lower, long m, long n, float alpha, const float* A, long lda, const float* B, long ldb,
                   float beta, float* C, long ldc, cudaStream_t st) {
  const long long ldq = round_up(m, kQB);
  char* ws = q8_scratch(q8_bytes(m, ldq) + q8_bytes(n, ldq));
  if (!ws) return TB_ERROR_ALLOC;
  Q8Op a = q8_carve(ws, m, ldq), b = q8_carve(ws, n, ldq);
  TB_TRY(quantize({A, lda, lower ? 2 : 3, 0}, m, m, a.Q, ldq, 0, a.s, a.scale_ld, 0, st));
  TB_TRY(quantize({B, ldb, 1, 0}, n, m, b.Q, ldq, 0, b.s, b.scale_ld, 0, st));
  std::vector<int4> plan = plan_rect((int)m, (int)n, kGemmBNFp8, 0, (int)(ldq / kQB));
  return q8_gemm(a, b, plan, (int)m, (int)n, 0, alpha, beta, C, ldc, 2.0 * m * m * (double)n, st);
}

// C = alpha op(A) op(B) + beta C.
tb_status gemm_fp8(bool ta, bool tb_, long m, long n, long k, float alpha, const float* A, long lda, const float* B,
                   long ldb, float beta, float* C, long ldc, cudaStream_t st) {
  const long long ldq = round_up(k > 0 ? k : 1, kQB);
  char* ws = q8_scratch(q8_bytes(m, ldq) + q8_bytes(n, ldq));
  if (!ws) return TB_ERROR_ALLOC;
  Q8Op a = q8_carve(ws, m, ldq), b = q8_carve(ws, n, ldq);
  // op(A)(i, p): A[i + p lda] ('N') or A[p + i lda] ('T'); op(B)^T rows j: B[p + j ldb] ('N') or B[j + p ldb] ('T')
  TB_TRY(quantize({A, lda, ta ? 1 : 0, 0}, m, k, a.Q, ldq, 0, a.s, a.scale_ld, 0, st));
  TB_TRY(quantize({B, ldb, tb_ ? 0 : 1, 0}, n, k, b.Q, ldq, 0, b.s, b.scale_ld, 0, st));
  std::vector<int4> plan = plan_rect((int)m, (int)n, kGemmBNFp8, 0, (int)(ldq / kQB));
  return q8_gemm(a, b, plan, (int)m, (int)n, 0, alpha, beta, C, ldc, 2.0 * m * n * (double)k, st);
}

}  // namespace tb
