// SYRK driver (reference: BLAS/tc_syrk.cu:41-157, tc_cumpsgemm_syrk.cu).
//
// The reference converts A to FP16 once (s2h_swpipe / s2hTranspose), then
// walks its chunk plan and, per chunk, issues the recursion levels as
// strided-batched GEMMs: nb x nb diagonal blocks, then off-diagonal squares of
// size nb, 2nb, 4nb, ... plus a rectangular panel below each chunk. Together
// those GEMMs cover exactly the lower triangle of C (and the upper halves of
// the diagonal blocks). Here the same region is issued as ONE launch of the
// persistent tcgen05 engine over the list of 128 x BN tiles that meet the
// lower triangle; diagonal tiles are computed whole and masked to i >= j at
// the store, so C's strict upper triangle is never written.
#include <cstdio>

#include "tb_internal.h"

namespace tb {

namespace {
__global__ void scale_lower_kernel(long long n, float beta, float* C, long long ldc, bool upper) {
  for (long long j = blockIdx.y; j < n; j += gridDim.y) {
    const long long i0 = upper ? 0 : j, i1 = upper ? j + 1 : n;
    for (long long i = i0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < i1;
         i += (long long)gridDim.x * blockDim.x)
      C[i + j * ldc] = beta == 0.f ? 0.f : beta * C[i + j * ldc];
  }
}
}  // namespace

// C(lower) (or C(upper)) *= beta (C = 0 when beta == 0), the k == 0 /
// alpha == 0 case.
tb_status scale_lower(long long n, float beta, float* C, long long ldc, cudaStream_t st, bool upper) {
  dim3 g((unsigned)((n + 255) / 256 < 64 ? (n + 255) / 256 : 64), (unsigned)(n < 65535 ? n : 65535));
  scale_lower_kernel<<<g, 256, 0, st>>>(n, beta, C, ldc, upper);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

tb_status syrk_impl(bool trans, long n, long k, float alpha, const float* A, long lda, float beta, float* C, long ldc,
                    long nb, Split split, void* ws, size_t ws_bytes, cudaStream_t st, bool upper = false) {
  if (n < 0 || k < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  if (ldc < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  if (lda < ((trans ? k : n) > 1 ? (trans ? k : n) : 1)) return TB_ERROR_INVALID_VALUE;
  if (n == 0) return TB_SUCCESS;
  if (k == 0 || alpha == 0.f) return beta == 1.f ? TB_SUCCESS : scale_lower(n, beta, C, ldc, st, upper);
  const bool hilo = split == Split::kHiLo;
  const long long rows = trans ? k : n, cols = trans ? n : k;
  const long long ldh = round_up(rows, 64);
  const size_t one = (size_t)ldh * cols * sizeof(__half);
  const size_t need = one * (hilo ? 2 : 1);
  void* buf = (ws && ws_bytes >= need) ? ws : pool_get(need);
  if (!buf) {
    set_last_error("syrk: cannot allocate %zu bytes of scratch", need);
    return TB_ERROR_ALLOC;
  }
  __half* hi = static_cast<__half*>(buf);
  __half* lo = hilo ? reinterpret_cast<__half*>(static_cast<char*>(buf) + one) : nullptr;
  TB_TRY(convert_f32_f16(rows, cols, A, lda, hi, lo, ldh, 2048.f, 0, st));

  Operand op;
  op.ptr = hi;
  op.rows = n;
  op.cols = k;
  op.ld = ldh;
  op.mn_major = !trans;
  Operand opl = op;
  opl.ptr = lo;

  const int kb = (int)((k + kGemmBK - 1) / kGemmBK);
  const int bn = gemm_bn(split, kb);
  const std::vector<int4> plan = upper ? plan_upper((int)n, bn, 0, kb) : plan_lower((int)n, bn, 0, kb);
  GemmCall c;
  c.a_hi = c.b_hi = op;
  c.a_lo = c.b_lo = opl;
  c.split = split;
  c.kblocks = kb;
  c.C = C;
  c.ldc = ldc;
  c.M = (int)n;
  c.N = (int)n;
  c.alpha = alpha;
  c.beta = beta;
  c.tri = upper ? 2 : 1;
  c.diag = 0;
  c.flops = (double)n * (double)(n + 1) * (double)k;  // one triangle incl. diagonal, 2 flops per MAC
  return gemm_launch_plan(c, plan, st);
}

}  // namespace tb

extern "C" tb_status tb_ssyrk(char uplo, char trans, long n, long k, float alpha, const float* A, long lda,
                              float beta, float* C, long ldc, long nb, int precision) {
  if (nb == TB_NB_AUTO) return tb::auto_ssyrk(uplo, trans, n, k, alpha, A, lda, beta, C, ldc, precision);
  const bool upper = (uplo == 'U' || uplo == 'u');
  if (!upper && uplo != 'L' && uplo != 'l') return TB_ERROR_INVALID_VALUE;
  const bool t = (trans == 'T' || trans == 't' || trans == 'C' || trans == 'c');
  if (!t && trans != 'N' && trans != 'n') return TB_ERROR_INVALID_VALUE;
  if (precision == TB_PREC_FP8 && n > 0 && k > 0 && alpha != 0.f) {
    if (nb <= 0 || ldc < (n > 1 ? n : 1) || lda < ((t ? k : n) > 1 ? (t ? k : n) : 1)) return TB_ERROR_INVALID_VALUE;
    return tb::syrk_fp8(t, n, k, alpha, A, lda, beta, C, ldc, tb::current_stream(), upper);
  }
  if (precision != TB_PREC_PLAIN && precision != TB_PREC_SPLIT && precision != TB_PREC_FP8)
    return TB_ERROR_INVALID_VALUE;
  return tb::syrk_impl(t, n, k, alpha, A, lda, beta, C, ldc, nb,
                       precision == TB_PREC_SPLIT ? tb::Split::kHiLo : tb::Split::kPlain, nullptr, 0,
                       tb::current_stream(), upper);
}

// ------------------------------------------------------------------ reference C++ API
#include "../../include/TensorBLAS.h"

static void report(const char* fn, tb_status s) {
  if (s != TB_SUCCESS) fprintf(stderr, "TensorBLAS %s: %s %s\n", fn, tb_status_string(s), tb_last_error());
}

void tc_syrk(cublasHandle_t, long int n, long int k, float alpha, float* A, long int lda, float beta, float* C,
             long int ldc, __half* Ah, long int nb) {
  report("tc_syrk", tb::syrk_impl(false, n, k, alpha, A, lda, beta, C, ldc, nb, tb::Split::kPlain, Ah,
                                  Ah ? (size_t)n * (size_t)k * sizeof(__half) : 0, tb::current_stream()));
}

void tc_cumpsgemm_syrk(cumpsgemm::handle_t, long int n, long int k, float alpha, float* A, long int lda, float beta,
                       float* C, long int ldc, long int nb) {
  report("tc_cumpsgemm_syrk", tb::syrk_impl(false, n, k, alpha, A, lda, beta, C, ldc, nb, tb::Split::kHiLo, nullptr,
                                            0, tb::current_stream()));
}
