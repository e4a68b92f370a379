// General FP32-in/FP32-out GEMM through the tensor-core engine, the
// library's equivalent of the cublasGemmEx(FP16 in, FP32 out) calls every
// reference routine is built from (e.g. BLAS/tc_syrk.cu:106-118) and of the
// reference's testing/testing_gemm.cu benchmark.
#include "tb_internal.h"

namespace tb {

tb_status gemm_impl(bool ta, bool tb_, long m, long n, long k, float alpha, const float* A, long lda, const float* B,
                    long ldb, float beta, float* C, long ldc, Split split, cudaStream_t st) {
  if (m < 0 || n < 0 || k < 0) return TB_ERROR_INVALID_VALUE;
  if (lda < ((ta ? k : m) > 1 ? (ta ? k : m) : 1)) return TB_ERROR_INVALID_VALUE;
  if (ldb < ((tb_ ? n : k) > 1 ? (tb_ ? n : k) : 1)) return TB_ERROR_INVALID_VALUE;
  if (ldc < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  if (k == 0) return TB_ERROR_NOT_SUPPORTED;
  const bool hilo = split == Split::kHiLo;
  // Stored shapes of A and B (column-major): A is (ta ? k x m : m x k).
  const long long ar = ta ? k : m, ac = ta ? m : k;
  const long long br = tb_ ? n : k, bc = tb_ ? k : n;
  const long long lda_h = round_up(ar, 64), ldb_h = round_up(br, 64);
  const size_t abytes = (size_t)lda_h * ac * 2, bbytes = (size_t)ldb_h * bc * 2;
  const size_t need = (abytes + bbytes) * (hilo ? 2 : 1);
  char* buf = static_cast<char*>(pool_get(need));
  if (!buf) return TB_ERROR_ALLOC;
  __half* ah = reinterpret_cast<__half*>(buf);
  __half* bh = reinterpret_cast<__half*>(buf + abytes);
  __half* al = hilo ? reinterpret_cast<__half*>(buf + abytes + bbytes) : nullptr;
  __half* bl = hilo ? reinterpret_cast<__half*>(buf + 2 * abytes + bbytes) : nullptr;
  TB_TRY(convert_f32_f16(ar, ac, A, lda, ah, al, lda_h, 2048.f, 0, st));
  TB_TRY(convert_f32_f16(br, bc, B, ldb, bh, bl, ldb_h, 2048.f, 0, st));

  GemmCall c;
  c.split = split;
  c.a_hi.ptr = ah;
  c.a_hi.rows = m;
  c.a_hi.cols = k;
  c.a_hi.ld = lda_h;
  c.a_hi.mn_major = !ta;
  c.a_lo = c.a_hi;
  c.a_lo.ptr = al;
  c.b_hi.ptr = bh;
  c.b_hi.rows = n;
  c.b_hi.cols = k;
  c.b_hi.ld = ldb_h;
  c.b_hi.mn_major = tb_;
  c.b_lo = c.b_hi;
  c.b_lo.ptr = bl;
  c.kblocks = (int)((k + kGemmBK - 1) / kGemmBK);
  const std::vector<int4> plan = plan_rect((int)m, (int)n, gemm_bn(split, c.kblocks), 0, c.kblocks);
  c.C = C;
  c.ldc = ldc;
  c.M = (int)m;
  c.N = (int)n;
  c.alpha = alpha;
  c.beta = beta;
  c.flops = 2.0 * m * n * k;
  return gemm_launch_plan(c, plan, st);
}

}  // namespace tb

static bool parse_trans(char t, bool* out) {
  if (t == 'N' || t == 'n') {
    *out = false;
    return true;
  }
  if (t == 'T' || t == 't' || t == 'C' || t == 'c') {
    *out = true;
    return true;
  }
  return false;
}

extern "C" tb_status tb_sgemm(char transa, char transb, long m, long n, long k, float alpha, const float* A, long lda,
                              const float* B, long ldb, float beta, float* C, long ldc, int precision) {
  bool ta, tbb;
  if (!parse_trans(transa, &ta) || !parse_trans(transb, &tbb)) return TB_ERROR_INVALID_VALUE;
  if (precision == TB_PREC_FP8 && m > 0 && n > 0 && k > 0 && alpha != 0.f) {
    if (lda < ((ta ? k : m) > 1 ? (ta ? k : m) : 1) || ldb < ((tbb ? n : k) > 1 ? (tbb ? n : k) : 1) ||
        ldc < (m > 1 ? m : 1))
      return TB_ERROR_INVALID_VALUE;
    return tb::gemm_fp8(ta, tbb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tb::current_stream());
  }
  if (precision != TB_PREC_PLAIN && precision != TB_PREC_SPLIT && precision != TB_PREC_FP8)
    return TB_ERROR_INVALID_VALUE;
  return tb::gemm_impl(ta, tbb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                       precision == TB_PREC_SPLIT ? tb::Split::kHiLo : tb::Split::kPlain, tb::current_stream());
}
