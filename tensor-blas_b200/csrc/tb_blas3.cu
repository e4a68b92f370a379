// SYR2K, TRMM and SYMM on the tensor-core engine (reference:
// BLAS/tc_syr2k.cu:3-152, BLAS/tc_trmm.cu:4-135, BLAS/tc_symm.cu:3-19 and
// their tc_cumpsgemm_* twins).
//
//  * SYR2K: the reference issues A*B^T and B*A^T as two GEMMs per recursion
//    block (BLAS/tc_syr2k.cu:6-33). Here one FP16 buffer holds the column
//    blocks [A | B | A]; the A operand reads columns [0, 2k) and the B
//    operand columns [k, 3k), so a single K = 2k product over the
//    lower-triangle tile list gives A B^T + B A^T in one accumulator.
//  * TRMM: C = alpha * op(A) * B with A triangular. The reference multiplies
//    full diagonal blocks and therefore needs a zeroed opposite triangle
//    (testing/testing_trmm.cu:51); here the FP16 copy of A is masked during
//    conversion and every output tile runs only the K-blocks its triangle
//    touches (lower: k < m0 + 128; upper: k >= m0).
//  * SYMM: the reference mirrors the caller's A in place before a full GEMM
//    (BLAS/tc_symm.cu:7); here the symmetric FP16 copy is built by a tiled
//    conversion kernel and the caller's A is never written.
#include <cstdio>

#include "tb_internal.h"

namespace tb {

namespace {

void* scratch(void* ws, size_t ws_bytes, size_t need) {
  return (ws && ws_bytes >= need) ? ws : pool_get(need);
}

tb_status run(GemmCall& c, const std::vector<int4>& plan, cudaStream_t st) { return gemm_launch_plan(c, plan, st); }

}  // namespace

tb_status syr2k_impl(long n, long k, float alpha, const float* A, long lda, const float* B, long ldb, float beta,
                     float* C, long ldc, long nb, Split split, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (n < 0 || k < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  if (lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1) || ldc < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  if (n == 0) return TB_SUCCESS;
  if (k == 0 || alpha == 0.f) return beta == 1.f ? TB_SUCCESS : scale_lower(n, beta, C, ldc, st);
  const bool hilo = split == Split::kHiLo;
  const long long ldh = round_up(n, 64);
  const size_t one = (size_t)ldh * 3 * k * sizeof(__half);
  char* buf = static_cast<char*>(scratch(ws, ws_bytes, one * (hilo ? 2 : 1)));
  if (!buf) return TB_ERROR_ALLOC;
  __half* hi = reinterpret_cast<__half*>(buf);
  __half* lo = hilo ? reinterpret_cast<__half*>(buf + one) : nullptr;
  const long long blk = ldh * k;  // elements per column block
  // column blocks [A | B | A]: the A-operand is [A | B], the B-operand [B | A];
  // A is read once for both of its copies
  TB_TRY(convert_f32_f16(n, k, A, lda, hi, lo, ldh, 2048.f, 0, st, 2 * blk));
  TB_TRY(convert_f32_f16(n, k, B, ldb, hi + blk, lo ? lo + blk : nullptr, ldh, 2048.f, 0, st));
  GemmCall c;
  c.split = split;
  c.a_hi = {hi, n, 2 * k, ldh, true};
  c.a_lo = {lo, n, 2 * k, ldh, true};
  c.b_hi = {hi + blk, n, 2 * k, ldh, true};
  c.b_lo = {lo ? lo + blk : nullptr, n, 2 * k, ldh, true};
  c.C = C;
  c.ldc = ldc;
  c.M = c.N = (int)n;
  c.alpha = alpha;
  c.beta = beta;
  c.tri = 1;
  c.flops = 2.0 * (double)n * (double)(n + 1) * (double)k;
  c.kblocks = (int)((2 * k + kGemmBK - 1) / kGemmBK);
  return run(c, plan_lower((int)n, gemm_bn(split, c.kblocks), 0, c.kblocks), st);
}

// General TRMM, out of place: C = alpha op(A) B (left, A m x m) or
// C = alpha B op(A) (right, A n x n); op(A) = A or A^T, A lower or upper
// triangular (the other triangle is never read), unit or stored diagonal.
// The triangle becomes a per-tile K range; op(A) is read from one FP16 copy
// of A in whichever orientation the product needs.
tb_status trmm_ex_impl(bool right, bool upper, bool trans, bool unit, long m, long n, float alpha, const float* A,
                       long lda, const float* B, long ldb, float* C, long ldc, Split split, void* ws, size_t ws_bytes,
                       cudaStream_t st, float beta) {
  const long na = right ? n : m;  // order of A
  if (m < 0 || n < 0) return TB_ERROR_INVALID_VALUE;
  if (lda < (na > 1 ? na : 1) || ldb < (m > 1 ? m : 1) || ldc < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  const bool hilo = split == Split::kHiLo;
  const long long lda_h = round_up(na, 64), ldb_h = round_up(m, 64);
  const size_t abytes = (size_t)round_up(lda_h * na * 2, 256), bbytes = (size_t)round_up(ldb_h * n * 2, 256);
  const size_t need = (abytes + bbytes) * (hilo ? 2 : 1);
  char* buf = static_cast<char*>(scratch(ws, ws_bytes, need));
  if (!buf) return TB_ERROR_ALLOC;
  __half* ah = reinterpret_cast<__half*>(buf);
  __half* bh = reinterpret_cast<__half*>(buf + abytes);
  __half* al = hilo ? reinterpret_cast<__half*>(buf + abytes + bbytes) : nullptr;
  __half* bl = hilo ? reinterpret_cast<__half*>(buf + 2 * abytes + bbytes) : nullptr;
  // left, op(A) = A: the tiles read A's triangle plus a band next to the
  // diagonal only, so only that is converted
  const int tri = (!right && !trans) ? (upper ? 4 : 5) : (upper ? 3 : 1);
  TB_TRY(convert_f32_f16(na, na, A, lda, ah, al, lda_h, 2048.f, tri, st));
  if (unit) TB_TRY(set_unit_diag(na, ah, al, lda_h, st));
  TB_TRY(convert_f32_f16(m, n, B, ldb, bh, bl, ldb_h, 2048.f, 0, st));
  const bool op_lower = upper == trans;  // op(A) lower triangular
  GemmCall c;
  c.split = split;
  if (!right) {
    // C(i, j) = sum_p op(A)(i, p) B(p, j): op(A) rows from the copy (MN-major
    // for A, K-major for A^T); B as K-major rows j
    c.a_hi = {ah, m, m, lda_h, !trans};
    c.a_lo = {al, m, m, lda_h, !trans};
    c.b_hi = {bh, n, m, ldb_h, false};
    c.b_lo = {bl, n, m, ldb_h, false};
  } else {
    // C(i, j) = sum_p B(i, p) op(A)(p, j): B MN-major; op(A)^T rows j (K-major
    // for A, MN-major for A^T)
    c.a_hi = {bh, m, n, ldb_h, true};
    c.a_lo = {bl, m, n, ldb_h, true};
    c.b_hi = {ah, n, n, lda_h, trans};
    c.b_lo = {al, n, n, lda_h, trans};
  }
  c.C = C;
  c.ldc = ldc;
  c.M = (int)m;
  c.N = (int)n;
  c.alpha = alpha;
  c.beta = beta;
  c.flops = (double)m * n * na;
  const int kb = (int)((na + kGemmBK - 1) / kGemmBK);
  c.kblocks = kb;
  const int bn = gemm_bn(split, kb);
  std::vector<int4> plan = plan_rect((int)m, (int)n, bn, 0, kb);
  for (int4& t : plan) {
    if (!right) {
      if (op_lower) {
        const long lim = (long)t.x + kGemmBM < na ? (long)t.x + kGemmBM : na;
        t.w = (int)((lim + kGemmBK - 1) / kGemmBK);  // op(A)(i, p) = 0 for p > i
      } else {
        t.z = t.x / kGemmBK;  // op(A)(i, p) = 0 for p < i
      }
    } else {
      if (op_lower) {
        t.z = t.y / kGemmBK;  // op(A)(p, j) = 0 for p < j
      } else {
        const long lim = (long)t.y + bn < na ? (long)t.y + bn : na;
        t.w = (int)((lim + kGemmBK - 1) / kGemmBK);  // op(A)(p, j) = 0 for p > j
      }
    }
  }
  return run(c, plan, st);
}

tb_status trmm_impl(bool upper, long m, long n, float alpha, const float* A, long lda, const float* B, long ldb,
                    float* C, long ldc, long nb, Split split, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (nb <= 0) return TB_ERROR_INVALID_VALUE;
  return trmm_ex_impl(false, upper, false, false, m, n, alpha, A, lda, B, ldb, C, ldc, split, ws, ws_bytes, st);
}

tb_status symm_impl(bool lower, long m, long n, float alpha, const float* A, long lda, const float* B, long ldb,
                    float beta, float* C, long ldc, Split split, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (m < 0 || n < 0) return TB_ERROR_INVALID_VALUE;
  if (lda < (m > 1 ? m : 1) || ldb < (m > 1 ? m : 1) || ldc < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  const bool hilo = split == Split::kHiLo;
  const long long ldh = round_up(m, 64);
  const size_t abytes = (size_t)ldh * m * 2, bbytes = (size_t)ldh * n * 2;
  const size_t need = (abytes + bbytes) * (hilo ? 2 : 1);
  char* buf = static_cast<char*>(scratch(ws, ws_bytes, need));
  if (!buf) return TB_ERROR_ALLOC;
  __half* ah = reinterpret_cast<__half*>(buf);
  __half* bh = reinterpret_cast<__half*>(buf + abytes);
  __half* al = hilo ? reinterpret_cast<__half*>(buf + abytes + bbytes) : nullptr;
  __half* bl = hilo ? reinterpret_cast<__half*>(buf + 2 * abytes + bbytes) : nullptr;
  TB_TRY(convert_sym_f32_f16(m, A, lda, lower, ah, al, ldh, 2048.f, st));
  TB_TRY(convert_f32_f16(m, n, B, ldb, bh, bl, ldh, 2048.f, 0, st));
  GemmCall c;
  c.split = split;
  c.a_hi = {ah, m, m, ldh, true};
  c.a_lo = {al, m, m, ldh, true};
  c.b_hi = {bh, n, m, ldh, false};
  c.b_lo = {bl, n, m, ldh, false};
  c.C = C;
  c.ldc = ldc;
  c.M = (int)m;
  c.N = (int)n;
  c.alpha = alpha;
  c.beta = beta;
  c.flops = 2.0 * (double)m * m * n;
  c.kblocks = (int)((m + kGemmBK - 1) / kGemmBK);
  return run(c, plan_rect((int)m, (int)n, gemm_bn(split, c.kblocks), 0, c.kblocks), st);
}

}  // namespace tb

// ------------------------------------------------------------------ C ABI
static bool prec_ok(int p) { return p == TB_PREC_PLAIN || p == TB_PREC_SPLIT; }
static tb::Split to_split(int p) { return p == TB_PREC_SPLIT ? tb::Split::kHiLo : tb::Split::kPlain; }

extern "C" tb_status tb_ssyr2k(char uplo, char trans, long n, long k, float alpha, const float* A, long lda,
                               const float* B, long ldb, float beta, float* C, long ldc, long nb, int precision) {
  if (nb == TB_NB_AUTO) return tb::auto_ssyr2k(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C, ldc, precision);
  if (uplo != 'L' && uplo != 'l') {
    tb::set_last_error("tb_ssyr2k: only uplo='L' is supported");
    return TB_ERROR_NOT_SUPPORTED;
  }
  if (trans != 'N' && trans != 'n') {
    tb::set_last_error("tb_ssyr2k: only trans='N' is supported");
    return TB_ERROR_NOT_SUPPORTED;
  }
  if (precision == TB_PREC_FP8) {
    if (n < 0 || k < 0 || nb <= 0 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1) || ldc < (n > 1 ? n : 1))
      return TB_ERROR_INVALID_VALUE;
    if (n == 0) return TB_SUCCESS;
    if (k > 0 && alpha != 0.f) return tb::syr2k_fp8(n, k, alpha, A, lda, B, ldb, beta, C, ldc, tb::current_stream());
    precision = TB_PREC_PLAIN;  // k == 0 / alpha == 0: C = beta C, no products
  }
  if (!prec_ok(precision)) return TB_ERROR_INVALID_VALUE;
  return tb::syr2k_impl(n, k, alpha, A, lda, B, ldb, beta, C, ldc, nb, to_split(precision), nullptr, 0,
                        tb::current_stream());
}

extern "C" tb_status tb_strmm(char uplo, long m, long n, float alpha, const float* A, long lda, const float* B,
                              long ldb, float* C, long ldc, long nb, int precision) {
  if (nb == TB_NB_AUTO) return tb::auto_strmm(uplo, m, n, alpha, A, lda, B, ldb, C, ldc, precision);
  bool upper;
  if (uplo == 'L' || uplo == 'l')
    upper = false;
  else if (uplo == 'U' || uplo == 'u')
    upper = true;
  else
    return TB_ERROR_INVALID_VALUE;
  if (precision == TB_PREC_FP8) {
    if (m < 0 || n < 0 || nb <= 0 || lda < (m > 1 ? m : 1) || ldb < (m > 1 ? m : 1) || ldc < (m > 1 ? m : 1))
      return TB_ERROR_INVALID_VALUE;
    if (m == 0 || n == 0) return TB_SUCCESS;
    return tb::trmm_fp8(false, upper, false, false, m, n, alpha, A, lda, B, ldb, C, ldc, tb::current_stream());
  }
  if (!prec_ok(precision)) return TB_ERROR_INVALID_VALUE;
  return tb::trmm_impl(upper, m, n, alpha, A, lda, B, ldb, C, ldc, nb, to_split(precision), nullptr, 0,
                       tb::current_stream());
}

extern "C" tb_status tb_strmm_ex(char side, char uplo, char transa, char diag, long m, long n, float alpha,
                                 const float* A, long lda, const float* B, long ldb, float* C, long ldc, int precision) {
  auto flag = [](char c, char a, char b, bool* v) {
    if (c == a || c == a + ('a' - 'A')) {
      *v = false;
      return true;
    }
    if (c == b || c == b + ('a' - 'A')) {
      *v = true;
      return true;
    }
    return false;
  };
  bool right, upper, trans, unit;
  if (!flag(side, 'L', 'R', &right) || !flag(uplo, 'L', 'U', &upper) || !flag(diag, 'N', 'U', &unit))
    return TB_ERROR_INVALID_VALUE;
  if (!flag(transa, 'N', 'T', &trans) && !flag(transa, 'N', 'C', &trans)) return TB_ERROR_INVALID_VALUE;
  if (precision == TB_PREC_FP8) {
    const long na = right ? n : m;
    if (m < 0 || n < 0 || lda < (na > 1 ? na : 1) || ldb < (m > 1 ? m : 1) || ldc < (m > 1 ? m : 1))
      return TB_ERROR_INVALID_VALUE;
    if (m == 0 || n == 0) return TB_SUCCESS;
    return tb::trmm_fp8(right, upper, trans, unit, m, n, alpha, A, lda, B, ldb, C, ldc, tb::current_stream());
  }
  if (!prec_ok(precision)) return TB_ERROR_INVALID_VALUE;
  return tb::trmm_ex_impl(right, upper, trans, unit, m, n, alpha, A, lda, B, ldb, C, ldc, to_split(precision),
                          nullptr, 0, tb::current_stream());
}

extern "C" tb_status tb_ssymm(char uplo, long m, long n, float alpha, const float* A, long lda, const float* B,
                              long ldb, float beta, float* C, long ldc, int precision) {
  bool lower;
  if (uplo == 'L' || uplo == 'l')
    lower = true;
  else if (uplo == 'U' || uplo == 'u')
    lower = false;
  else
    return TB_ERROR_INVALID_VALUE;
  if (precision == TB_PREC_FP8) {
    if (m < 0 || n < 0 || lda < (m > 1 ? m : 1) || ldb < (m > 1 ? m : 1) || ldc < (m > 1 ? m : 1))
      return TB_ERROR_INVALID_VALUE;
    if (m == 0 || n == 0) return TB_SUCCESS;
    return tb::symm_fp8(lower, m, n, alpha, A, lda, B, ldb, beta, C, ldc, tb::current_stream());
  }
  if (!prec_ok(precision)) return TB_ERROR_INVALID_VALUE;
  return tb::symm_impl(lower, m, n, alpha, A, lda, B, ldb, beta, C, ldc, to_split(precision), nullptr, 0,
                       tb::current_stream());
}

// ------------------------------------------------------------------ reference C++ API
#include "../../include/TensorBLAS.h"

static void report(const char* fn, tb_status s) {
  if (s != TB_SUCCESS) fprintf(stderr, "TensorBLAS %s: %s %s\n", fn, tb_status_string(s), tb_last_error());
}

void tc_syr2k(cublasHandle_t, long int n, long int k, float alpha, float* A, long int lda, float* B, long int ldb,
              float beta, float* C, long int ldc, __half* Ah, long int nb) {
  report("tc_syr2k", tb::syr2k_impl(n, k, alpha, A, lda, B, ldb, beta, C, ldc, nb, tb::Split::kPlain, Ah,
                                    Ah ? (size_t)2 * n * k * sizeof(__half) : 0, tb::current_stream()));
}

void tc_cumpsgemm_syr2k(cumpsgemm::handle_t, long int n, long int k, float alpha, float* A, long int lda, float* B,
                        long int ldb, float beta, float* C, long int ldc, long int nb) {
  report("tc_cumpsgemm_syr2k", tb::syr2k_impl(n, k, alpha, A, lda, B, ldb, beta, C, ldc, nb, tb::Split::kHiLo,
                                              nullptr, 0, tb::current_stream()));
}

void tc_trmm(cublasHandle_t, long int m, long int n, float alpha, float* A, long int lda, float* B, long int ldb,
             float* C, long int ldc, __half* hwork, long int nb) {
  report("tc_trmm", tb::trmm_impl(false, m, n, alpha, A, lda, B, ldb, C, ldc, nb, tb::Split::kPlain, hwork,
                                  hwork ? ((size_t)m * m + (size_t)m * n) * sizeof(__half) : 0,
                                  tb::current_stream()));
}

void tc_cumpsgemm_trmm(cumpsgemm::handle_t, long int m, long int n, float alpha, float* A, long int lda, float* B,
                       long int ldb, float* C, long int ldc, long int nb) {
  report("tc_cumpsgemm_trmm", tb::trmm_impl(false, m, n, alpha, A, lda, B, ldb, C, ldc, nb, tb::Split::kHiLo,
                                            nullptr, 0, tb::current_stream()));
}

void tc_symm(cublasHandle_t, long int m, long int n, float alpha, float* A, long int lda, float* B, int ldb,
             float beta, float* C, long int ldc, __half* Ah) {
  report("tc_symm", tb::symm_impl(true, m, n, alpha, A, lda, B, ldb, beta, C, ldc, tb::Split::kPlain, Ah,
                                  Ah ? ((size_t)m * m + (size_t)m * n) * sizeof(__half) : 0,
                                  tb::current_stream()));
}

void tc_cumpsgemm_symm(cumpsgemm::handle_t, long int m, long int n, float alpha, float* A, long int lda, float* B,
                       int ldb, float beta, float* C, long int ldc) {
  report("tc_cumpsgemm_symm", tb::symm_impl(true, m, n, alpha, A, lda, B, ldb, beta, C, ldc, tb::Split::kHiLo,
                                            nullptr, 0, tb::current_stream()));
}
