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
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "tb_gemm.cuh"
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

// Lower SYRK with the conversion of A overlapped with the tensor-core work:
// A's FP16 copy is made in syrk_parts() row bands (256-aligned) on the
// caller's stream, and the tiles of row band q (which read bands 0..q only)
// are launched as soon as band q is converted, alternately on two auxiliary
// streams, so the later bands' conversion and each launch's last wave run
// beside other bands' tiles. The tiles, their K ranges and the FP32 sums are
// those of the single launch (the results are bit-identical).
// TB_SYRK_PARTS in the environment sets the number of bands (1: one
// conversion and one launch; read once).
constexpr int kSyrkPartsMax = 16;

int syrk_parts() {
  static const int parts = [] {
    const char* e = getenv("TB_SYRK_PARTS");
    const int v = e ? atoi(e) : 0;
    return (v >= 1 && v <= kSyrkPartsMax) ? v : 4;
  }();
  return parts;
}

tb_status syrk_lower_overlapped(bool trans, long n, long k, float alpha, const float* A, long lda, float beta, float* C,
                                long ldc, Split split, __half* hi, __half* lo, long long ldh, cudaStream_t st) {
  const cudaStream_t sq[2] = {aux_stream(0), aux_stream(1)};
  if (!sq[0] || !sq[1]) return TB_ERROR_CUDA;
  const int kb = (int)((k + kGemmBK - 1) / kGemmBK);
  const int bn = gemm_bn(split, kb);
  const std::vector<int4> plan = plan_lower((int)n, bn, 0, kb);
  const int parts = syrk_parts();
  long bounds[kSyrkPartsMax + 1];
  // equal row bands: bands that double in size (the first band's
  // conversion, the one no tiles hide, smallest) measured 3-5 % slower at
  // n = k = 16384 (their largest launch holds three quarters of the tiles)
  for (int q = 0; q <= parts; ++q) bounds[q] = std::min<long>(n, round_up((long long)n * q / parts, 256));
  cudaEvent_t ev[kSyrkPartsMax + 3];
  for (auto& e : ev) TB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  tb_status rs = TB_SUCCESS;
  // the auxiliary streams start after the work queued before this call
  if (cudaEventRecord(ev[parts], st) != cudaSuccess || cudaStreamWaitEvent(sq[0], ev[parts], 0) != cudaSuccess ||
      cudaStreamWaitEvent(sq[1], ev[parts], 0) != cudaSuccess)
    rs = TB_ERROR_CUDA;
  for (int q = 0; q < parts && rs == TB_SUCCESS; ++q) {
    const long r0 = bounds[q], r1 = bounds[q + 1];
    if (r1 <= r0) continue;
    // band q of the operand: rows [r0, r1) of A ('N') or columns of A ('T')
    if (trans)
      rs = convert_f32_f16(k, r1 - r0, A + r0 * lda, lda, hi + r0 * ldh, lo ? lo + r0 * ldh : nullptr, ldh, 2048.f, 0,
                           st);
    else
      rs = convert_f32_f16(r1 - r0, k, A + r0, lda, hi + r0, lo ? lo + r0 : nullptr, ldh, 2048.f, 0, st);
    if (rs != TB_SUCCESS) break;
    if (cudaEventRecord(ev[q], st) != cudaSuccess || cudaStreamWaitEvent(sq[q & 1], ev[q], 0) != cudaSuccess) {
      rs = TB_ERROR_CUDA;
      break;
    }
    std::vector<int4> part;
    for (const int4& t : plan)
      if (t.x >= r0 && t.x < r1) part.push_back(t);
    Operand op;
    op.ptr = hi;
    op.rows = n;
    op.cols = k;
    op.ld = ldh;
    op.mn_major = !trans;
    Operand opl = op;
    opl.ptr = lo;
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
    c.tri = 1;
    c.flops = (double)k * ((double)r1 * (r1 + 1) - (double)r0 * (r0 + 1));  // rows [r0, r1) of the lower triangle
    rs = gemm_launch_plan(c, part, sq[q & 1]);
  }
  // the caller's stream continues after both auxiliary streams
  if (cudaEventRecord(ev[parts + 1], sq[0]) != cudaSuccess ||
      cudaEventRecord(ev[parts + 2], sq[1]) != cudaSuccess ||
      cudaStreamWaitEvent(st, ev[parts + 1], 0) != cudaSuccess ||
      cudaStreamWaitEvent(st, ev[parts + 2], 0) != cudaSuccess)
    rs = rs == TB_SUCCESS ? TB_ERROR_CUDA : rs;
  for (auto& e : ev) cudaEventDestroy(e);
  return rs;
}

namespace {

// Split-K form (a choice of the autotuner, for plain 'N' SYRKs whose
// triangle has fewer tiles than the GPU has SMs: small n, long k). The K
// range is cut into `splits` contiguous parts of whole K-blocks; part q is
// problem q of ONE grouped launch of the tcgen05 engine and writes its FP32
// partial triangle (alpha 1, beta 0) to plane q of a scratch array, and
// syrk_splitk_reduce adds the planes in part order (deterministic) and
// applies alpha and beta. The sums are grouped differently from the one-pass
// form, so the results differ from it in FP32 rounding only.
__global__ void syrk_splitk_reduce(int n, int splits, const float* __restrict__ P, long long plane, int ldp,
                                   float alpha, float beta, float* C, long long ldc, int upper) {
  const int j = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || (upper ? i > j : i < j)) return;
  float s = 0.f;
  for (int q = 0; q < splits; ++q) s += __ldcs(P + q * plane + i + (long long)j * ldp);
  float* c = C + i + (long long)j * ldc;
  *c = beta == 0.f ? alpha * s : alpha * s + beta * *c;
}

thread_local int t_splitk = 1;

}  // namespace

void set_splitk_override(int splits) { t_splitk = splits > 1 ? splits : 1; }
int splitk_override() { return t_splitk; }

namespace {

tb_status syrk_splitk(long n, long k, float alpha, float beta, float* C, long ldc, const __half* hi, long long ldh,
                      float* P, int ldp, int splits, bool upper, cudaStream_t st) {
  const int kb = (int)((k + kGemmBK - 1) / kGemmBK);
  const long long plane = (long long)ldp * n;
  Operand op;
  op.ptr = hi;
  op.rows = n;
  op.cols = k;
  op.ld = ldh;
  op.mn_major = true;
  std::vector<GemmArgs> probs(splits);
  std::vector<int4> tiles;
  std::vector<int> tprob;
  for (int q = 0; q < splits; ++q) {
    const int k0 = (int)((long long)kb * q / splits), k1 = (int)((long long)kb * (q + 1) / splits);
    GemmCall c;
    c.a_hi = c.b_hi = op;
    c.split = Split::kPlain;
    c.kblocks = kb;  // > kGemmPfMaxKb: the 256-row B box of the grouped plain kernel (the tiles carry [k0, k1))
    c.C = P + q * plane;
    c.ldc = ldp;
    c.M = (int)n;
    c.N = (int)n;
    c.alpha = 1.f;
    c.beta = 0.f;
    c.tri = upper ? 2 : 1;
    c.diag = 0;
    TB_TRY(gemm_build_args(c, &probs[q]));
    const std::vector<int4> part = upper ? plan_upper((int)n, 256, k0, k1) : plan_lower((int)n, 256, k0, k1);
    tiles.insert(tiles.end(), part.begin(), part.end());
    tprob.insert(tprob.end(), part.size(), q);
  }
  // problems (64-byte multiples) followed by the tiles' problem indices, in
  // one device list cached by content
  static_assert(sizeof(GemmArgs) % 64 == 0, "grouped problems are 64-byte aligned");
  const size_t pb = probs.size() * sizeof(GemmArgs), ib = round_up((long long)tprob.size() * sizeof(int), 16);
  std::vector<int4> blob((pb + ib) / sizeof(int4));
  memset(blob.data(), 0, pb + ib);
  memcpy(blob.data(), probs.data(), pb);
  memcpy(reinterpret_cast<char*>(blob.data()) + pb, tprob.data(), tprob.size() * sizeof(int));
  const int4* d_blob = upload_tiles(blob, st);
  const int4* d_tiles = upload_tiles(tiles, st);
  if (!d_blob || !d_tiles) {
    set_last_error("syrk: cannot upload the split-K tables");
    return TB_ERROR_ALLOC;
  }
  const double flops = (double)n * (double)(n + 1) * (double)k;
  TB_TRY(gemm_launch_grouped(Split::kPlain, reinterpret_cast<const GemmArgs*>(d_blob), d_tiles,
                             reinterpret_cast<const int*>(reinterpret_cast<const char*>(d_blob) + pb), (int)tiles.size(),
                             flops, st));
  syrk_splitk_reduce<<<dim3((unsigned)((n + 255) / 256), (unsigned)n), 256, 0, st>>>(
      (int)n, splits, P, plane, ldp, alpha, beta, C, ldc, upper ? 1 : 0);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

}  // namespace

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
  // split-K (autotuner's choice): plain 'N' only, each part >= 4 K-blocks,
  // partial planes of ldp x n FP32 after the FP16 copy
  const int kb_all = (int)((k + kGemmBK - 1) / kGemmBK);
  int splits = (split == Split::kPlain && !trans && n <= kSplitKMaxN && kb_all > kGemmPfMaxKb)
                   ? std::min(splitk_override(), kb_all / 4)
                   : 1;
  const int ldp = (int)round_up(n, 32);
  const size_t pbytes = splits > 1 ? (size_t)splits * ldp * n * sizeof(float) : 0;
  const size_t need = one * (hilo ? 2 : 1);
  if (splits > 1) ws = nullptr;  // partials go to the pool after the copy
  void* buf = (ws && ws_bytes >= need) ? ws : pool_get(round_up(need, 256) + pbytes);
  if (!buf) {
    set_last_error("syrk: cannot allocate %zu bytes of scratch", need);
    return TB_ERROR_ALLOC;
  }
  __half* hi = static_cast<__half*>(buf);
  __half* lo = hilo ? reinterpret_cast<__half*>(static_cast<char*>(buf) + one) : nullptr;
  const int kb = (int)((k + kGemmBK - 1) / kGemmBK);
  const int bn = gemm_bn(split, kb);
  if (!upper && syrk_parts() > 1 && n >= 8192 && kb > kGemmPfMaxKb && splits <= 1)
    return syrk_lower_overlapped(trans, n, k, alpha, A, lda, beta, C, ldc, split, hi, lo, ldh, st);
  TB_TRY(convert_f32_f16(rows, cols, A, lda, hi, lo, ldh, 2048.f, 0, st));
  if (splits > 1)
    return syrk_splitk(n, k, alpha, beta, C, ldc, hi, ldh,
                       reinterpret_cast<float*>(static_cast<char*>(buf) + round_up(need, 256)), ldp, splits, upper, st);

  Operand op;
  op.ptr = hi;
  op.rows = n;
  op.cols = k;
  op.ld = ldh;
  op.mn_major = !trans;
  Operand opl = op;
  opl.ptr = lo;

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
