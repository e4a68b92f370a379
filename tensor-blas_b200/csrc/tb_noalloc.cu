// SYRK entry point that performs no device-memory allocation.
//
// Some callers of this library cannot call cudaMalloc: code embedded in an
// application whose GPU memory is already owned by another allocator (for
// example a framework's caching allocator that has reserved nearly all of
// HBM, where a fresh cudaMalloc fails or fragments the reserve), and
// latency-sensitive callers that cannot afford the implicit device-wide
// synchronisation of cudaMalloc / cudaFree. tb_ssyrk_noalloc serves them:
// its scratch (the tile list and the FP16 copy of A) lives in one statically
// sized __device__ array of this file, which every GPU that loads the
// library holds until the process exits.
//
//  * Capacity: kNoAllocScratchBytes (64 MiB). A call whose tile list plus
//    FP16 copy (round_up(rows, 64) * cols halves, twice that for the split
//    precision) does not fit is rejected with TB_ERROR_INVALID_VALUE and a
//    message giving the bytes it would need.
//  * Set-up: the first call on each device resolves the array's device
//    address with cudaGetSymbolAddress (the array's name in host code is
//    only a host-side stand-in). Make that first call before any stream
//    capture.
//  * Sharing: all calls use the same array, which keeps the previous call's
//    contents; the call's own device error block (a second static array) has
//    its code cleared at the start of every call. Calls that overlap on the
//    GPU (different streams, or different host threads) race on the array
//    and must be serialised by the caller.
//  * Errors: a bounded wait that runs out inside the kernel is recorded in
//    that error block, which the set-up registers with the library's
//    runtime, so tb_synchronize reports it (TB_ERROR_TIMEOUT) without
//    allocating anything.
//  * Scope: uplo 'L' or 'U', trans 'N' or 'T', TB_PREC_PLAIN or
//    TB_PREC_SPLIT, nb > 0 (TB_PREC_FP8 and TB_NB_AUTO need scratch of
//    their own and are rejected); k == 0 or alpha == 0 only scales C.
#include <cstdio>
#include <mutex>

#include "tb_internal.h"

namespace tb {
namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
__device__ __align__(16) int g_noalloc_err[4];

constexpr int kMaxDev = 64;
struct Symbols {
  bool ready = false;
  unsigned char* scratch = nullptr;
  int* err = nullptr;
};
Symbols g_sym[kMaxDev];
std::mutex g_sym_mu;

tb_status resolve_symbols(Symbols** out) {
  int dev = 0;
  TB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDev) return TB_ERROR_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lk(g_sym_mu);
  Symbols& s = g_sym[dev];
  if (!s.ready) {
    void* p = nullptr;
    TB_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    s.scratch = static_cast<unsigned char*>(p);
    TB_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_err));
    s.err = static_cast<int*>(p);
    register_error_block(s.err);
    s.ready = true;
  }
  *out = &s;
  return TB_SUCCESS;
}

}  // namespace
}  // namespace tb

extern "C" tb_status tb_ssyrk_noalloc(char uplo, char trans, long n, long k, float alpha, const float* A, long lda,
                                      float beta, float* C, long ldc, long nb, int precision) {
  using namespace tb;
  const bool upper = (uplo == 'U' || uplo == 'u');
  if (!upper && uplo != 'L' && uplo != 'l') return TB_ERROR_INVALID_VALUE;
  const bool t = (trans == 'T' || trans == 't' || trans == 'C' || trans == 'c');
  if (!t && trans != 'N' && trans != 'n') return TB_ERROR_INVALID_VALUE;
  if (precision != TB_PREC_PLAIN && precision != TB_PREC_SPLIT) {
    set_last_error("tb_ssyrk_noalloc: precision must be TB_PREC_PLAIN or TB_PREC_SPLIT");
    return TB_ERROR_INVALID_VALUE;
  }
  if (n < 0 || k < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  if (ldc < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  if (lda < ((t ? k : n) > 1 ? (t ? k : n) : 1)) return TB_ERROR_INVALID_VALUE;
  if (n == 0) return TB_SUCCESS;
  cudaStream_t st = current_stream();
  // nothing to multiply: C = beta C on the referenced triangle (no scratch)
  if (k == 0 || alpha == 0.f) return beta == 1.f ? TB_SUCCESS : scale_lower(n, beta, C, ldc, st, upper);
  const Split split = precision == TB_PREC_SPLIT ? Split::kHiLo : Split::kPlain;
  const bool hilo = split == Split::kHiLo;
  const long long rows = t ? k : n, cols = t ? n : k;
  const long long ldh = round_up(rows, 64);
  const int bn = gemm_bn(split);
  const int kb = (int)((k + kGemmBK - 1) / kGemmBK);
  const std::vector<int4> plan = upper ? plan_upper((int)n, bn, 0, kb) : plan_lower((int)n, bn, 0, kb);
  const size_t tiles_bytes = (size_t)round_up((long long)(plan.size() * sizeof(int4)), 256);
  const size_t one = (size_t)round_up(ldh * cols * (long long)sizeof(__half), 256);
  const size_t need = tiles_bytes + one * (hilo ? 2 : 1);
  if (need > kNoAllocScratchBytes) {
    set_last_error("tb_ssyrk_noalloc: needs %zu bytes of scratch, the static maximum is %zu bytes", need,
                   kNoAllocScratchBytes);
    return TB_ERROR_INVALID_VALUE;
  }
  Symbols* sym = nullptr;
  TB_TRY(resolve_symbols(&sym));
  int4* tiles = reinterpret_cast<int4*>(sym->scratch);
  __half* hi = reinterpret_cast<__half*>(sym->scratch + tiles_bytes);
  __half* lo = hilo ? reinterpret_cast<__half*>(sym->scratch + tiles_bytes + one) : nullptr;
  TB_CUDA_TRY(cudaMemsetAsync(sym->err, 0, sizeof(int), st));
  // pageable source: the copy is staged by the runtime before the call returns
  TB_CUDA_TRY(cudaMemcpyAsync(tiles, plan.data(), plan.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
  TB_TRY(convert_f32_f16(rows, cols, A, lda, hi, lo, ldh, 2048.f, 0, st));
  GemmCall c;
  c.a_hi = {hi, n, k, ldh, !t};
  c.a_lo = {lo, n, k, ldh, !t};
  c.b_hi = c.a_hi;
  c.b_lo = c.a_lo;
  c.split = split;
  c.tiles = tiles;
  c.num_tiles = (int)plan.size();
  c.C = C;
  c.ldc = ldc;
  c.M = c.N = (int)n;
  c.alpha = alpha;
  c.beta = beta;
  c.tri = upper ? 2 : 1;
  c.err = sym->err;
  c.flops = (double)n * (double)(n + 1) * (double)k;
  return gemm_launch(c, st);
}
