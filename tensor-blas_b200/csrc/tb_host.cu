// Host-memory forms of SYRK and TRSM (tb_ssyrk_host, tb_strsm_host).
//
// The reference's callers copy whole operands to the device, run the routine
// and copy the results back, one step after the other (python/TensorBLAS.py:
// 11-68 goes through torch CUDA tensors; testing/testing_syrk.cu copies with
// cudaMemcpy around tc_syrk). Here the operands stay in host memory
// (page-locked for full PCIe speed) and each call moves them through device
// staging buffers in panels on two copy streams, so host->device copies,
// tensor-core work and device->host copies of different panels overlap; only
// the referenced triangle of a triangular operand crosses the bus, and SYRK
// returns only the lower triangle it computes.
//
//  SYRK, C = alpha A A^T + beta C (lower): row panel i of A (rows [r0, r1),
//   all k columns) is copied as FP32 and converted on the device into the
//   FP16 copy of A (optionally, in plain precision, converted to FP16 on the
//   host's cores first, tb_host_convert.cpp, so half the bytes cross PCIe),
//   and row panel i of C (rows [r0, r1), columns [0, r1)) is computed from
//   it and the panels before it and copied back while panel i+1 is on its
//   way.
//  TRSM: A's lower triangle is copied once and prepared (FP16 copy, leaf
//   inverses); B then flows through a ring of device panels (columns for the
//   left side, rows for the right side: those are independent systems).
//
// Calls are synchronous: they return when the results are in host memory.
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "tb_internal.h"

namespace tb {
namespace {

constexpr int kMaxDev = 64;
constexpr int kEvents = 32;
constexpr int kSyrkSlots = 3;  // SYRK staging slots for A and C panels

struct HostPipes {
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev[kEvents] = {};
};
HostPipes g_pipes[kMaxDev];
std::mutex g_pipe_mu;

tb_status pipes(HostPipes** out) {
  int d = 0;
  TB_CUDA_TRY(cudaGetDevice(&d));
  if (d < 0 || d >= kMaxDev) return TB_ERROR_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lk(g_pipe_mu);
  HostPipes& p = g_pipes[d];
  if (!p.h2d) {
    TB_CUDA_TRY(cudaStreamCreateWithFlags(&p.h2d, cudaStreamNonBlocking));
    TB_CUDA_TRY(cudaStreamCreateWithFlags(&p.d2h, cudaStreamNonBlocking));
    for (cudaEvent_t& e : p.ev) TB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  *out = &p;
  return TB_SUCCESS;
}

// Makes `waiter` wait for all work queued so far on `signaller`.
tb_status join(cudaStream_t waiter, cudaStream_t signaller, cudaEvent_t ev) {
  TB_CUDA_TRY(cudaEventRecord(ev, signaller));
  TB_CUDA_TRY(cudaStreamWaitEvent(waiter, ev, 0));
  return TB_SUCCESS;
}

// Event slots of the per-device set.
enum : int {
  kEvStart = 0,
  kEvEndH2d,
  kEvEndD2h,
  kEvA,         // [3] A panel staged
  kEvC = 6,     // [3] C panel staged
  kEvConv = 9,  // [3] A staging slot consumed
  kEvGemm = 12, // [3] C panel computed
  kEvOut = 15,  // [3] panel copied back
  kEvIn = 18,   // [3] B panel staged
  kEvDone = 21, // [3] B panel solved
  kEvTri = 24,  // A triangle staged
};

// Page-locked host staging for the FP16 row panels of A (plain SYRK), per
// device, grown on demand and kept until tb_release_scratch.
struct HostStage {
  void* p = nullptr;
  size_t bytes = 0;
};
HostStage g_stage[kMaxDev];

void* host_stage(size_t bytes) {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDev) return nullptr;
  std::lock_guard<std::mutex> lk(g_pipe_mu);
  HostStage& h = g_stage[d];
  if (h.bytes >= bytes) return h.p;
  if (h.p) {
    cudaDeviceSynchronize();  // copies still reading the old buffer must finish
    cudaFreeHost(h.p);
    h.p = nullptr;
    h.bytes = 0;
  }
  if (cudaHostAlloc(&h.p, bytes, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    h.p = nullptr;
    return nullptr;
  }
  h.bytes = bytes;
  return h.p;
}

// Which of SYRK's A panels the host converts (plain precision): every
// n-th (TB_HOST_F16_EVERY in the environment, read once). Default 0, none:
// on the B200 boxes measured, 16 host cores converted a 64 MB panel more
// slowly than PCIe moved it as FP32 (SYRK n = k = 16384 from host memory:
// 24.7-25.5 ms with the device converting, 28.8-29.1 ms with the host
// converting every panel), so the option pays only on hosts with more
// memory bandwidth per PCIe link.
int host_convert_every() {
  static const int v = [] {
    const char* e = getenv("TB_HOST_F16_EVERY");
    const int x = e ? atoi(e) : 0;
    return x >= 0 ? x : 0;
  }();
  return v;
}

tb_status finish(cudaStream_t cs, HostPipes& p) {
  TB_TRY(join(cs, p.h2d, p.ev[kEvEndH2d]));
  TB_TRY(join(cs, p.d2h, p.ev[kEvEndD2h]));
  TB_CUDA_TRY(cudaStreamSynchronize(cs));
  return check_device_error(cs);
}

}  // namespace

tb_status syrk_host(long n, long k, float alpha, const float* hA, long lda, float beta, float* hC, long ldc, long nb,
                    Split split) {
  if (n < 0 || k < 0 || nb <= 0 || lda < (n > 1 ? n : 1) || ldc < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  if (n == 0) return TB_SUCCESS;
  if (!hA && k > 0) return TB_ERROR_INVALID_VALUE;
  if (!hC) return TB_ERROR_INVALID_VALUE;
  if (k == 0 || alpha == 0.f) {
    set_last_error("tb_ssyrk_host: k == 0 / alpha == 0 are not supported (use tb_ssyrk)");
    return TB_ERROR_NOT_SUPPORTED;
  }
  HostPipes* pp = nullptr;
  TB_TRY(pipes(&pp));
  HostPipes& p = *pp;
  const cudaStream_t cs = current_stream();
  const bool hilo = split == Split::kHiLo;
  const long P = 1024;  // panel rows (a multiple of the 128-row tile)
  const long long ldh = round_up(n, 64);
  const size_t half_bytes = (size_t)round_up(ldh * k * 2, 256);
  const size_t stA_bytes = (size_t)round_up((long long)P * k * 4, 256);
  const size_t cb_bytes = (size_t)round_up((long long)P * n * 4, 256);
  // plain: A's row panels are converted to FP16 on the host's cores into
  // page-locked slots and copied straight into the device FP16 copy (half
  // the bytes of FP32 across PCIe, no device conversion); split keeps the
  // FP32 upload and the device conversion (hi and lo are as many bytes as
  // FP32). Without the page-locked slots, plain falls back to the latter.
  uint16_t* h16 = nullptr;
  const size_t h16_slot = (size_t)P * (size_t)k * 2;
  const int every = host_convert_every();
  if (!hilo && every > 0) h16 = static_cast<uint16_t*>(host_stage(kSyrkSlots * h16_slot));
  const bool all_host = h16 && every == 1;
  const size_t total = half_bytes * (hilo ? 2 : 1) + kSyrkSlots * ((all_host ? 0 : stA_bytes) + cb_bytes);
  char* ws = static_cast<char*>(pool_get(total, 1));
  if (!ws) {
    set_last_error("tb_ssyrk_host: cannot allocate %zu bytes of staging", total);
    return TB_ERROR_ALLOC;
  }
  __half* hi = reinterpret_cast<__half*>(ws);
  __half* lo = hilo ? reinterpret_cast<__half*>(ws + half_bytes) : nullptr;
  char* w2 = ws + half_bytes * (hilo ? 2 : 1);
  // three slots: the upload of panel i's C block waits for panel i-3's C to
  // have come back, so a long download does not hold up the uploads behind it
  float* stA[kSyrkSlots];
  float* cb[kSyrkSlots];
  const size_t stA_used = all_host ? 0 : stA_bytes;
  for (int q = 0; q < kSyrkSlots; ++q) {
    stA[q] = reinterpret_cast<float*>(w2 + q * stA_used);
    cb[q] = reinterpret_cast<float*>(w2 + kSyrkSlots * stA_used + q * cb_bytes);
  }

  // everything starts after the work already queued on the caller's stream
  TB_TRY(join(p.h2d, cs, p.ev[kEvStart]));
  TB_CUDA_TRY(cudaStreamWaitEvent(p.d2h, p.ev[kEvStart], 0));

  Operand op;
  op.ptr = hi;
  op.rows = n;
  op.cols = k;
  op.ld = ldh;
  op.mn_major = true;
  Operand opl = op;
  opl.ptr = lo;
  const int kb = (int)((k + kGemmBK - 1) / kGemmBK);
  const int bn = gemm_bn(split, kb);
  const long npan = (n + P - 1) / P;
  for (long i = 0; i < npan; ++i) {
    const long r0 = i * P, r1 = std::min(n, r0 + P), pr = r1 - r0;
    const int s = (int)(i % kSyrkSlots);
    const bool on_host = h16 && i % every == 0;
    if (on_host) {
      // A rows [r0, r1) -> FP16 on the host into page-locked slot s (free
      // once panel i-3's copy out of it has completed) -> the device copy
      uint16_t* slot = h16 + (size_t)s * (h16_slot / 2);
      if (i >= kSyrkSlots) TB_CUDA_TRY(cudaEventSynchronize(p.ev[kEvA + s]));
      host_f32_to_f16(hA + r0, lda, pr, k, slot, P);
      TB_CUDA_TRY(cudaMemcpy2DAsync(hi + r0, (size_t)ldh * 2, slot, (size_t)P * 2, (size_t)pr * 2, (size_t)k,
                                    cudaMemcpyHostToDevice, p.h2d));
    } else {
      // A rows [r0, r1) -> staging slot s (reused once panel i-3 was converted)
      if (i >= kSyrkSlots) TB_CUDA_TRY(cudaStreamWaitEvent(p.h2d, p.ev[kEvConv + s], 0));
      TB_CUDA_TRY(cudaMemcpy2DAsync(stA[s], P * 4, hA + r0, (size_t)lda * 4, (size_t)pr * 4, (size_t)k,
                                    cudaMemcpyHostToDevice, p.h2d));
    }
    TB_CUDA_TRY(cudaEventRecord(p.ev[kEvA + s], p.h2d));
    // C rows [r0, r1): the diagonal block (its strict upper part must come
    // back unchanged), or all columns [0, r1) when beta != 0
    if (i >= kSyrkSlots) TB_CUDA_TRY(cudaStreamWaitEvent(p.h2d, p.ev[kEvOut + s], 0));
    const long c0 = beta != 0.f ? 0 : r0;
    TB_CUDA_TRY(cudaMemcpy2DAsync(cb[s] + c0 * P, P * 4, hC + r0 + (size_t)c0 * ldc, (size_t)ldc * 4, (size_t)pr * 4,
                                  (size_t)(r1 - c0), cudaMemcpyHostToDevice, p.h2d));
    TB_CUDA_TRY(cudaEventRecord(p.ev[kEvC + s], p.h2d));
    // convert into the FP16 copy of A (unless the host did), then the
    // panel's lower tiles
    TB_CUDA_TRY(cudaStreamWaitEvent(cs, p.ev[kEvA + s], 0));
    if (!on_host) {
      TB_TRY(convert_f32_f16(pr, k, stA[s], P, hi + r0, lo ? lo + r0 : nullptr, ldh, 2048.f, 0, cs));
      TB_CUDA_TRY(cudaEventRecord(p.ev[kEvConv + s], cs));
    }
    TB_CUDA_TRY(cudaStreamWaitEvent(cs, p.ev[kEvC + s], 0));
    std::vector<int4> plan;
    for (int g = 0; g < (int)((r1 + bn - 1) / bn); g += 8)
      for (long m0 = 0; m0 < pr; m0 += kGemmBM)
        for (int j = g; j < std::min<int>(g + 8, (int)((r1 + bn - 1) / bn)); ++j)
          if ((long)j * bn <= r0 + m0 + kGemmBM - 1) plan.push_back(make_int4((int)m0, j * bn, 0, kb));
    GemmCall c;
    c.a_hi = op;
    c.a_lo = opl;
    c.b_hi = op;
    c.b_lo = opl;
    c.a_off = (int)r0;
    c.split = split;
    c.kblocks = kb;
    c.C = cb[s];
    c.ldc = P;
    c.M = (int)pr;
    c.N = (int)r1;
    c.alpha = alpha;
    c.beta = beta;
    c.tri = 1;
    c.diag = (int)-r0;  // global row r0 + i >= column j
    c.flops = (double)pr * (double)(r0 + r1 + 1) * (double)k;
    TB_TRY(gemm_launch_plan(c, plan, cs));
    TB_CUDA_TRY(cudaEventRecord(p.ev[kEvGemm + s], cs));
    // C rows [r0, r1), columns [0, r1) -> host
    TB_CUDA_TRY(cudaStreamWaitEvent(p.d2h, p.ev[kEvGemm + s], 0));
    TB_CUDA_TRY(cudaMemcpy2DAsync(hC + r0, (size_t)ldc * 4, cb[s], P * 4, (size_t)pr * 4, (size_t)r1,
                                  cudaMemcpyDeviceToHost, p.d2h));
    TB_CUDA_TRY(cudaEventRecord(p.ev[kEvOut + s], p.d2h));
  }
  return finish(cs, p);
}

tb_status trsm_host(bool right, long m, long n, const float* hA, long lda, float* hB, long ldb, long nb, Split split) {
  if (m < 0 || n < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  const long nt = right ? n : m;
  if (lda < (nt > 1 ? nt : 1) || ldb < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  if (!hA || !hB) return TB_ERROR_INVALID_VALUE;
  HostPipes* pp = nullptr;
  TB_TRY(pipes(&pp));
  HostPipes& p = *pp;
  const cudaStream_t cs = current_stream();
  const long W = 1024;  // panel width (left: columns of B) / height (right: rows of B)
  const long other = right ? m : n;
  const long w_max = std::min(W, other);
  const size_t a_bytes = (size_t)round_up((long long)nt * nt * 4, 256);
  const size_t pb_bytes = (size_t)round_up((long long)w_max * nt * 4, 256);
  const size_t total = a_bytes + 3 * pb_bytes;
  char* ws = static_cast<char*>(pool_get(total, 1));
  if (!ws) {
    set_last_error("tb_strsm_host: cannot allocate %zu bytes of staging", total);
    return TB_ERROR_ALLOC;
  }
  float* dA = reinterpret_cast<float*>(ws);
  float* pb[3];
  for (int s = 0; s < 3; ++s) pb[s] = reinterpret_cast<float*>(ws + a_bytes + s * pb_bytes);

  TB_TRY(join(p.h2d, cs, p.ev[kEvStart]));
  TB_CUDA_TRY(cudaStreamWaitEvent(p.d2h, p.ev[kEvStart], 0));
  // lower triangle of A, in column panels: columns [c0, c1), rows [c0, nt)
  for (long c0 = 0; c0 < nt; c0 += W) {
    const long c1 = std::min(nt, c0 + W);
    TB_CUDA_TRY(cudaMemcpy2DAsync(dA + c0 + (size_t)c0 * nt, (size_t)nt * 4, hA + c0 + (size_t)c0 * lda,
                                  (size_t)lda * 4, (size_t)(nt - c0) * 4, (size_t)(c1 - c0), cudaMemcpyHostToDevice,
                                  p.h2d));
  }
  TB_CUDA_TRY(cudaEventRecord(p.ev[kEvTri], p.h2d));
  TB_CUDA_TRY(cudaStreamWaitEvent(cs, p.ev[kEvTri], 0));
  TrsmCtx ctx;
  std::vector<long> leaf_start;
  TB_TRY(trsm_setup(right, right ? w_max : m, right ? n : w_max, dA, nt, nb, split, cs, nullptr, ctx, leaf_start));

  const long npan = (other + W - 1) / W;
  for (long i = 0; i < npan; ++i) {
    const long q0 = i * W, q = std::min(W, other - q0);
    const int s = (int)(i % 3);
    if (i >= 3) TB_CUDA_TRY(cudaStreamWaitEvent(p.h2d, p.ev[kEvOut + s], 0));
    if (right) {
      // rows [q0, q0 + q) of B (q x n) -> panel (ld w_max)
      TB_CUDA_TRY(cudaMemcpy2DAsync(pb[s], (size_t)w_max * 4, hB + q0, (size_t)ldb * 4, (size_t)q * 4, (size_t)n,
                                    cudaMemcpyHostToDevice, p.h2d));
    } else {
      // columns [q0, q0 + q) of B (m x q) -> panel (ld m)
      TB_CUDA_TRY(cudaMemcpy2DAsync(pb[s], (size_t)m * 4, hB + (size_t)q0 * ldb, (size_t)ldb * 4, (size_t)m * 4,
                                    (size_t)q, cudaMemcpyHostToDevice, p.h2d));
    }
    TB_CUDA_TRY(cudaEventRecord(p.ev[kEvIn + s], p.h2d));
    TB_CUDA_TRY(cudaStreamWaitEvent(cs, p.ev[kEvIn + s], 0));
    if (right)
      TB_TRY(trsm_solve(ctx, leaf_start, pb[s], w_max, q, n));
    else
      TB_TRY(trsm_solve(ctx, leaf_start, pb[s], m, m, q));
    TB_CUDA_TRY(cudaEventRecord(p.ev[kEvDone + s], cs));
    TB_CUDA_TRY(cudaStreamWaitEvent(p.d2h, p.ev[kEvDone + s], 0));
    if (right)
      TB_CUDA_TRY(cudaMemcpy2DAsync(hB + q0, (size_t)ldb * 4, pb[s], (size_t)w_max * 4, (size_t)q * 4, (size_t)n,
                                    cudaMemcpyDeviceToHost, p.d2h));
    else
      TB_CUDA_TRY(cudaMemcpy2DAsync(hB + (size_t)q0 * ldb, (size_t)ldb * 4, pb[s], (size_t)m * 4, (size_t)m * 4,
                                    (size_t)q, cudaMemcpyDeviceToHost, p.d2h));
    TB_CUDA_TRY(cudaEventRecord(p.ev[kEvOut + s], p.d2h));
  }
  return finish(cs, p);
}

void release_host_staging() {
  std::lock_guard<std::mutex> lk(g_pipe_mu);
  for (HostStage& h : g_stage) {
    if (h.p) cudaFreeHost(h.p);
    h.p = nullptr;
    h.bytes = 0;
  }
}

}  // namespace tb

namespace {
tb::Split prec(int precision) { return precision == TB_PREC_SPLIT ? tb::Split::kHiLo : tb::Split::kPlain; }
}  // namespace

extern "C" tb_status tb_ssyrk_host(char uplo, char trans, long n, long k, float alpha, const float* A, long lda,
                                   float beta, float* C, long ldc, long nb, int precision) {
  if (uplo != 'L' && uplo != 'l') {
    tb::set_last_error("tb_ssyrk_host: only uplo='L' is supported");
    return TB_ERROR_NOT_SUPPORTED;
  }
  if (trans != 'N' && trans != 'n') {
    tb::set_last_error("tb_ssyrk_host: only trans='N' is supported");
    return TB_ERROR_NOT_SUPPORTED;
  }
  if (precision != TB_PREC_PLAIN && precision != TB_PREC_SPLIT) return TB_ERROR_INVALID_VALUE;
  return tb::syrk_host(n, k, alpha, A, lda, beta, C, ldc, nb, prec(precision));
}

extern "C" tb_status tb_strsm_host(char side, long m, long n, const float* A, long lda, float* B, long ldb, long nb,
                                   int precision) {
  bool right;
  if (side == 'R' || side == 'r')
    right = true;
  else if (side == 'L' || side == 'l')
    right = false;
  else
    return TB_ERROR_INVALID_VALUE;
  if (precision != TB_PREC_PLAIN && precision != TB_PREC_SPLIT) return TB_ERROR_INVALID_VALUE;
  return tb::trsm_host(right, m, n, A, lda, B, ldb, nb, prec(precision));
}
