// Host-buffer entry points around the REFERENCE library's own routines
// (compiled from its sources by oracle/Makefile). Test infrastructure: used by
// tests/golden/make_golden.py to record the reference's outputs, and by
// bench.py's reference arm to time the reference on the same B200.
// Column-major host arrays; every call uploads, runs the reference routine on
// its default stream through its C++ API, and downloads.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "TensorBLAS.h"  // the reference's include/TensorBLAS.h

namespace {
cublasHandle_t handle() {
  static cublasHandle_t h = nullptr;
  if (!h) cublasCreate(&h);
  return h;
}
template <class T>
T* up(const T* h, size_t n) {
  T* d = nullptr;
  if (cudaMalloc(&d, n * sizeof(T)) != cudaSuccess) return nullptr;
  if (h) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
  return d;
}
template <class T>
int down(T* h, const T* d, size_t n) {
  return cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : 1;
}
int finish() {
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? 0 : 2;
}
struct Events {
  cudaEvent_t a, b;
  Events() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Events() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};
double median(std::vector<float>& v) {
  std::sort(v.begin(), v.end());
  return v.empty() ? -1.0 : v[v.size() / 2];
}
}  // namespace

extern "C" {

// C(lower) = alpha A A^T + beta C ; A n x k (lda = n), C n x n (ldc = n).
int ref_syrk(long n, long k, float alpha, const float* hA, float beta, float* hC, long nb) {
  float* A = up(hA, (size_t)n * k);
  float* C = up(hC, (size_t)n * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * 2 * n * k);
  tc_syrk(handle(), n, k, alpha, A, n, beta, C, n, w, nb);
  int rc = finish();
  if (!rc) rc = down(hC, C, (size_t)n * n);
  cudaFree(A);
  cudaFree(C);
  cudaFree(w);
  return rc;
}

// X A^T = B (right/lower/T/non-unit), A n x n (lda = n), B m x n (ldb = m), B <- X.
int ref_trsm(long m, long n, const float* hA, float* hB, long nb) {
  float* A = up(hA, (size_t)n * n);
  float* B = up(hB, (size_t)m * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * ((size_t)n / 2 * n / 2 + (size_t)m / 2 * n + 16));
  tc_trsm(handle(), m, n, A, n, B, m, w, nb);
  int rc = finish();
  if (!rc) rc = down(hB, B, (size_t)m * n);
  cudaFree(A);
  cudaFree(B);
  cudaFree(w);
  return rc;
}

// C = alpha A B, A m x m lower (strict upper must be zero), B, C m x n.
int ref_trmm(long m, long n, float alpha, const float* hA, const float* hB, float* hC, long nb) {
  float* A = up(hA, (size_t)m * m);
  float* B = up(hB, (size_t)m * n);
  float* C = up(hC, (size_t)m * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * ((size_t)m * n + (size_t)m * m));
  tc_trmm(handle(), m, n, alpha, A, m, B, m, C, m, w, nb);
  int rc = finish();
  if (!rc) rc = down(hC, C, (size_t)m * n);
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  cudaFree(w);
  return rc;
}

// C(lower) = alpha (A B^T + B A^T) + beta C ; A, B n x k, C n x n.
int ref_syr2k(long n, long k, float alpha, const float* hA, const float* hB, float beta, float* hC, long nb) {
  float* A = up(hA, (size_t)n * k);
  float* B = up(hB, (size_t)n * k);
  float* C = up(hC, (size_t)n * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * 2 * n * k);
  tc_syr2k(handle(), n, k, alpha, A, n, B, n, beta, C, n, w, nb);
  int rc = finish();
  if (!rc) rc = down(hC, C, (size_t)n * n);
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  cudaFree(w);
  return rc;
}

// C = alpha A B + beta C, A m x m symmetric (lower stored), B, C m x n (m == n
// only: the reference's grids assume it, BLAS/tc_symm.cu:5-14).
int ref_symm(long m, long n, float alpha, const float* hA, const float* hB, float beta, float* hC) {
  float* A = up(hA, (size_t)m * m);
  float* B = up(hB, (size_t)m * n);
  float* C = up(hC, (size_t)m * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * ((size_t)m * m + (size_t)m * n));
  tc_symm(handle(), m, n, alpha, A, m, B, (int)m, beta, C, m, w);
  int rc = finish();
  if (!rc) rc = down(hC, C, (size_t)m * n);
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  cudaFree(w);
  return rc;
}

// FP64 SYRK through the reference's "ozimmu" driver (native FP64 cuBLAS).
int ref_ozimmu_syrk(long n, long k, double alpha, const double* hA, double beta, double* hC, long nb) {
  double* A = up(hA, (size_t)n * k);
  double* C = up(hC, (size_t)n * n);
  tc_ozimmu_syrk(handle(), n, k, alpha, A, n, beta, C, n, nb);
  int rc = finish();
  if (!rc) rc = down(hC, C, (size_t)n * n);
  cudaFree(A);
  cudaFree(C);
  return rc;
}

// FP64 X A^T = B through the reference's tc_ozimmu_trsm (native FP64 cuBLAS).
int ref_ozimmu_trsm(long m, long n, const double* hA, double* hB, long nb) {
  double* A = up(hA, (size_t)n * n);
  double* B = up(hB, (size_t)m * n);
  tc_ozimmu_trsm(handle(), m, n, A, n, B, m, nb);
  int rc = finish();
  if (!rc) rc = down(hB, B, (size_t)m * n);
  cudaFree(A);
  cudaFree(B);
  return rc;
}

// FP64 C = alpha A B (A lower, zero strict upper) through tc_ozimmu_trmm.
int ref_ozimmu_trmm(long m, long n, double alpha, const double* hA, const double* hB, double* hC, long nb) {
  double* A = up(hA, (size_t)m * m);
  double* B = up(hB, (size_t)m * n);
  double* C = up(hC, (size_t)m * n);
  tc_ozimmu_trmm(handle(), m, n, alpha, A, m, B, m, C, m, nb);
  int rc = finish();
  if (!rc) rc = down(hC, C, (size_t)m * n);
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  return rc;
}

// FP64 C = alpha (A B^T + B A^T) + beta C through tc_ozimmu_syr2k.
int ref_ozimmu_syr2k(long n, long k, double alpha, const double* hA, const double* hB, double beta, double* hC,
                     long nb) {
  double* A = up(hA, (size_t)n * k);
  double* B = up(hB, (size_t)n * k);
  double* C = up(hC, (size_t)n * n);
  tc_ozimmu_syr2k(handle(), n, k, alpha, A, n, B, n, beta, C, n, nb);
  int rc = finish();
  if (!rc) rc = down(hC, C, (size_t)n * n);
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  return rc;
}

// Median device time (ms) of tc_syrk(n, k, nb) on device-resident inputs.
double ref_time_syrk(long n, long k, long nb, const float* hA, int warmup, int iters) {
  float* A = up(hA, (size_t)n * k);
  float* C = up<float>(nullptr, (size_t)n * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * 2 * n * k);
  if (!A || !C || !w) return -1.0;
  Events ev;
  std::vector<float> t;
  for (int i = 0; i < warmup + iters; ++i) {
    cudaEventRecord(ev.a);
    tc_syrk(handle(), n, k, 1.0f, A, n, 0.0f, C, n, w, nb);
    cudaEventRecord(ev.b);
    cudaEventSynchronize(ev.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (i >= warmup) t.push_back(ms);
  }
  int rc = finish();
  cudaFree(A);
  cudaFree(C);
  cudaFree(w);
  return rc ? -1.0 : median(t);
}

// Median device time (ms) of tc_trsm(m, n, nb); B restored before each call
// (outside the timed region).
double ref_time_trsm(long m, long n, long nb, const float* hA, const float* hB, int warmup, int iters) {
  float* A = up(hA, (size_t)n * n);
  float* B0 = up(hB, (size_t)m * n);
  float* B = up<float>(nullptr, (size_t)m * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * ((size_t)n / 2 * n / 2 + (size_t)m / 2 * n + 16));
  if (!A || !B0 || !B || !w) return -1.0;
  Events ev;
  std::vector<float> t;
  for (int i = 0; i < warmup + iters; ++i) {
    cudaMemcpy(B, B0, sizeof(float) * m * n, cudaMemcpyDeviceToDevice);
    cudaEventRecord(ev.a);
    tc_trsm(handle(), m, n, A, n, B, m, w, nb);
    cudaEventRecord(ev.b);
    cudaEventSynchronize(ev.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (i >= warmup) t.push_back(ms);
  }
  int rc = finish();
  cudaFree(A);
  cudaFree(B0);
  cudaFree(B);
  cudaFree(w);
  return rc ? -1.0 : median(t);
}

}  // extern "C"

extern "C" {
// Median device time (ms) of the reference's tc_ozimmu_syrk (native FP64
// cuBLAS in its recursion) on device-resident inputs.
double ref_time_ozimmu_syrk(long n, long k, long nb, const double* hA, int warmup, int iters) {
  double* A = up(hA, (size_t)n * k);
  double* C = up<double>(nullptr, (size_t)n * n);
  if (!A || !C) return -1.0;
  Events ev;
  std::vector<float> t;
  for (int i = 0; i < warmup + iters; ++i) {
    cudaEventRecord(ev.a);
    tc_ozimmu_syrk(handle(), n, k, 1.0, A, n, 0.0, C, n, nb);
    cudaEventRecord(ev.b);
    cudaEventSynchronize(ev.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (i >= warmup) t.push_back(ms);
  }
  int rc = finish();
  cudaFree(A);
  cudaFree(C);
  return rc ? -1.0 : median(t);
}
}  // extern "C"

extern "C" {
// Median device times (ms) of the reference's tc_syr2k / tc_trmm / tc_symm
// on device-resident inputs (alpha = 1, beta = 0 where there is one).
double ref_time_syr2k(long n, long k, long nb, const float* hA, const float* hB, int warmup, int iters) {
  float* A = up(hA, (size_t)n * k);
  float* B = up(hB, (size_t)n * k);
  float* C = up<float>(nullptr, (size_t)n * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * 2 * n * k);
  if (!A || !B || !C || !w) return -1.0;
  Events ev;
  std::vector<float> t;
  for (int i = 0; i < warmup + iters; ++i) {
    cudaEventRecord(ev.a);
    tc_syr2k(handle(), n, k, 1.0f, A, n, B, n, 0.0f, C, n, w, nb);
    cudaEventRecord(ev.b);
    cudaEventSynchronize(ev.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (i >= warmup) t.push_back(ms);
  }
  int rc = finish();
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  cudaFree(w);
  return rc ? -1.0 : median(t);
}

double ref_time_trmm(long m, long n, long nb, const float* hA, const float* hB, int warmup, int iters) {
  float* A = up(hA, (size_t)m * m);
  float* B = up(hB, (size_t)m * n);
  float* C = up<float>(nullptr, (size_t)m * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * ((size_t)m * n + (size_t)m * m));
  if (!A || !B || !C || !w) return -1.0;
  Events ev;
  std::vector<float> t;
  for (int i = 0; i < warmup + iters; ++i) {
    cudaEventRecord(ev.a);
    tc_trmm(handle(), m, n, 1.0f, A, m, B, m, C, m, w, nb);
    cudaEventRecord(ev.b);
    cudaEventSynchronize(ev.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (i >= warmup) t.push_back(ms);
  }
  int rc = finish();
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  cudaFree(w);
  return rc ? -1.0 : median(t);
}

// tc_symm symmetrises A in place, which is idempotent, so repeated calls
// see the same operand.
double ref_time_symm(long m, long n, const float* hA, const float* hB, int warmup, int iters) {
  float* A = up(hA, (size_t)m * m);
  float* B = up(hB, (size_t)m * n);
  float* C = up<float>(nullptr, (size_t)m * n);
  __half* w = nullptr;
  cudaMalloc(&w, sizeof(__half) * ((size_t)m * m + (size_t)m * n));
  if (!A || !B || !C || !w) return -1.0;
  Events ev;
  std::vector<float> t;
  for (int i = 0; i < warmup + iters; ++i) {
    cudaEventRecord(ev.a);
    tc_symm(handle(), m, n, 1.0f, A, m, B, (int)m, 0.0f, C, m, w);
    cudaEventRecord(ev.b);
    cudaEventSynchronize(ev.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (i >= warmup) t.push_back(ms);
  }
  int rc = finish();
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  cudaFree(w);
  return rc ? -1.0 : median(t);
}
}  // extern "C"

extern "C" {
// End to end through the reference's public API, measured like the library's
// own end-to-end number: per step, page-locked host -> device copies of the
// SYRK input A (n x n) and the TRSM inputs A_tri (n x n) and B (n x n),
// tc_syrk(n, n, nb_syrk), tc_trsm(n, n, nb_trsm), device -> host copies of C
// and X, all on the default stream between two events. Median ms per step.
double ref_time_e2e(long n, long nb_syrk, long nb_trsm, const float* hA, const float* hT, const float* hB, int warmup,
                    int iters) {
  const size_t bytes = sizeof(float) * (size_t)n * n;
  float *pA = nullptr, *pT = nullptr, *pB = nullptr, *pC = nullptr, *pX = nullptr;
  if (cudaMallocHost(&pA, bytes) != cudaSuccess || cudaMallocHost(&pT, bytes) != cudaSuccess ||
      cudaMallocHost(&pB, bytes) != cudaSuccess || cudaMallocHost(&pC, bytes) != cudaSuccess ||
      cudaMallocHost(&pX, bytes) != cudaSuccess)
    return -1.0;
  memcpy(pA, hA, bytes);
  memcpy(pT, hT, bytes);
  memcpy(pB, hB, bytes);
  float *A = nullptr, *T = nullptr, *B = nullptr, *C = nullptr;
  __half *ws = nullptr, *wt = nullptr;
  cudaMalloc(&A, bytes);
  cudaMalloc(&T, bytes);
  cudaMalloc(&B, bytes);
  cudaMalloc(&C, bytes);
  cudaMalloc(&ws, sizeof(__half) * 2 * n * n);
  cudaMalloc(&wt, sizeof(__half) * ((size_t)n / 2 * n / 2 + (size_t)n / 2 * n + 16));
  if (!A || !T || !B || !C || !ws || !wt) return -1.0;
  Events ev;
  std::vector<float> t;
  for (int i = 0; i < warmup + iters; ++i) {
    cudaEventRecord(ev.a);
    cudaMemcpyAsync(A, pA, bytes, cudaMemcpyHostToDevice);
    cudaMemcpyAsync(T, pT, bytes, cudaMemcpyHostToDevice);
    cudaMemcpyAsync(B, pB, bytes, cudaMemcpyHostToDevice);
    tc_syrk(handle(), n, n, 1.0f, A, n, 0.0f, C, n, ws, nb_syrk);
    tc_trsm(handle(), n, n, T, n, B, n, wt, nb_trsm);
    cudaMemcpyAsync(pC, C, bytes, cudaMemcpyDeviceToHost);
    cudaMemcpyAsync(pX, B, bytes, cudaMemcpyDeviceToHost);
    cudaEventRecord(ev.b);
    cudaEventSynchronize(ev.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (i >= warmup) t.push_back(ms);
  }
  int rc = finish();
  cudaFree(A);
  cudaFree(T);
  cudaFree(B);
  cudaFree(C);
  cudaFree(ws);
  cudaFree(wt);
  cudaFreeHost(pA);
  cudaFreeHost(pT);
  cudaFreeHost(pB);
  cudaFreeHost(pC);
  cudaFreeHost(pX);
  return rc ? -1.0 : median(t);
}
}  // extern "C"

extern "C" {
// Median device time (ms) of one cuBLAS DSYRK (lower, 'N', alpha = 1,
// beta = 0) on device-resident inputs: the plain native-FP64 routine beside
// the reference's tc_ozimmu_syrk recursion, for the FP64 comparison.
double ref_time_cublas_dsyrk(long n, long k, const double* hA, int warmup, int iters) {
  double* A = up(hA, (size_t)n * k);
  double* C = up<double>(nullptr, (size_t)n * n);
  if (!A || !C) return -1.0;
  const double one = 1.0, zero = 0.0;
  Events ev;
  std::vector<float> t;
  for (int i = 0; i < warmup + iters; ++i) {
    cudaEventRecord(ev.a);
    cublasDsyrk(handle(), CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, (int)n, (int)k, &one, A, (int)n, &zero, C, (int)n);
    cudaEventRecord(ev.b);
    cudaEventSynchronize(ev.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.a, ev.b);
    if (i >= warmup) t.push_back(ms);
  }
  int rc = finish();
  cudaFree(A);
  cudaFree(C);
  return rc ? -1.0 : median(t);
}
}  // extern "C"
