// Reference-facing entry points: the extern "C" wrappers the reference's
// python/TensorBLAS.py binds (BLAS/tc_syrk.cu:4-39, BLAS/tc_trsm.cu:4-28),
// print_env (util/util.cu:318-349) and the symmetrise helper
// (copy_lower_to_upper, util/util.cu:148-157).
#include <cstdio>

#include "tb_internal.h"

namespace tb {
namespace {

// Mirror the strict lower triangle into the upper one through 32x32 shared
// tiles so both the read of the lower tile and the write of the upper tile
// are coalesced (the reference's kernel reads with stride lda).
__global__ void __launch_bounds__(256) symmetrize_kernel(long long n, float* A, long long lda) {
  __shared__ float tile[32][33];
  const long long bi = blockIdx.x, bj = blockIdx.y;  // source tile (row block bi >= col block bj)
  if (bi < bj) return;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const long long i = bi * 32 + tx, j = bj * 32 + r;
    tile[r][tx] = (i < n && j < n) ? A[i + j * lda] : 0.f;
  }
  __syncthreads();
  // write upper element (j, i) = lower (i, j) for i > j
  for (int r = ty; r < 32; r += 8) {
    const long long row = bj * 32 + tx, col = bi * 32 + r;  // destination (row < col)
    if (row < n && col < n && row < col) A[row + col * lda] = tile[tx][r];
  }
}

}  // namespace

tb_status symmetrize_lower(long long n, float* A, long long lda, cudaStream_t st) {
  if (n <= 1) return TB_SUCCESS;
  const long long nt = (n + 31) / 32;
  if (nt > 65535) return TB_ERROR_NOT_SUPPORTED;
  dim3 grid((unsigned)nt, (unsigned)nt);
  symmetrize_kernel<<<grid, 256, 0, st>>>(n, A, lda);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

}  // namespace tb

extern "C" {

tb_status tb_ssymmetrize(long n, float* A, long lda) {
  if (n < 0 || lda < (n > 1 ? n : 1)) return TB_ERROR_INVALID_VALUE;
  return tb::symmetrize_lower(n, A, lda, tb::current_stream());
}

// BLAS/tc_syrk.cu:4-39: C = A A^T for the row-major n x k torch tensor A
// (column-major k x n in memory), full symmetric C, 0 on success / 1 on error.
// Like the reference's wrapper (whose cudaFree of its workspace waits for the
// device), it returns only once the result is complete: it synchronises the
// library's stream and reports a CUDA error or a device-side wait that ran
// out as 1.
int tc_syrk_wrapper(long n, long k, float* A, float* C, long nb) {
  tb_status s = tb_ssyrk('L', 'T', n, k, 1.0f, A, k > 1 ? k : 1, 0.0f, C, n > 1 ? n : 1, nb, TB_PREC_PLAIN);
  if (s == TB_SUCCESS) s = tb_ssymmetrize(n, C, n > 1 ? n : 1);
  if (s == TB_SUCCESS) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) s = tb::cuda_status(e);
  }
  if (s == TB_SUCCESS) s = tb_synchronize();
  if (s != TB_SUCCESS) {
    printf("TensorBLAS error: %s %s\n", tb_status_string(s), tb_last_error());
    return 1;
  }
  return 0;
}

// BLAS/tc_trsm.cu:4-28: X A^T = B, A n x n lower (lda = n), B m x n (ldb = m),
// B overwritten; 0 on success / 1 on error (synchronous, errors as in
// tc_syrk_wrapper).
int tc_trsm_wrapper(long m, long n, float* A, float* B, long nb) {
  tb_status s = tb_strsm('R', m, n, A, n > 1 ? n : 1, B, m > 1 ? m : 1, nb, TB_PREC_PLAIN);
  if (s == TB_SUCCESS) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) s = tb::cuda_status(e);
  }
  if (s == TB_SUCCESS) s = tb_synchronize();
  if (s != TB_SUCCESS) {
    printf("TensorBLAS error: %s %s\n", tb_status_string(s), tb_last_error());
    return 1;
  }
  return 0;
}

void print_env(void) {
  cudaDeviceProp prop;
  int dev = 0, rt = 0, drv = 0;
  cudaGetDevice(&dev);
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    printf("=== Device information ===\nno CUDA device\n=== END Device Information ===\n");
    return;
  }
  cudaRuntimeGetVersion(&rt);
  cudaDriverGetVersion(&drv);
  printf("=== Device information ===\n");
  printf("Device name: %s\n", prop.name);
  printf("Compute Capability: %d.%d\n", prop.major, prop.minor);
  printf("CUDA Runtime Version: %d\nCUDA Driver Version: %d\n", rt, drv);
  printf("GMem %zu\nSMem per block (opt-in) %zu\nSMem per MP %zu\n", prop.totalGlobalMem,
         prop.sharedMemPerBlockOptin, prop.sharedMemPerMultiprocessor);
  printf("Regs per block %d\nL2 $ size %d\n# MP %d\n", prop.regsPerBlock, prop.l2CacheSize,
         prop.multiProcessorCount);
  printf("=== END Device Information ===\n");
}

}  // extern "C"
