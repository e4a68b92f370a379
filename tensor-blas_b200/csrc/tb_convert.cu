// FP32 -> FP16 conversion kernels (the reference's s2h / s2h_swpipe /
// s2hTranspose family, include/TensorBLAS.h:185-283 and util/util.cu:127-145),
// re-done for HBM3e: 8 elements per thread, two 128-bit loads and one (hi) or
// two (hi+lo) 128-bit stores, 64-bit indexing, grid sized in SM multiples.
// Round-to-nearest-even as __float2half in the reference.
//
// The split form writes hi = fp16(x) and lo = fp16((x - hi) * lo_scale), the
// error-corrected FP16 pair of Ootomo & Yokota (IJHPCA 2022).
#include <algorithm>
#include "tb_convert.cuh"
#include "tb_internal.h"

namespace tb {

namespace {

// Vector path: rows % 8 == 0, lds % 4 == 0, ldd % 8 == 0, 16-byte aligned bases.
__global__ void __launch_bounds__(256) convert8_kernel(long long rows, long long cols, const float* __restrict__ src,
                                                       long long lds, __half* __restrict__ hi, __half* __restrict__ lo,
                                                       long long ldd, float lo_scale, int tri, long long dup) {
  conv::convert8_body(blockIdx.x, gridDim.x, blockIdx.y, gridDim.y, rows, cols, src, lds, hi, lo, ldd, lo_scale, tri,
                      dup);
}

// Scalar fallback for ragged or unaligned shapes.
__global__ void __launch_bounds__(256) convert1_kernel(long long rows, long long cols, const float* __restrict__ src,
                                                       long long lds, __half* __restrict__ hi, __half* __restrict__ lo,
                                                       long long ldd, float lo_scale, int tri, long long dup) {
  conv::convert1_body(blockIdx.x, gridDim.x, blockIdx.y, gridDim.y, rows, cols, src, lds, hi, lo, ldd, lo_scale, tri,
                      dup);
}

// Full symmetric FP16 copy of an n x n matrix of which only one triangle is
// stored: out(i, j) = A(i, j) on the stored side, A(j, i) on the other. Each
// 32 x 32 output tile reads its own tile (stored side) or the mirrored one
// (other side; both for diagonal tiles) through shared memory, so every
// global read and write is coalesced and A is read about once (the
// reference instead mirrors the caller's A in place with strided reads,
// BLAS/tc_symm.cu:7).
__global__ void __launch_bounds__(256) convert_sym_kernel(long long n, const float* __restrict__ A, long long lda,
                                                          int lower, __half* __restrict__ hi, __half* __restrict__ lo,
                                                          long long ldd, float lo_scale) {
  __shared__ float own[32][33], mir[32][33];
  const long long bi = blockIdx.x, bj = blockIdx.y;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const bool need_own = lower ? bi >= bj : bi <= bj;  // the tile has elements on the stored side
  const bool need_mir = lower ? bi <= bj : bi >= bj;  // ... and on the other side
  for (int r = ty; r < 32; r += 8) {
    const long long i = bi * 32 + tx, j = bj * 32 + r;  // own tile element (i, j)
    if (need_own) own[r][tx] = (i < n && j < n) ? A[i + j * lda] : 0.f;
    const long long mi = bj * 32 + tx, mj = bi * 32 + r;  // mirrored tile element (mi, mj)
    if (need_mir) mir[r][tx] = (mi < n && mj < n) ? A[mi + mj * lda] : 0.f;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const long long i = bi * 32 + tx, j = bj * 32 + r;
    if (i >= n || j >= n) continue;
    const bool stored = lower ? (i >= j) : (i <= j);
    const float f = stored ? own[r][tx] : mir[tx][r];  // mir[tx][r] = A(j, i)
    const __half h = __float2half_rn(f);
    hi[i + j * ldd] = h;
    if (lo) lo[i + j * ldd] = __float2half_rn((f - __half2float(h)) * lo_scale);
  }
}

}  // namespace

tb_status convert_sym_f32_f16(long long n, const float* A, long long lda, bool lower, __half* hi, __half* lo,
                              long long ldd, float lo_scale, cudaStream_t stream) {
  if (n <= 0) return TB_SUCCESS;
  const long long nt = (n + 31) / 32;
  if (nt > 65535) return TB_ERROR_NOT_SUPPORTED;
  convert_sym_kernel<<<dim3((unsigned)nt, (unsigned)nt), 256, 0, stream>>>(n, A, lda, lower ? 1 : 0, hi, lo, ldd,
                                                                           lo_scale);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

tb_status convert_f32_f16(long long rows, long long cols, const float* src, long long lds, __half* hi, __half* lo,
                          long long ldd, float lo_scale, int tri, cudaStream_t stream, long long dup) {
  if (rows <= 0 || cols <= 0) return TB_SUCCESS;
  const bool vec = (rows % 8 == 0) && (lds % 4 == 0) && (ldd % 8 == 0) &&
                   (reinterpret_cast<uintptr_t>(src) % 16 == 0) && (reinterpret_cast<uintptr_t>(hi) % 16 == 0) &&
                   (lo == nullptr || reinterpret_cast<uintptr_t>(lo) % 16 == 0);
  const int threads = 256;
  long long gx = 0, gy = 0;
  conv::convert_grid(rows, cols, tri, vec, sm_count(), threads, &gx, &gy);
  dim3 grid((unsigned)gx, (unsigned)gy);
  if (vec)
    convert8_kernel<<<grid, threads, 0, stream>>>(rows, cols, src, lds, hi, lo, ldd, lo_scale, tri, dup);
  else
    convert1_kernel<<<grid, threads, 0, stream>>>(rows, cols, src, lds, hi, lo, ldd, lo_scale, tri, dup);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

namespace {
__global__ void unit_diag_kernel(long long n, __half* hi, __half* lo, long long ld) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  hi[i + i * ld] = __float2half_rn(1.f);
  if (lo) lo[i + i * ld] = __float2half_rn(0.f);
}
}  // namespace

// Unit diagonal in an FP16 copy (hi = 1, lo = 0) for diag = 'U' operands.
tb_status set_unit_diag(long long n, __half* hi, __half* lo, long long ld, cudaStream_t stream) {
  if (n <= 0) return TB_SUCCESS;
  unit_diag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(n, hi, lo, ld);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

}  // namespace tb

// The conversion as an entry point of its own: the reference's s2h
// (util/util.cu:127-136; the FP32 -> FP16 step of every routine), with the
// optional scaled-lo half of the split form.
extern "C" tb_status tb_s2h(long m, long n, const float* as, long ldas, void* ah, long ldah, void* al,
                            float lo_scale) {
  if (m < 0 || n < 0 || ldas < (m > 1 ? m : 1) || ldah < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  if (!as || !ah) return TB_ERROR_INVALID_VALUE;
  return tb::convert_f32_f16(m, n, as, ldas, static_cast<__half*>(ah), static_cast<__half*>(al), ldah, lo_scale, 0,
                             tb::current_stream());
}
