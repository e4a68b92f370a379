// Declaration-only stand-in for the un-vendored cuMpSGEMM header, so that the
// reference's include/TensorBLAS.h (which includes <cumpsgemm/cumpsgemm.hpp>
// unconditionally) compiles. It declares the API shapes the reference's call
// sites use (BLAS/tc_cumpsgemm_*.cu) and nothing else; the tc_cumpsgemm_*
// sources are not compiled into oracle/_ref, so none of this is ever linked.
#pragma once
#include <cublas_v2.h>

#include <cstdint>

enum cuMpSGEMM_compute_mode_t {
  CUMPSGEMM_AUTO = 0,
  CUMPSGEMM_FP16TCEC,
  CUMPSGEMM_FP16TC,
  CUMPSGEMM_TF32TCEC,
  CUMPSGEMM_TF32TC,
  CUMPSGEMM_FP32_SIMT
};

namespace cumpsgemm {
struct handle_struct;
typedef handle_struct* handle_t;
void create(handle_t& handle);
template <class T>
cublasStatus_t gemm(handle_t handle, cublasOperation_t op_A, cublasOperation_t op_B, uint64_t m, uint64_t n,
                    uint64_t k, const T* alpha, const T* a_ptr, uint64_t lda, const T* b_ptr, uint64_t ldb,
                    const T* beta, T* c_ptr, uint64_t ldc, cuMpSGEMM_compute_mode_t mode);
template <class T>
cublasStatus_t gemm_stridedBatch(handle_t handle, cublasOperation_t op_A, cublasOperation_t op_B, uint64_t m,
                                 uint64_t n, uint64_t k, const T* alpha, const T* a_ptr, uint64_t lda,
                                 uint64_t stridea, const T* b_ptr, uint64_t ldb, uint64_t strideb, const T* beta,
                                 T* c_ptr, uint64_t ldc, uint64_t stridec, uint64_t batch_count,
                                 cuMpSGEMM_compute_mode_t mode);
}  // namespace cumpsgemm
