/*
 * TensorBLAS.h — source-compatible replacement of the reference library's
 * public header (Orgline/Tensor-BLAS include/TensorBLAS.h:135-171) for the
 * B200 (sm_100a) implementation in libTensorBLAS.so.
 *
 * Same routine names, parameter lists and semantics as the reference:
 * column-major FP32 (or FP64 for tc_ozimmu_*) device pointers, the FP16
 * workspace argument of the plain routines, void return. Differences that a
 * caller can observe are listed per routine. Status-returning C entry points
 * with explicit flags and precision live in tb_capi.h.
 *
 * Handles: the cuBLAS and cuMpSGEMM handles are accepted only for source
 * compatibility; nothing here calls cuBLAS or cuMpSGEMM. Work is queued on
 * the stream set with tb_set_stream (default: the legacy default stream,
 * which is also where the reference's handles run unless told otherwise).
 *
 * Workspace: the plain routines take the reference's FP16 workspace. When
 * it is too small for this implementation's layout (row-padded FP16 copies)
 * or NULL, a library-owned scratch buffer is used instead (grow-only, one per
 * device; calls that overlap on different streams must pass their own).
 */
#ifndef TENSORBLAS_B200_H_
#define TENSORBLAS_B200_H_

#include <cuda_fp16.h>

#include "tb_capi.h"

/* Opaque handle types with the reference's spelling. */
#ifndef CUBLAS_V2_H_
struct cublasContext;
typedef struct cublasContext* cublasHandle_t;
#endif
#ifndef TB_HAVE_CUMPSGEMM
namespace cumpsgemm {
struct handle_struct;
typedef handle_struct* handle_t;
}  // namespace cumpsgemm
#endif

/* include/TensorBLAS.h:139 — lower triangle of C = alpha A A^T + beta C,
 * A n x k (lda). Ah: FP16 workspace of n*k halves. Unlike the reference the
 * strict upper triangle of C is not written, odd n/k need no padding copies,
 * and beta is honoured for every size (reference: BLAS/tc_syrk.cu:140). */
TB_API void tc_syrk(cublasHandle_t handle, long int n, long int k, float alpha, float* A, long int lda, float beta,
                    float* C, long int ldc, __half* Ah, long int nb);

/* include/TensorBLAS.h:141 — FP32-accurate SYRK (split FP16 products). */
TB_API void tc_cumpsgemm_syrk(cumpsgemm::handle_t cumpsgemm_handle, long int n, long int k, float alpha, float* A,
                              long int lda, float beta, float* C, long int ldc, long int nb);

/* include/TensorBLAS.h:147 — X A^T = B (right, lower, transpose, non-unit),
 * B (m x n, ldb) overwritten; hwork: FP16 workspace. */
TB_API void tc_trsm(cublasHandle_t handle, long int m, long int n, float* A, long int lda, float* B, long int ldb,
                    __half* hwork, long int nb);

/* include/TensorBLAS.h:149 — FP32-accurate TRSM (split FP16 products). */
TB_API void tc_cumpsgemm_trsm(cublasHandle_t handle, cumpsgemm::handle_t cumpsgemm_handle, long int m, long int n,
                              float* A, long int lda, float* B, long int ldb, long int nb);

/* include/TensorBLAS.h:159 — lower triangle of C = alpha (A B^T + B A^T)
 * + beta C, A and B n x k. Ah: FP16 workspace (2 n k halves in the
 * reference; used when large enough for this layout). */
TB_API void tc_syr2k(cublasHandle_t handle, long int n, long int k, float alpha, float* A, long int lda, float* B,
                     long int ldb, float beta, float* C, long int ldc, __half* Ah, long int nb);

/* include/TensorBLAS.h:161 — FP32-accurate SYR2K. */
TB_API void tc_cumpsgemm_syr2k(cumpsgemm::handle_t cumpsgemm_handle, long int n, long int k, float alpha, float* A,
                               long int lda, float* B, long int ldb, float beta, float* C, long int ldc, long int nb);

/* include/TensorBLAS.h:153 — C = alpha A B, A m x m lower (left, out of
 * place). The strict upper triangle of A is ignored (the reference requires
 * it to be zero). */
TB_API void tc_trmm(cublasHandle_t handle, long int m, long int n, float alpha, float* A, long int lda, float* B,
                    long int ldb, float* C, long int ldc, __half* hwork, long int nb);

/* include/TensorBLAS.h:155 — FP32-accurate TRMM. */
TB_API void tc_cumpsgemm_trmm(cumpsgemm::handle_t cumpsgemm_handle, long int m, long int n, float alpha, float* A,
                              long int lda, float* B, long int ldb, float* C, long int ldc, long int nb);

/* include/TensorBLAS.h:165 — C = alpha A B + beta C, A symmetric with its
 * lower triangle stored (left). Unlike the reference, A is not modified. */
TB_API void tc_symm(cublasHandle_t handle, long int m, long int n, float alpha, float* A, long int lda, float* B,
                    int ldb, float beta, float* C, long int ldc, __half* Ah);

/* include/TensorBLAS.h:167 — FP32-accurate SYMM. */
TB_API void tc_cumpsgemm_symm(cumpsgemm::handle_t cumpsgemm_handle, long int m, long int n, float alpha, float* A,
                              long int lda, float* B, int ldb, float beta, float* C, long int ldc);

/* include/TensorBLAS.h:143 — FP64 SYRK, here on the INT8 tensor cores
 * (Ozaki scheme, 10 slices; see tb_dsyrk_ozaki). nb is accepted and unused. */
TB_API void tc_ozimmu_syrk(cublasHandle_t handle, long int n, long int k, double alpha, double* A, long int lda,
                           double beta, double* C, long int ldc, long int nb);

/* include/TensorBLAS.h:151 — FP64 TRSM X A^T = B (right/lower/transpose/
 * non-unit), B overwritten; Ozaki-scheme updates and FP64 leaf inverses of
 * nb (<= 512) columns (see tb_dtrsm_ozaki). */
TB_API void tc_ozimmu_trsm(cublasHandle_t handle, long int m, long int n, double* A, long int lda, double* B,
                           long int ldb, long int nb);

/* include/TensorBLAS.h:157 — FP64 TRMM C = alpha A B, A lower, left side,
 * out of place; the strict upper triangle of A is never read (see
 * tb_dtrmm_ozaki). nb is accepted and unused. */
TB_API void tc_ozimmu_trmm(cublasHandle_t handle, long int m, long int n, double alpha, double* A, long int lda,
                           double* B, long int ldb, double* C, long int ldc, long int nb);

/* include/TensorBLAS.h:163 — FP64 SYR2K, lower triangle of
 * alpha (A B^T + B A^T) + beta C (see tb_dsyr2k_ozaki). nb is accepted and
 * unused. */
TB_API void tc_ozimmu_syr2k(cublasHandle_t handle, long int n, long int k, double alpha, double* A, long int lda,
                            double* B, long int ldb, double beta, double* C, long int ldc, long int nb);

#endif /* TENSORBLAS_B200_H_ */
