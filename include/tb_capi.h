/*
 * tb_capi.h — plain C ABI of the B200 TensorBLAS library (libTensorBLAS.so).
 *
 * Every entry point takes raw device pointers to column-major matrices and
 * plain integers, returns a tb_status, and runs asynchronously on the stream
 * set with tb_set_stream (default: the legacy default stream). No torch or
 * cuBLAS types appear here; ctypes, cgo or any FFI can bind it directly.
 *
 * Each function names the reference interface it replaces
 * (Orgline/Tensor-BLAS, paths relative to that project).
 */
#ifndef TB_CAPI_H_
#define TB_CAPI_H_

#ifdef __cplusplus
extern "C" {
#endif

#define TB_API __attribute__((visibility("default")))

typedef enum {
  TB_SUCCESS = 0,
  TB_ERROR_INVALID_VALUE = 1, /* bad size, stride, flag or pointer */
  TB_ERROR_ALLOC = 2,         /* device scratch could not be allocated */
  TB_ERROR_CUDA = 3,          /* a CUDA runtime/driver call failed */
  TB_ERROR_TIMEOUT = 4,       /* a bounded device-side wait gave up */
  TB_ERROR_NOT_SUPPORTED = 5  /* no sm_100 device / unsupported option */
} tb_status;

typedef enum {
  /* FP16 operands, FP32 accumulation: the reference's plain tc_* form. */
  TB_PREC_PLAIN = 0,
  /* FP16 hi + scaled-lo split of both operands, 3 tensor-core products with
   * the correction in a separate FP32 accumulator: FP32-level accuracy (the
   * role of the reference's tc_cumpsgemm_* / CUMPSGEMM_FP16TCEC). */
  TB_PREC_SPLIT = 1,
  /* e4m3 operands scaled per 128 x 128 block, FP32 accumulation (normwise
   * error ~1e-2 on wide-range data): SYRK, SYR2K, TRMM, SYMM and GEMM only. */
  TB_PREC_FP8 = 2,
  /* TRSM only: plain solve plus one refinement sweep (residual with the
   * split products, correction with a second plain solve): FP32-level
   * accuracy from the FP16 path. */
  TB_PREC_REFINE = 3
} tb_precision;

/* Library/stream control. `stream` is a cudaStream_t (NULL = default). */
TB_API tb_status tb_set_stream(void* stream);
TB_API void* tb_get_stream(void);
TB_API const char* tb_status_string(tb_status s);
/* Text of the last error recorded on the calling thread ("" if none). */
TB_API const char* tb_last_error(void);
/* Blocks until queued work finishes; returns TB_ERROR_TIMEOUT if a kernel
 * reported a bounded-wait timeout, TB_ERROR_CUDA on a CUDA error. */
TB_API tb_status tb_synchronize(void);
TB_API int tb_version(void);
/* Number of kernels this library has launched in this process. */
TB_API unsigned long long tb_launch_count(void);
/* Number of device allocations (cudaMalloc) this library has made in this
 * process: scratch pool growth, cached tile lists, error blocks, batches and
 * autotuner trial outputs (no reference counterpart; a diagnostic). */
TB_API unsigned long long tb_alloc_count(void);
/* Waits for the device, then frees the library's scratch pool and cached
 * device tile lists on the current device (no reference counterpart: the
 * reference's wrappers malloc and free per call). The next routine call
 * allocates again. Batches keep their own memory until tb_batch_destroy. */
TB_API tb_status tb_release_scratch(void);
/* Test hook of the failure path (no reference counterpart). From now on the
 * GEMM kernels' producers skip the operand loads of tile `tile` of every
 * launch (-1: none), and every bounded device wait gives up after `wait_ns`
 * ns (0: the default of 4 s): a launch that reaches that tile stops with its
 * output partly written and tb_synchronize returns TB_ERROR_TIMEOUT, while
 * the context stays usable. tb_debug_stall(-1, 0) restores normal
 * operation. Not for production use. */
TB_API tb_status tb_debug_stall(long tile, unsigned long long wait_ns);
/* Host-only check of the task plan the persistent TRSM solve would use for
 * tb_strsm(side, m, n, ..., nb, precision) (no reference counterpart; no
 * device memory is touched): every tile and counter index in range and the
 * claim order topological, so that no task can wait for a later one.
 * stats[4] receives {tasks, counters, ops, simulated makespan in cost
 * units}; TB_ERROR_INVALID_VALUE and the reason in tb_last_error if the
 * plan is not valid. */
TB_API tb_status tb_debug_trsm_plan(char side, long m, long n, long nb, int precision, long* stats);
/* Event timing of every GEMM-engine launch between begin and end (events on
 * the launching stream): device ms during which at least one of them ran (the
 * union of their intervals: launches on two streams may overlap), total
 * algorithmic flops, launches. */
TB_API tb_status tb_profile_begin(void);
TB_API tb_status tb_profile_end(double* gemm_ms, double* gemm_flops, long* gemm_launches);
/* The launches of the last begin/end window by kernel: kind 0 the single-CTA
 * GEMM kernel, 1 the CTA-pair GEMM kernel, 2 the persistent TRSM kernel, 3
 * the Ozaki INT8 kernels. Device ms during which at least one launch of that
 * kernel ran (the union of their intervals), their algorithmic flops, their
 * algorithmic DRAM bytes (GEMM kernels: operands once, C read when beta != 0
 * and written, FP16 side copies; 0 for the others) and their number. */
TB_API tb_status tb_profile_kernel(int kind, double* ms, double* flops, double* bytes, long* launches);

/*
 * GEMM: C = alpha * op(A) * op(B) + beta * C, op(A) m x k, op(B) k x n, all
 * FP32 in memory, products on the tensor cores at `precision`.
 * Replaces the cublasGemmEx(CUDA_R_16F in, CUDA_R_32F out) calls the
 * reference builds every routine from (e.g. BLAS/tc_syrk.cu:106-118) and the
 * FP16 GEMM of testing/testing_gemm.cu:62-130.
 */
TB_API tb_status tb_sgemm(char transa, char transb, long m, long n, long k, float alpha, const float* A, long lda,
                          const float* B, long ldb, float beta, float* C, long ldc, int precision);

/*
 * SYRK: C = alpha * op(A) * op(A)^T + beta * C, the `uplo` triangle of C
 * ('L' lower, 'U' upper, diagonal included) written; the other strict
 * triangle is left untouched.
 *   trans 'N': A is n x k (lda >= n).   trans 'T': A is k x n (lda >= k).
 * Replaces tc_syrk (BLAS/tc_syrk.cu:126-157, include/TensorBLAS.h:139) and,
 * with TB_PREC_SPLIT, tc_cumpsgemm_syrk (BLAS/tc_cumpsgemm_syrk.cu:3-125).
 * nb is the recursion block of the reference method (> 0).
 */
TB_API tb_status tb_ssyrk(char uplo, char trans, long n, long k, float alpha, const float* A, long lda, float beta,
                          float* C, long ldc, long nb, int precision);

/*
 * nb = TB_NB_AUTO in tb_ssyrk, tb_strsm, tb_ssyr2k and tb_strmm: the
 * library's autotuner picks nb (the TRSM leaf size: 128, 256 or 512) and the
 * GEMM engine, i.e. the tile shape and cluster size of the large plain
 * launches (engine 1: 256 x 256 tiles on CTA pairs; 0: single-CTA 128 x 256
 * tiles; 2: single-CTA 128 x 128 tiles, a candidate in plain precision only)
 * for this (routine, flags, sizes, precision). The first call with a new key times
 * each candidate once on zero-filled scratch outputs of the same shape, on
 * the library's current stream, and caches the fastest per device; the call
 * then runs with it. The cache lives in memory and, when a file is set
 * (tb_autotune_set_file, or TB_AUTOTUNE_CACHE in the environment), is loaded
 * from that file and rewritten to it (temporary file + rename) on every new
 * entry. Keys carry the device name, compute capability and driver version.
 */
#define TB_NB_AUTO (-1L)
TB_API tb_status tb_autotune_set_file(const char* path); /* NULL: memory only */
TB_API tb_status tb_autotune_clear(void);                /* forget every entry (the file is kept) */
TB_API int tb_autotune_entries(void);
/* routine: "ssyrk" (flags uplo+trans, a = n, b = k), "strsm" (flags side,
 * a = m, b = n), "ssyr2k" (uplo+trans, n, k), "strmm" (uplo, m, n).
 * engine: 0, 1 or 2 as above (others: TB_ERROR_INVALID_VALUE); an entry put
 * here drives later TB_NB_AUTO calls of that key.
 * tb_autotune_get returns TB_ERROR_NOT_SUPPORTED when there is no entry. */
TB_API tb_status tb_autotune_put(const char* routine, const char* flags, long a, long b, int precision, long nb,
                                 int engine, double ms);
TB_API tb_status tb_autotune_get(const char* routine, const char* flags, long a, long b, int precision, long* nb,
                                 int* engine);
/* The same with the split-K count of a plain 'N' SYRK (1: one pass). */
TB_API tb_status tb_autotune_put_ex(const char* routine, const char* flags, long a, long b, int precision, long nb,
                                    int engine, int splitk, double ms);
TB_API tb_status tb_autotune_get_ex(const char* routine, const char* flags, long a, long b, int precision, long* nb,
                                    int* engine, int* splitk);

/*
 * TRSM with a lower-triangular, non-unit A, B overwritten by X:
 *   side 'R': X * A^T = B,  A n x n, B m x n  (the reference's tc_trsm:
 *             BLAS/tc_trsm.cu:139-174, right/lower/transpose/non-unit)
 *   side 'L': A * X = B,    A m x m, B m x n  (left/lower/no-trans)
 * Replaces tc_trsm (include/TensorBLAS.h:147) and, with TB_PREC_SPLIT,
 * tc_cumpsgemm_trsm (BLAS/tc_cumpsgemm_trsm.cu:3-126).
 * In plain precision, when B has at least 4096 independent columns (left)
 * or rows (right), the two halves are solved on the library's stream and
 * on an internal second stream of the same device, which is joined back
 * into the library's stream (event wait) before the call returns: work
 * queued afterwards on that stream sees the whole result.
 */
TB_API tb_status tb_strsm(char side, long m, long n, const float* A, long lda, float* B, long ldb, long nb,
                          int precision);

/*
 * General TRSM, B overwritten by X, BLAS flag meanings (no single reference
 * counterpart: the reference solves right/lower/transpose/non-unit only):
 *   side 'L': op(A) X = B, A m x m;   side 'R': X op(A) = B, A n x n
 *   uplo 'L'/'U': the triangle of A that is read; transa 'N'/'T': op(A) = A / A^T;
 *   diag 'N'/'U': stored or unit diagonal (a unit diagonal is never read).
 * The six forms other than left/lower/'N' and right/lower/'T' run on those
 * two through a remapped copy of A's triangle (transposed and/or order-
 * reversed) and, where the order is reversed, an in-place reversal of B's
 * rows (left) or columns (right) around the solve.
 */
TB_API tb_status tb_strsm_ex(char side, char uplo, char transa, char diag, long m, long n, const float* A, long lda,
                             float* B, long ldb, long nb, int precision);

/*
 * SYR2K: C = alpha (A B^T + B A^T) + beta C, lower triangle written, A and B
 * n x k (trans 'N'). Replaces tc_syr2k (BLAS/tc_syr2k.cu:116-152) and, with
 * TB_PREC_SPLIT, tc_cumpsgemm_syr2k (BLAS/tc_cumpsgemm_syr2k.cu).
 */
TB_API tb_status tb_ssyr2k(char uplo, char trans, long n, long k, float alpha, const float* A, long lda,
                           const float* B, long ldb, float beta, float* C, long ldc, long nb, int precision);

/*
 * TRMM (left, out of place): C = alpha op(A) B, A m x m triangular ('L' lower
 * or 'U' upper; the other triangle is never read), B and C m x n.
 * Replaces tc_trmm (BLAS/tc_trmm.cu:99-135, lower) and tc_cumpsgemm_trmm.
 */
TB_API tb_status tb_strmm(char uplo, long m, long n, float alpha, const float* A, long lda, const float* B, long ldb,
                          float* C, long ldc, long nb, int precision);

/*
 * General TRMM, out of place, BLAS flag meanings (no single reference
 * counterpart: the reference has left/lower/no-trans/non-unit only):
 *   side 'L': C = alpha op(A) B, A m x m;   side 'R': C = alpha B op(A), A n x n
 *   uplo 'L'/'U': the triangle of A that is read; transa 'N'/'T': op(A) = A / A^T;
 *   diag 'N'/'U': stored or unit diagonal. B and C are m x n.
 */
TB_API tb_status tb_strmm_ex(char side, char uplo, char transa, char diag, long m, long n, float alpha,
                             const float* A, long lda, const float* B, long ldb, float* C, long ldc, int precision);

/*
 * SYMM (left): C = alpha A B + beta C, A m x m symmetric with triangle `uplo`
 * stored; A is not modified. Replaces tc_symm (BLAS/tc_symm.cu:3-19) and
 * tc_cumpsgemm_symm (BLAS/tc_cumpsgemm_symm.cu).
 */
TB_API tb_status tb_ssymm(char uplo, long m, long n, float alpha, const float* A, long lda, const float* B, long ldb,
                          float beta, float* C, long ldc, int precision);

/*
 * Host-memory forms (no single reference counterpart: the reference's
 * callers copy whole operands to the device around tc_syrk / tc_trsm, e.g.
 * python/TensorBLAS.py:11-68, testing/testing_syrk.cu). A, B and C are host
 * pointers (page-locked memory gives full PCIe speed; pageable memory works
 * but its copies do not overlap). The call streams them through device
 * staging buffers in panels, overlapping host->device copies, the tensor-core
 * work and device->host copies on two internal copy streams; only the
 * referenced triangle of A (TRSM) and of C (SYRK) crosses the bus. Arguments
 * and results are those of tb_ssyrk ('L', 'N'; k > 0, alpha != 0) and
 * tb_strsm. Synchronous: returns when the results are in host memory.
 */
TB_API tb_status tb_ssyrk_host(char uplo, char trans, long n, long k, float alpha, const float* A, long lda,
                               float beta, float* C, long ldc, long nb, int precision);
TB_API tb_status tb_strsm_host(char side, long m, long n, const float* A, long lda, float* B, long ldb, long nb,
                               int precision);

/*
 * tb_ssyrk_noalloc: tb_ssyrk for callers that cannot allocate device memory
 * (no counterpart in the reference library). Arguments and results as
 * tb_ssyrk, but every byte of scratch comes from one static 64 MiB device
 * array compiled into the library, so the call makes no cudaMalloc/cudaFree.
 * It is meant for callers whose GPU memory is owned by another allocator
 * (e.g. a framework's caching allocator holding nearly all HBM) and for
 * latency-critical code that cannot absorb the device-wide synchronisation
 * cudaMalloc/cudaFree imply. Limits: the tile list plus the FP16 copy of A
 * (round_up(rows, 64) * cols * 2 bytes, twice that for TB_PREC_SPLIT) must
 * fit in 64 MiB, else TB_ERROR_INVALID_VALUE with the size in tb_last_error;
 * precision TB_PREC_PLAIN or TB_PREC_SPLIT only (TB_PREC_FP8 is rejected)
 * and nb > 0 (TB_NB_AUTO is rejected). k == 0 or alpha == 0 only scales C.
 * The first call on a device looks up the array's address; make it before
 * any stream capture. All calls share the array: calls that overlap on the
 * GPU race and must be serialised by the caller. A device-side wait that
 * runs out is reported by tb_synchronize (TB_ERROR_TIMEOUT), which reads
 * the call's own static error block and allocates nothing.
 */
TB_API tb_status tb_ssyrk_noalloc(char uplo, char trans, long n, long k, float alpha, const float* A, long lda,
                                  float beta, float* C, long ldc, long nb, int precision);

/*
 * FP64 routines on the INT8 tensor cores (Ozaki scheme). Each operand row is
 * split into `slices` INT8 slices (1..14) under a per-row power-of-two
 * exponent; every slice-pair product is exact (INT32, K chunked so the level
 * sums cannot overflow), and the result is FP64-accurate once 7 * slices
 * exceeds 53 bits plus the in-row exponent spread. slices <= 0 selects the
 * count automatically (SYRK, SYR2K, TRMM): one pass over the operands
 * measures each row's spread d = e_max - log2(rms) in bits, and the count is
 * the smallest with 7 * slices >= 50 + max d, within [8, 14] (the call then
 * waits for that measurement); TRSM takes 10. The reference's tc_ozimmu_*
 * drivers run native FP64 cuBLAS GEMMs instead; the tc_ozimmu_* entry points
 * here use the automatic count (TRSM: 10).
 *
 * Scratch: the slice planes, plus each product's INT32 level sums
 * (4 * slices bytes per element of the output's bounding rectangle) when
 * they fit in 32 GB; the levels are then folded into C by a second kernel
 * (TB_OZ_FOLD=fused in the environment folds them inside the GEMM instead,
 * with the same results).
 *
 * SYRK: C = alpha op(A) op(A)^T + beta C, the `uplo` triangle ('L' or 'U');
 * A n x k ('N') or k x n ('T'). Replaces tc_ozimmu_syrk
 * (BLAS/tc_ozimmu_syrk.cu:108-143).
 */
TB_API tb_status tb_dsyrk_ozaki(char uplo, char trans, long n, long k, double alpha, const double* A, long lda,
                                double beta, double* C, long ldc, int slices);
/* SYR2K: C = alpha (A B^T + B A^T) + beta C, lower triangle, A and B n x k
 * (trans 'N'). Replaces tc_ozimmu_syr2k (BLAS/tc_ozimmu_syr2k.cu:97-123). */
TB_API tb_status tb_dsyr2k_ozaki(char uplo, char trans, long n, long k, double alpha, const double* A, long lda,
                                 const double* B, long ldb, double beta, double* C, long ldc, int slices);
/* TRMM (left, out of place): C = alpha op(A) B, A m x m lower ('L') or upper
 * ('U'), the other triangle never read. Replaces tc_ozimmu_trmm
 * (BLAS/tc_ozimmu_trmm.cu:118-149, lower). */
TB_API tb_status tb_dtrmm_ozaki(char uplo, long m, long n, double alpha, const double* A, long lda, const double* B,
                                long ldb, double* C, long ldc, int slices);
/* TRSM, A lower-triangular non-unit, B overwritten by X:
 *   side 'R': X A^T = B (A n x n, B m x n; tc_ozimmu_trsm,
 *             BLAS/tc_ozimmu_trsm.cu:103-136)
 *   side 'L': A X = B   (A m x m)
 * Leaves of nb (<= 512) columns are multiplied by their FP64 inverses. */
TB_API tb_status tb_dtrsm_ozaki(char side, long m, long n, const double* A, long lda, double* B, long ldb, long nb,
                                int slices);
/* The slicing step alone: `slices` int8 planes Q[s][i][p] (row stride ldq,
 * plane stride n * ldq, ldq a multiple of 16 and >= k rounded up to 16) and
 * row exponents, exactly as tb_dsyrk_ozaki forms them. */
TB_API tb_status tb_ozaki_slice(long n, long k, const double* A, long lda, int slices, signed char* Q, long ldq,
                                int* exponents);
/* The exact INT32 level product P_L = sum_{s+t=L} Q_s Q_t^T (lower triangle,
 * column-major, ldp) that tb_dsyrk_ozaki folds into C, for checking. */
TB_API tb_status tb_ozaki_level_product(long n, long k, const double* A, long lda, int slices, int level, int* P,
                                        long ldp);

/*
 * Batched uneven instances (no reference counterpart: the reference loops
 * over tc_syrk / tc_trsm, BLAS/tc_syrk.cu:126-157, BLAS/tc_trsm.cu:139-174).
 * kind[i] = 0: SYRK, C_i(lower) = A_i A_i^T, A_i n_i x n_i, BC[i] = C_i.
 * kind[i] = 1: TRSM, X_i A_i^T = B_i (A_i lower n_i x n_i), BC[i] = B_i,
 *              overwritten by X_i (the reference's tc_trsm semantics).
 * tb_batch_create plans everything (scratch, FP16 copies' layout, tile lists,
 * per-problem descriptors); tb_batch_run enqueues a few grouped launches on
 * the current stream, allocates nothing and does not synchronise (it may be
 * captured in a CUDA graph); the pointers given at creation must stay valid.
 * nb: TRSM leaf-block cap (<= 0: 512); precision as elsewhere.
 */
typedef struct tb_batch_s* tb_batch_t;
TB_API tb_status tb_batch_create(tb_batch_t* batch, int count, const int* kind, const long* n, const float* const* A,
                                 const long* lda, float* const* BC, const long* ldbc, long nb, int precision);
TB_API tb_status tb_batch_run(tb_batch_t batch);
TB_API tb_status tb_batch_destroy(tb_batch_t batch);

/* FP32 -> FP16 conversion of an m x n column-major matrix, round to
 * nearest even: ah = fp16(as) (ldah), and when al is not NULL also the
 * scaled low half al = fp16((as - ah) * lo_scale) of the split form.
 * Replaces the reference's s2h / s2h_swpipe kernels (util/util.cu:127-136,
 * include/TensorBLAS.h:185-283); ah and al are __half arrays. */
TB_API tb_status tb_s2h(long m, long n, const float* as, long ldas, void* ah, long ldah, void* al, float lo_scale);
/* The same plain conversion (no low half) on the host's cores, host buffers
 * in and out: what tb_ssyrk_host does to A's row panels before they cross
 * PCIe. Round to nearest, ties to even, as the device conversion. */
TB_API tb_status tb_host_s2h(long m, long n, const float* as, long ldas, void* ah, long ldah);

/* Mirror lower -> upper of an n x n matrix (util/util.cu:148-157). */
TB_API tb_status tb_ssymmetrize(long n, float* A, long lda);

/* Reference C-ABI wrappers (include/TensorBLAS.h:135,137,145), same
 * argument meaning and return convention (0 ok, 1 error). */
TB_API int tc_syrk_wrapper(long n, long k, float* A, float* C, long nb);
TB_API int tc_trsm_wrapper(long m, long n, float* A, float* B, long nb);
TB_API void print_env(void);

#ifdef __cplusplus
}
#endif

#endif /* TB_CAPI_H_ */
