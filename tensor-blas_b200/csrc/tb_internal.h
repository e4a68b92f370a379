// Internal host-side interfaces shared by the routine drivers.
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/tb_capi.h"

namespace tb {

// ------------------------------------------------------------------ status
#define TB_CUDA_TRY(expr)                              \
  do {                                                 \
    cudaError_t e_ = (expr);                           \
    if (e_ != cudaSuccess) return tb::cuda_status(e_); \
  } while (0)
#define TB_TRY(expr)                       \
  do {                                     \
    tb_status s_ = (expr);                 \
    if (s_ != TB_SUCCESS) return s_;       \
  } while (0)

tb_status cuda_status(cudaError_t e);
void set_last_error(const char* fmt, ...);

// ------------------------------------------------------------------ streams / pool
cudaStream_t current_stream();
// More (non-blocking) streams per device (i = 0 .. kAuxStreams - 1) for work
// the library splits; joined back into the caller's stream before a routine
// returns.
constexpr int kAuxStreams = 4;
cudaStream_t aux_stream(int i = 0);
// Device scratch owned by the library (grow-only, per device and slot).
// Slot 0 serves the routines' own scratch; slot 1 the host-memory entry
// points' staging buffers, which live across routine calls; slot 2 the Ozaki
// engine's per-level INT32 sums; slot 3 the persistent TRSM solve's per-leaf
// operand copies, progress counters and op descriptors. Returns nullptr on
// allocation failure. Growing synchronises the device.
constexpr int kPoolSlots = 4;
void* pool_get(size_t bytes, int slot = 0);
// Bytes currently held by a pool slot of the current device.
size_t pool_capacity(int slot);
// Device error block used by bounded waits inside kernels (per device):
// kErrBlockInts ints, word 0 the error code (layout in tb_ptx.cuh).
constexpr int kErrBlockInts = 4;
int* device_error_word();
// A second error block of the current device (the allocation-free entry
// point's static one), read by check_device_error alongside the library's.
void register_error_block(int* block);
// Synchronises `stream`, then reads and clears the error code of every error
// block of the current device that exists; creates none (allocates nothing).
tb_status check_device_error(cudaStream_t stream);
// cudaMalloc, counted (tb_alloc_count): every device allocation the library
// makes goes through here.
cudaError_t dev_malloc(void** p, size_t bytes);
// Frees the scratch pool slots / the cached device tile lists of the
// current device (tb_release_scratch; the device must be idle).
void release_pool();
void release_tile_cache();
// Free device memory of the current device (cudaMemGetInfo), 0 on error.
size_t free_device_bytes();
int sm_count();
// Counts kernel launches issued by the library (tb_launch_count).
void note_launch(int n = 1);
// Event timing of GEMM-engine launches between tb_profile_begin/end, by
// kernel (the kinds of tb_profile_kernel).
enum ProfKind { kProfGemm = 0, kProfPair = 1, kProfDag = 2, kProfOzaki = 3, kProfKinds = 4 };
bool profiling();
void* prof_begin(cudaStream_t st, ProfKind kind);
void prof_end(void* token, cudaStream_t st, double flops, double bytes = 0);

inline long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

// ------------------------------------------------------------------ operands
// An fp16/bf16 matrix operand in global memory, indexed (row, k):
//   mn_major: element (r, k) at ptr[r + k * ld]  (rows contiguous)
//   k-major : element (r, k) at ptr[k + r * ld]  (k contiguous)
struct Operand {
  const void* ptr = nullptr;
  long long rows = 0;
  long long cols = 0;  // K extent
  long long ld = 0;
  bool mn_major = true;
};

enum class Split { kPlain = 1, kHiLo = 3 };

// Split products: K-blocks (of 64) the tensor core accumulates in TMEM
// between two round-to-nearest folds into FP32 registers (its own FP32
// accumulation truncates): 4 unless TB_SPLIT_KCHUNK (1..64) is set in the
// environment (read once).
int split_kchunk();

struct GemmCall {
  Operand a_hi, a_lo, b_hi, b_lo;  // lo used in kHiLo only
  Split split = Split::kPlain;
  int a_off = 0, b_off = 0, k_off = 0;
  const int4* tiles = nullptr;  // device tile list
  int num_tiles = 0;
  float* C = nullptr;
  long long ldc = 0;
  int M = 0, N = 0;
  float alpha = 1.f, beta = 0.f;
  int tri = 0, diag = 0;
  float corr_scale = 1.0f / 2048.0f;
  int kchunk = split_kchunk();  // split mode: K-blocks (64) per round-to-nearest fold
  __half* out_hi = nullptr;
  __half* out_lo = nullptr;
  long long ld_out = 0;
  float out_lo_scale = 2048.0f;
  int out_m = -1, out_n = -1;  // side-copy region (default: all of C)
  int kblocks = 0;   // most K-blocks (64) of any tile; 0 < kblocks <= kGemmPfMaxKb selects the prefetch variants
  const int* ranges = nullptr;  // per-CTA tile ranges of a balanced list (set by gemm_launch_plan)
  // FP8 (e4m3) operands: K-major byte matrices (Operand.ld in bytes), K
  // blocks of 128, per-(128-row block, K block) scales (row-block-major,
  // scale_ld K blocks per row block); tiles 128 x 128.
  bool pair = false;  // set by gemm_launch_plan: 256 x 256 tiles on CTA pairs (cta_group::2)
  bool fp8 = false;
  const float* scale_a = nullptr;
  const float* scale_b = nullptr;
  int scale_ld = 0;
  double flops = 0;  // algorithmic flops of this launch (profiling only)
  int* err = nullptr;  // device error word (nullptr: the library's per-device word)
};

// Tile width along N used by the engine for a given split mode (and, with
// kblocks = the most K-blocks of any tile, for the prefetch variants that
// launches with short K ranges use: plain tiles are then 128 wide).
constexpr int kGemmBM = 128;
constexpr int kGemmBK = 64;
constexpr int kGemmPfMaxKb = 16;
constexpr int kGemmBNFp8 = 128;  // FP8 tiles: 128 x 128, K blocks of 128
int gemm_bn(Split s);
int gemm_bn(Split s, int kblocks);

tb_status gemm_launch(const GemmCall& call, cudaStream_t stream);
// GEMM engine for the large plain launches of this thread: -1 the default
// (CTA pairs unless TB_GEMM_PAIR=0), 0 single-CTA 128 x 256 tiles, 1 CTA
// pairs (256 x 256), 2 single-CTA 128 x 128 tiles (kEngineNarrow: twice the
// tiles of engine 0, for launches whose 128 x 256 tiles leave SMs idle).
// The override also sets the tile width that gemm_bn(split, kblocks) gives
// the plans of plain long-K launches, so plan and kernel agree.
constexpr int kEngineNarrow = 2;
void set_engine_override(int engine);
int engine_override();
struct EngineScope {
  int saved;
  explicit EngineScope(int engine) : saved(engine_override()) { set_engine_override(engine); }
  ~EngineScope() { set_engine_override(saved); }
};
// Uploads `plan` (128-row tiles) and launches; plain launches that are large
// enough run on CTA pairs, with the plan merged into 256-row tiles.
tb_status gemm_launch_plan(GemmCall& call, const std::vector<int4>& plan, cudaStream_t stream);

// Grouped launches: each problem's descriptor is built on the host by
// gemm_build_args (tensor maps included), copied to a 64-byte aligned device
// array, and every tile carries the index of its problem. d_sched: a zeroed
// device counter selects the device-side tile scheduler (CTAs claim tiles
// in list order as they free up); nullptr keeps static striding.
struct GemmArgs;
tb_status gemm_build_args(const GemmCall& c, GemmArgs* out);
tb_status gemm_launch_grouped(Split split, const GemmArgs* d_problems, const int4* d_tiles, const int* d_tile_prob,
                              int num_tiles, double flops, cudaStream_t stream, int* d_sched = nullptr);

// Tile plans (host vectors of {m0, n0, kb_begin, kb_end}); uploaded and
// cached on the device by `upload_tiles`.
std::vector<int4> plan_rect(int M, int N, int bn, int kb0, int kb1);
std::vector<int4> plan_lower(int n, int bn, int kb0, int kb1);
std::vector<int4> plan_upper(int n, int bn, int kb0, int kb1);
const int4* upload_tiles(const std::vector<int4>& tiles, cudaStream_t stream);

// ------------------------------------------------------------------ conversion
// rows x cols column-major FP32 -> FP16 (bits) on the host's cores
// (tb_host_convert.cpp); round to nearest even, as __float2half_rn.
void host_f32_to_f16(const float* src, long lds, long rows, long cols, uint16_t* dst, long ldd);
// Frees the host-memory forms' page-locked staging (tb_release_scratch).
void release_host_staging();
// fp32 (rows x cols, column-major, lds) -> fp16 hi [and lo] with the same
// orientation (ldd). lo = fp16((x - hi) * lo_scale).
//   tri == 0: whole matrix; tri == 1: zero the strict upper triangle;
//   tri == 2: only rows i >= j (rounded down to 8) are written;
//   tri == 3: zero the strict lower triangle;
//   tri == 4: upper triangle, and zeros below the diagonal only in the rows
//             [j, (j / 256 + 1) * 256) of column j (nothing else is written);
//   tri == 5: lower triangle, and zeros above the diagonal only in the rows
//             [(j / 256) * 256, j) of column j (nothing else is written).
// Modes 4 / 5 serve products whose tiles (at most 256 rows, row-aligned to
// their height) take the K range from / up to their own diagonal block.
// dup != 0: the same values are also written `dup` elements further on (hi
// and lo alike), from one read of src.
tb_status convert_f32_f16(long long rows, long long cols, const float* src, long long lds, __half* hi, __half* lo,
                          long long ldd, float lo_scale, int tri, cudaStream_t stream, long long dup = 0);
// Unit diagonal in an FP16 copy (hi = 1, lo = 0) for diag = 'U' operands.
tb_status set_unit_diag(long long n, __half* hi, __half* lo, long long ld, cudaStream_t stream);
// ------------------------------------------------------------------ grouped TRSM pieces
// 32x32 diagonal-block inverses of one triangular matrix: sub-blocks
// [first, first + ceil(n/32)) of a grouped launch write D[0 ..].
struct DiagJob {
  const float* A;
  long long lda;
  long long n;
  double* D;
  long long first;
};
// One leaf inverse (rows/cols [s, s+size) of A) as FP16 hi/lo, column-major.
struct ChainJob {
  const float* A;
  long long lda;
  int s, size;
  const double* D;  // the instance's 32x32 inverses
  __half* Whi;
  __half* Wlo;
  long long ldw;
  double* Wg;  // FP64 working panels of the inverse (ldw x size)
};
tb_status trsm_inverses_grouped(const DiagJob* d_diag, int ndiag, long long nblocks, const ChainJob* d_chain,
                                int nchain, cudaStream_t st);
// FP64 inverses of the diagonal leaf blocks {s, size} (s a multiple of 32,
// size <= 512) of an FP64 lower-triangular matrix of order nt; W_b at
// W + b * wstride, leading dimension ldw. D: (nt + 31) / 32 * 1024 doubles.
tb_status trsm_leaf_inverses_f64(long nt, const double* A, long lda, const int2* d_leaves, int nleaf, int max_size,
                                 double* D, double* W, long long ldw, long long wstride, cudaStream_t st,
                                 bool unit = false);
// FP32 TRSM with its triangular operand prepared once (FP16 copy, leaf
// inverses) and applied to one or more right-hand-side blocks.
struct TrsmCtx {
  bool right;
  long m, n;  // B is m x n
  long nt;    // order of A (n for right, m for left)
  float* B;
  long ldb;
  Split split;
  int leaf;  // leaf block size (multiple of 64)
  // FP16 copies
  __half *ah, *al;  // A (nt x nt, MN-major, lda_h)
  long long lda_h;
  __half *xh, *xl;  // X: right: m x n col-major (ld ldx, MN-major operand)
                    //    left : m x n col-major (ld ldx, K-major operand, rows = n)
  long long ldx;
  __half *wh, *wl;  // per-leaf inverses (ldw x leaf each)
  long long ldw, wstride;
  __half *rh, *rl;  // current leaf block of B
  long long ldr;
  cudaStream_t st;
  // persistent solve (tb_trsm_dag.cu): per-leaf operand copies of B (slice b
  // holds leaf block b), progress counters, and whether the set-up launch
  // already wrote the first copy and zeroed the counters for B = dag_B
  __half *rfh = nullptr, *rfl = nullptr;
  long long ldrf = 0;
  int* dag_ctr = nullptr;
  const float* dag_B = nullptr;
  bool dag_prepped = false;
  // launch-per-product path: the set-up launch already wrote the first leaf's
  // operand copy (rh / rl) from the B it was given
  bool r0_ready = false;
};
// Jobs of the one-launch TRSM preparation (trsm_prep_launch, tb_trsm.cu).
struct PrepConv {  // fp32 rows x cols (lds) -> fp16 hi [lo] (ldd), triangle mode tri (convert_f32_f16)
  long long rows = 0, cols = 0;
  const float* src = nullptr;
  long long lds = 0;
  __half* hi = nullptr;
  __half* lo = nullptr;
  long long ldd = 0;
  int tri = 0;
};
struct PrepJobs {
  PrepConv conv[2];
  int nconv = 0;
  const float* A = nullptr;  // 32 x 32 FP64 inverses of A's diagonal (order n) into D
  long long lda = 0, n = 0;
  double* D = nullptr;
  bool unit = false;
  int* zero = nullptr;  // nzero ints set to 0
  long long nzero = 0;
};
tb_status trsm_prep_launch(const PrepJobs& jobs, cudaStream_t st);
// unit: A's diagonal is taken as 1 (diag = 'U'); the stored diagonal is never read.
// B, ldb (optional): the right-hand side the first solve will take; when it
// qualifies for the persistent solve, that solve's first operand copy and
// counter zeroing join the set-up launch.
tb_status trsm_setup(bool right, long m, long n, const float* A, long lda, long nb, Split split, cudaStream_t st,
                     void* scratch, TrsmCtx& c, std::vector<long>& leaf_start, bool unit = false,
                     float* B = nullptr, long ldb = 0);
size_t trsm_scratch_bytes(bool right, long m, long n, long nb, Split split);
tb_status trsm_solve(TrsmCtx& c, const std::vector<long>& leaf_start, float* B, long ldb, long rows, long cols);
// The recursion as one GEMM launch per leaf product and per update.
tb_status trsm_solve_launches(TrsmCtx& c, const std::vector<long>& leaf_start, float* B, long ldb, long rows,
                              long cols);
// The recursion as one persistent launch (tb_trsm_dag.cu): same tiles, K
// ranges and accumulation order, scheduled on the device by progress
// counters. Eligible when B can be written by TMA (16-byte aligned, ldb a
// multiple of 4) and A has more than one leaf, and switched on by
// TB_TRSM_DAG=1 in the environment (read once).
bool trsm_dag_eligible(const TrsmCtx& c, const float* B, long ldb);
// Scratch, plan and preparation jobs (first operand copy, zeroed counters)
// of the persistent solve of B with context c, added to `jobs`.
tb_status trsm_dag_prepare(TrsmCtx& c, const float* B, long ldb, PrepJobs& jobs);
tb_status trsm_solve_dag(TrsmCtx& c, const std::vector<long>& leaf_start, float* B, long ldb, long rows, long cols);
// The same solve with B's independent dimension (columns for the left side,
// rows for the right side) split in two halves solved on the context's
// stream and the auxiliary stream, so the tail of each launch of one half
// overlaps the other half's work; small problems and the split precision
// solve in one piece (TB_TRSM_STREAMS=1 in the environment: always).
tb_status trsm_solve_2s(TrsmCtx& c, const std::vector<long>& leaf_start, float* B, long ldb, long rows, long cols);
// One-time kernel attribute set-up for the grouped launches (not capturable).
tb_status gemm_prepare_grouped();
tb_status trsm_prepare_grouped();

// General TRMM (side, uplo, trans, unit diagonal), tb_blas3.cu.
// beta != 0 gives C = alpha op(A) B + beta C (the TRSM refinement residual).
tb_status trmm_ex_impl(bool right, bool upper, bool trans, bool unit, long m, long n, float alpha, const float* A,
                       long lda, const float* B, long ldb, float* C, long ldc, Split split, void* ws, size_t ws_bytes,
                       cudaStream_t st, float beta = 0.f);
// FP8-e4m3 (per-128x128-block scaled) forms, tb_fp8.cu.
tb_status syrk_fp8(bool trans, long n, long k, float alpha, const float* A, long lda, float beta, float* C, long ldc,
                   cudaStream_t st, bool upper = false);
tb_status syr2k_fp8(long n, long k, float alpha, const float* A, long lda, const float* B, long ldb, float beta,
                    float* C, long ldc, cudaStream_t st);
tb_status trmm_fp8(bool right, bool upper, bool trans, bool unit, long m, long n, float alpha, const float* A,
                   long lda, const float* B, long ldb, float* C, long ldc, cudaStream_t st);
tb_status symm_fp8(bool lower, long m, long n, float alpha, const float* A, long lda, const float* B, long ldb,
                   float beta, float* C, long ldc, cudaStream_t st);
tb_status gemm_fp8(bool ta, bool tb_, long m, long n, long k, float alpha, const float* A, long lda, const float* B,
                   long ldb, float beta, float* C, long ldc, cudaStream_t st);

// ------------------------------------------------------------------ autotuner (tb_tune.cu)
struct TuneChoice {
  long nb;
  int engine;  // 0 single-CTA 128 x 256 tiles, 1 CTA pairs, 2 single-CTA 128 x 128 tiles
  double ms;
  int splitk = 1;  // SYRK: K parts of a split-K launch (1: one pass)
};
// Split-K SYRK of this thread (the autotuner's trials and choice): parts of
// K, 1 = one pass. Applies to plain 'N' SYRKs of order <= kSplitKMaxN.
constexpr long kSplitKMaxN = 4096;
void set_splitk_override(int splits);
int splitk_override();
struct SplitKScope {
  int saved;
  explicit SplitKScope(int s) : saved(splitk_override()) { set_splitk_override(s); }
  ~SplitKScope() { set_splitk_override(saved); }
};
std::string tune_key(const char* routine, const char* flags, long a, long b, int precision);
// The cached choice for `key`, or the fastest of `candidates` under `trial`
// (run once to warm up, then timed twice with CUDA events on `st`).
tb_status autotune(const std::string& key, const std::vector<TuneChoice>& candidates,
                   const std::function<tb_status(const TuneChoice&)>& trial, cudaStream_t st, TuneChoice* out);

// nb = TB_NB_AUTO forms of the public entry points (tuned, then run).
tb_status auto_ssyrk(char uplo, char trans, long n, long k, float alpha, const float* A, long lda, float beta,
                     float* C, long ldc, int precision);
tb_status auto_strsm(char side, long m, long n, const float* A, long lda, float* B, long ldb, int precision);
tb_status auto_ssyr2k(char uplo, char trans, long n, long k, float alpha, const float* A, long lda, const float* B,
                      long ldb, float beta, float* C, long ldc, int precision);
tb_status auto_strmm(char uplo, long m, long n, float alpha, const float* A, long lda, const float* B, long ldb,
                     float* C, long ldc, int precision);

// C(lower) (or C(upper)) *= beta (C = 0 when beta == 0).
tb_status scale_lower(long long n, float beta, float* C, long long ldc, cudaStream_t st, bool upper = false);
// Full symmetric FP16 copy of an n x n matrix with one stored triangle.
tb_status convert_sym_f32_f16(long long n, const float* A, long long lda, bool lower, __half* hi, __half* lo,
                              long long ldd, float lo_scale, cudaStream_t stream);

}  // namespace tb
