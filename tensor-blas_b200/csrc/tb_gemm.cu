// Host side of the tcgen05 GEMM engine: tensor-map encoding, tile planning,
// variant dispatch and launch.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <queue>
#include <vector>
#include <map>
#include <mutex>
#include <string>

#include "tb_gemm.cuh"
#include "tb_internal.h"

namespace tb {

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// Tensor map for an fp16 operand; box_rows rows per load (K-major) or 64
// (MN-major), 64 elements along the contiguous dimension, 128B swizzle.
tb_status make_map(CUtensorMap* map, const Operand& op, int box_rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_last_error("cuTensorMapEncodeTiled unavailable");
    return TB_ERROR_CUDA;
  }
  if ((reinterpret_cast<uintptr_t>(op.ptr) & 15) != 0 || (op.ld * 2) % 16 != 0) {
    set_last_error("operand base must be 16-byte aligned and ld a multiple of 8 (ptr=%p ld=%lld)", op.ptr, op.ld);
    return TB_ERROR_INVALID_VALUE;
  }
  cuuint64_t dims[2];
  cuuint64_t strides[1] = {(cuuint64_t)op.ld * 2};
  cuuint32_t box[2];
  cuuint32_t estr[2] = {1, 1};
  if (op.mn_major) {
    dims[0] = (cuuint64_t)op.rows;
    dims[1] = (cuuint64_t)op.cols;
    box[0] = 64;
    box[1] = 64;
  } else {
    dims[0] = (cuuint64_t)op.cols;
    dims[1] = (cuuint64_t)op.rows;
    box[0] = 64;
    box[1] = (cuuint32_t)box_rows;
  }
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(op.ptr), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled failed (%d) rows=%lld cols=%lld ld=%lld", (int)r, op.rows, op.cols, op.ld);
    return TB_ERROR_CUDA;
  }
  return TB_SUCCESS;
}

// Tensor map for a K-major e4m3 operand (one byte per element): box
// {128 (K), box_rows}, 128B swizzle.
tb_status make_map8(CUtensorMap* map, const Operand& op, int box_rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_last_error("cuTensorMapEncodeTiled unavailable");
    return TB_ERROR_CUDA;
  }
  if (op.mn_major || (reinterpret_cast<uintptr_t>(op.ptr) & 15) != 0 || op.ld % 16 != 0) {
    set_last_error("fp8 operand must be K-major, 16-byte aligned, ld a multiple of 16 (ld=%lld)", op.ld);
    return TB_ERROR_INVALID_VALUE;
  }
  cuuint64_t dims[2] = {(cuuint64_t)op.cols, (cuuint64_t)op.rows};
  cuuint64_t strides[1] = {(cuuint64_t)op.ld};
  cuuint32_t box[2] = {128, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(op.ptr), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled (fp8) failed (%d)", (int)r);
    return TB_ERROR_CUDA;
  }
  return TB_SUCCESS;
}

// Tensor map for the fp32 output C (rows x cols, column-major, ldc), box
// {128 rows, 32 cols}, used by the TMA epilogue for loads and stores.
bool make_c_map(CUtensorMap* map, float* C, long long rows, long long cols, long long ldc) {
  EncodeTiledFn enc = encode_fn();
  if (!enc || (reinterpret_cast<uintptr_t>(C) & 15) != 0 || (ldc * 4) % 16 != 0) return false;
  cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
  cuuint64_t strides[1] = {(cuuint64_t)ldc * 4};
  cuuint32_t box[2] = {128, 32};
  cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map for an fp16 side copy restricted to rows x cols (the TMA store
// clips to this extent, which implements the out_m / out_n region).
bool make_half_out_map(CUtensorMap* map, __half* p, long long rows, long long cols, long long ld) {
  EncodeTiledFn enc = encode_fn();
  if (!enc || !p || rows <= 0 || cols <= 0 || (reinterpret_cast<uintptr_t>(p) & 15) != 0 || (ld * 2) % 16 != 0)
    return false;
  cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {128, 32};
  cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, p, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// TB_PDL=1 in the environment launches the GEMM engine's kernels with
// programmatic stream serialization (read once): a launch's CTAs may take
// the SMs that the previous grid on the stream frees during its last tiles
// and run their set-up (barriers, TMEM allocation) there, then wait in
// grid_dep_wait until that grid has completed. Off by default: on a B200
// the plain TRSM m = n = 16384 (nb 512, 63 dependent launches) took
// 6.11 ms with it against 6.04 ms without, SYRK 16384 3.48 ms either way,
// with identical results. Launches into a stream under graph capture are
// always plain.
static bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("TB_PDL");
    return e && e[0] == '1';
  }();
  return on;
}

template <class K>
static cudaError_t launch_engine(K* kernel, unsigned grid, unsigned block, size_t smem, cudaStream_t stream,
                                 const GemmArgs& args) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (pdl_enabled() && cudaStreamIsCapturing(stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args);
  }
  kernel<<<grid, block, smem, stream>>>(args);
  return cudaGetLastError();
}

template <class Cfg>
tb_status launch_pair(const GemmArgs& args, int num_tiles, cudaStream_t stream, double flops, double bytes = 0) {
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    TB_CUDA_TRY(cudaFuncSetAttribute(gemm_pair_kernel<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     Cfg::SMEM_BYTES));
    attr_set[dev] = true;
  }
  const int pairs_max = sm_count() / 2;
  const int pairs = num_tiles < pairs_max ? num_tiles : pairs_max;
  void* tok = prof_begin(stream, kProfPair);
  TB_CUDA_TRY(launch_engine(gemm_pair_kernel<Cfg>, 2 * pairs, Cfg::THREADS, Cfg::SMEM_BYTES, stream, args));
  prof_end(tok, stream, flops, bytes);
  note_launch();
  return TB_SUCCESS;
}

template <class Cfg, bool GROUPED>
tb_status launch_variant(const GemmArgs& args, int num_tiles, cudaStream_t stream, double flops, double bytes = 0) {
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    TB_CUDA_TRY(cudaFuncSetAttribute(gemm_kernel<Cfg, GROUPED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     Cfg::SMEM_BYTES));
    attr_set[dev] = true;
  }
  int grid = num_tiles < sm_count() ? num_tiles : sm_count();
  void* tok = prof_begin(stream, kProfGemm);
  TB_CUDA_TRY(launch_engine(gemm_kernel<Cfg, GROUPED>, grid, Cfg::THREADS, Cfg::SMEM_BYTES, stream, args));
  prof_end(tok, stream, flops, bytes);
  note_launch();
  return TB_SUCCESS;
}

}  // namespace

// 4 K-blocks (256-deep) between folds: at n = k = 16384 on a B200 the split
// SYRK / TRSM took 12.51 / 16.43 ms with 2, 11.69 / 15.18 ms with 4 and
// 11.22 / 14.01 ms with 8, at normwise errors vs FP64 of 2.8e-7 / 1.3e-7,
// 3.7e-7 / 1.6e-7 and 6.6e-7 / 2.4e-7; 4 keeps the 1e-6 target with margin
// as K grows.
int split_kchunk() {
  static const int k = [] {
    const char* e = getenv("TB_SPLIT_KCHUNK");
    const int v = e ? atoi(e) : 0;
    return (v >= 1 && v <= 64) ? v : 4;
  }();
  return k;
}

// CTA-pair epilogues load C one chunk ahead; TB_GEMM_C_AHEAD=0 in the
// environment turns it off (read once).
static bool c_ahead_enabled() {
  static const int on = [] {
    const char* e = getenv("TB_GEMM_C_AHEAD");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return on == 1;
}

// CTA-pair launches that store from registers get a seventh operand stage
// (TB_GEMM_PAIR_DIRECT in the environment, read once: 0 none, 1 the beta = 0
// launches without side copies, 2 all).
static int pair_direct_mode() {
  static const int mode = [] {
    const char* e = getenv("TB_GEMM_PAIR_DIRECT");
    return (e && e[0] >= '0' && e[0] <= '2') ? e[0] - '0' : 1;
  }();
  return mode;
}

int gemm_bn(Split s) { return s == Split::kPlain ? 256 : 128; }
int gemm_bn(Split s, int kblocks) {
  const bool pf = kblocks > 0 && kblocks <= kGemmPfMaxKb;
  if (s != Split::kPlain || pf) return 128;
  return engine_override() == kEngineNarrow ? 128 : 256;  // the narrow engine's plain tiles
}

tb_status gemm_build_args(const GemmCall& c, GemmArgs* out) {
  const bool split = c.split == Split::kHiLo && !c.fp8;
  // pair launches: each CTA loads half of the tile's B rows (128 of 256;
  // split: 64 of 128)
  const int bn = c.fp8 ? kGemmBNFp8 : (c.pair ? (split ? 64 : 128) : gemm_bn(c.split, c.kblocks));
  GemmArgs& a = *out;
  memset(&a, 0, sizeof(a));
  if (c.fp8) {
    if ((c.a_off % 128) != 0 || (c.b_off % 128) != 0 || (c.k_off % 128) != 0) {
      set_last_error("fp8 operand offsets must be multiples of the 128-wide scale blocks");
      return TB_ERROR_INVALID_VALUE;
    }
    TB_TRY(make_map8(&a.mapA[0], c.a_hi, kGemmBM));
    TB_TRY(make_map8(&a.mapB[0], c.b_hi, bn));
    a.scale_a = c.scale_a;
    a.scale_b = c.scale_b;
    a.scale_ld = c.scale_ld;
  } else {
    TB_TRY(make_map(&a.mapA[0], c.a_hi, kGemmBM));
    TB_TRY(make_map(&a.mapB[0], c.b_hi, bn));
  }
  if (split) {
    TB_TRY(make_map(&a.mapA[1], c.a_lo, kGemmBM));
    TB_TRY(make_map(&a.mapB[1], c.b_lo, bn));
  }
  a.tiles = c.tiles;
  a.num_tiles = c.num_tiles;
  a.ranges = c.ranges;
  a.a_off = c.a_off;
  a.b_off = c.b_off;
  a.k_off = c.k_off;
  a.M = c.M;
  a.N = c.N;
  a.C = c.C;
  a.ldc = c.ldc;
  a.alpha = c.alpha;
  a.beta = c.beta;
  a.tri = c.tri;
  a.diag = c.diag;
  a.corr_scale = c.corr_scale;
  a.kchunk = c.fp8 ? 1 : (c.kchunk > 0 ? c.kchunk : 1);
  a.tma_c = make_c_map(&a.mapC, c.C, c.M, c.N, c.ldc) ? 1 : 0;
  a.out_hi = c.out_hi;
  a.out_lo = c.out_lo;
  a.ld_out = c.ld_out;
  a.out_lo_scale = c.out_lo_scale;
  a.out_m = c.out_m >= 0 ? (c.out_m < c.M ? c.out_m : c.M) : c.M;
  a.out_n = c.out_n >= 0 ? (c.out_n < c.N ? c.out_n : c.N) : c.N;
  a.tma_out = 0;
  a.c_ahead = c_ahead_enabled() ? 1 : 0;
  if (c.out_hi && a.tma_c && c.tri == 0 && make_half_out_map(&a.mapOut[0], c.out_hi, a.out_m, a.out_n, c.ld_out) &&
      (!c.out_lo || make_half_out_map(&a.mapOut[1], c.out_lo, a.out_m, a.out_n, c.ld_out)))
    a.tma_out = 1;
  a.err = c.err ? c.err : device_error_word();
  // TMA coordinates along the contiguous dimension must be 16-byte aligned.
  if (c.a_hi.mn_major && (c.a_off % 8) != 0) return TB_ERROR_INVALID_VALUE;
  if (c.b_hi.mn_major && (c.b_off % 8) != 0) return TB_ERROR_INVALID_VALUE;
  if ((!c.a_hi.mn_major || !c.b_hi.mn_major) && (c.k_off % 8) != 0) return TB_ERROR_INVALID_VALUE;
  return TB_SUCCESS;
}

// Algorithmic DRAM bytes of a launch (profiling only): the operands once
// (hi and lo in split mode), C read when beta != 0 and written (half of the
// rectangle for triangle launches), and the FP16 side copies.
static double gemm_algorithmic_bytes(const GemmCall& c) {
  const double elem = c.fp8 ? 1.0 : 2.0, nops = (c.split == Split::kHiLo && !c.fp8) ? 2.0 : 1.0;
  const double K = (double)c.kblocks * kGemmBK;
  const double ops = ((double)c.M + (double)c.N) * K * elem * nops;
  const double cbytes = (double)c.M * c.N * 4.0 * (c.beta != 0.f ? 2.0 : 1.0) * (c.tri ? 0.5 : 1.0);
  double side = 0;
  if (c.out_hi) {
    const double om = c.out_m >= 0 ? std::min<double>(c.out_m, c.M) : c.M;
    const double on = c.out_n >= 0 ? std::min<double>(c.out_n, c.N) : c.N;
    side = om * on * 2.0 * (c.out_lo ? 2.0 : 1.0);
  }
  return ops + cbytes + side;
}

tb_status gemm_launch(const GemmCall& c, cudaStream_t stream) {
  if (c.num_tiles <= 0) return TB_SUCCESS;
  GemmArgs a;
  TB_TRY(gemm_build_args(c, &a));
  const double bytes = gemm_algorithmic_bytes(c);
  const bool split = c.split == Split::kHiLo;
  const bool amn = c.a_hi.mn_major, bmn = c.b_hi.mn_major;
  if (c.fp8) return launch_variant<GemmCfg<kGemmBNFp8, 1, false, false, false, true>, false>(a, c.num_tiles, stream,
                                                                                            c.flops, bytes);
  if (c.pair && split) {
    if (amn && bmn) return launch_pair<PairCfg<true, true, false, 3>>(a, c.num_tiles, stream, c.flops, bytes);
    if (amn && !bmn) return launch_pair<PairCfg<true, false, false, 3>>(a, c.num_tiles, stream, c.flops, bytes);
    if (!amn && !bmn) return launch_pair<PairCfg<false, false, false, 3>>(a, c.num_tiles, stream, c.flops, bytes);
    return launch_pair<PairCfg<false, true, false, 3>>(a, c.num_tiles, stream, c.flops, bytes);
  }
  if (c.pair) {
    const int direct = pair_direct_mode();
    if (direct == 2 || (direct == 1 && c.beta == 0.f && !c.out_hi)) {
      if (amn && bmn) return launch_pair<PairCfg<true, true, true>>(a, c.num_tiles, stream, c.flops, bytes);
      if (amn && !bmn) return launch_pair<PairCfg<true, false, true>>(a, c.num_tiles, stream, c.flops, bytes);
      if (!amn && !bmn) return launch_pair<PairCfg<false, false, true>>(a, c.num_tiles, stream, c.flops, bytes);
      return launch_pair<PairCfg<false, true, true>>(a, c.num_tiles, stream, c.flops, bytes);
    }
    if (amn && bmn) return launch_pair<PairCfg<true, true>>(a, c.num_tiles, stream, c.flops, bytes);
    if (amn && !bmn) return launch_pair<PairCfg<true, false>>(a, c.num_tiles, stream, c.flops, bytes);
    if (!amn && !bmn) return launch_pair<PairCfg<false, false>>(a, c.num_tiles, stream, c.flops, bytes);
    return launch_pair<PairCfg<false, true>>(a, c.num_tiles, stream, c.flops, bytes);
  }
  if (c.kblocks > 0 && c.kblocks <= kGemmPfMaxKb) {
    if (!split) {
      if (amn && bmn) return launch_variant<GemmCfg<128, 1, true, true, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
      if (amn && !bmn) return launch_variant<GemmCfg<128, 1, true, false, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
      if (!amn && !bmn)
        return launch_variant<GemmCfg<128, 1, false, false, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
      return launch_variant<GemmCfg<128, 1, false, true, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
    }
    if (amn && bmn) return launch_variant<GemmCfg<128, 3, true, true, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
    if (amn && !bmn) return launch_variant<GemmCfg<128, 3, true, false, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
    if (!amn && !bmn) return launch_variant<GemmCfg<128, 3, false, false, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
    return launch_variant<GemmCfg<128, 3, false, true, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
  }
  if (!split && engine_override() == kEngineNarrow) {  // plans built with gemm_bn() = 128
    if (amn && bmn) return launch_variant<GemmCfg<128, 1, true, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
    if (amn && !bmn) return launch_variant<GemmCfg<128, 1, true, false>, false>(a, c.num_tiles, stream, c.flops, bytes);
    if (!amn && !bmn) return launch_variant<GemmCfg<128, 1, false, false>, false>(a, c.num_tiles, stream, c.flops, bytes);
    return launch_variant<GemmCfg<128, 1, false, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
  }
  if (!split) {
    if (amn && bmn) return launch_variant<GemmCfg<256, 1, true, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
    if (amn && !bmn) return launch_variant<GemmCfg<256, 1, true, false>, false>(a, c.num_tiles, stream, c.flops, bytes);
    if (!amn && !bmn) return launch_variant<GemmCfg<256, 1, false, false>, false>(a, c.num_tiles, stream, c.flops, bytes);
    return launch_variant<GemmCfg<256, 1, false, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
  } else {
    if (amn && bmn) return launch_variant<GemmCfg<128, 3, true, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
    if (amn && !bmn) return launch_variant<GemmCfg<128, 3, true, false>, false>(a, c.num_tiles, stream, c.flops, bytes);
    if (!amn && !bmn) return launch_variant<GemmCfg<128, 3, false, false>, false>(a, c.num_tiles, stream, c.flops, bytes);
    return launch_variant<GemmCfg<128, 3, false, true>, false>(a, c.num_tiles, stream, c.flops, bytes);
  }
}

// Large plain launches run on CTA pairs; TB_GEMM_PAIR=0 in the environment
// keeps them on single CTAs (read once; for comparing the two engines). The
// autotuner overrides the choice per thread.
static thread_local int t_engine_override = -1;
void set_engine_override(int engine) { t_engine_override = engine; }
int engine_override() { return t_engine_override; }

// Long split launches (hi/lo operands, three products) that write no FP16
// side copies run on CTA pairs too (256 x 128 tiles); TB_GEMM_PAIR_SPLIT=0
// in the environment keeps them on single-CTA 128 x 128 tiles (read once).
// On a B200: split SYRK n = k = 16384 11.62-11.67 ms on pairs against
// 12.22-12.37 ms, results bit-identical; the split TRSM's long updates
// (which stage the next leaf's hi/lo copies) took 1 % longer on pairs and
// stay on single CTAs. Per SM a 256 x 128 pair MMA runs as long as the
// single-CTA 128 x 128 one, so the pair saves shared-memory and L2 traffic
// only; a 256-column split tile would need 256 fold registers per thread.
static bool pair_split_enabled() {
  static const bool on = [] {
    const char* e = getenv("TB_GEMM_PAIR_SPLIT");
    return !(e && e[0] == '0');
  }();
  return on;
}

bool pair_engine_enabled() {
  if (t_engine_override >= 0) return t_engine_override == 1;
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("TB_GEMM_PAIR");
    on = (e && e[0] == '0') ? 0 : 1;
  }
  return on == 1;
}

// Static assignment for a tile list whose K ranges differ (TRMM, TRSM leaf
// products): the host simulates `workers` CTAs (or CTA pairs) claiming the
// tiles in list order as they free up, with a tile's cost its K-blocks plus
// a fixed epilogue share, and regroups the list by worker; the returned
// list is the tiles followed by the workers + 1 range bounds (packed into
// int4s). Lists with uniform K ranges are returned unchanged (striding is
// balanced for them). Claiming in list order keeps the tiles in flight at
// any moment close together in the list, as the plans' L2-friendly order
// intends, while no worker ends more than about one tile after the others.
static std::vector<int4> balance_tiles(const std::vector<int4>& tiles, int workers, bool* balanced) {
  *balanced = false;
  if (tiles.size() <= (size_t)workers || workers <= 1) return tiles;
  int kmin = 1 << 30, kmax = 0;
  for (const int4& t : tiles) {
    kmin = std::min(kmin, t.w - t.z);
    kmax = std::max(kmax, t.w - t.z);
  }
  if (kmin == kmax) return tiles;
  constexpr long long kEpilogueKb = 4;
  std::vector<std::vector<int>> own(workers);
  std::priority_queue<std::pair<long long, int>, std::vector<std::pair<long long, int>>, std::greater<>> q;
  for (int w = 0; w < workers; ++w) q.push({0, w});
  for (size_t i = 0; i < tiles.size(); ++i) {
    auto [tw, w] = q.top();
    q.pop();
    own[w].push_back((int)i);
    q.push({tw + (tiles[i].w - tiles[i].z) + kEpilogueKb, w});
  }
  std::vector<int4> out;
  out.reserve(tiles.size() + (workers + 4) / 4);
  std::vector<int> bounds(1, 0);
  for (int w = 0; w < workers; ++w) {
    for (int i : own[w]) out.push_back(tiles[i]);
    bounds.push_back((int)out.size());
  }
  while (bounds.size() % 4) bounds.push_back((int)out.size());
  for (size_t i = 0; i < bounds.size(); i += 4) out.push_back(make_int4(bounds[i], bounds[i + 1], bounds[i + 2], bounds[i + 3]));
  *balanced = true;
  return out;
}

// Uploads a (possibly balanced) list and points the call at it.
static tb_status set_tiles(GemmCall& c, const std::vector<int4>& tiles, int workers, cudaStream_t stream) {
  bool balanced = false;
  const std::vector<int4> list = balance_tiles(tiles, workers, &balanced);
  const int4* d = upload_tiles(list, stream);
  if (!d) return TB_ERROR_ALLOC;
  c.tiles = d;
  c.num_tiles = (int)tiles.size();
  c.ranges = balanced ? reinterpret_cast<const int*>(d + tiles.size()) : nullptr;
  return TB_SUCCESS;
}

tb_status gemm_launch_plan(GemmCall& c, const std::vector<int4>& plan, cudaStream_t stream) {
  const bool pf = c.kblocks > 0 && c.kblocks <= kGemmPfMaxKb;
  c.pair = !c.fp8 && (c.split == Split::kPlain || (pair_split_enabled() && !c.out_hi)) && !pf && c.M >= 512 &&
           c.N >= 512 && pair_engine_enabled();
  if (!c.pair) {
    TB_TRY(set_tiles(c, plan, std::min<int>((int)plan.size(), sm_count()), stream));
    return gemm_launch(c, stream);
  }
  // merge vertically adjacent 128-row tiles into 256-row pair tiles (the K
  // range of a pair tile spans both halves; products outside an operand's
  // support multiply stored zeros, and masked outputs are never written)
  // (a flat index over (256-row block, 128-column block): plans have
  // thousands of tiles and this runs on every call)
  std::vector<int4> merged;
  merged.reserve(plan.size());
  const long long rb = ((long long)c.M + 255) / 256, cb = ((long long)c.N + 127) / 128;
  std::vector<int> where((size_t)(rb * cb), -1);
  for (const int4& t : plan) {
    int& w = where[(size_t)((long long)(t.x >> 8) * cb + (t.y >> 7))];
    if (w < 0) {
      w = (int)merged.size();
      merged.push_back(make_int4((t.x >> 8) << 8, t.y, t.z, t.w));
    } else {
      int4& m = merged[w];
      m.z = t.z < m.z ? t.z : m.z;
      m.w = t.w > m.w ? t.w : m.w;
    }
  }
  TB_TRY(set_tiles(c, merged, std::min<int>((int)merged.size(), sm_count() / 2), stream));
  return gemm_launch(c, stream);
}

// Kernel attributes of the grouped variants, set outside any stream capture.
tb_status gemm_prepare_grouped() {
  TB_CUDA_TRY(cudaFuncSetAttribute(gemm_kernel<GemmCfg<128, 3, true, true>, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, GemmCfg<128, 3, true, true>::SMEM_BYTES));
  TB_CUDA_TRY(cudaFuncSetAttribute(gemm_kernel<GemmCfg<256, 1, true, true>, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, GemmCfg<256, 1, true, true>::SMEM_BYTES));
  return TB_SUCCESS;
}

// Grouped launch over problems whose descriptors (built by gemm_build_args
// and copied to the device) all use MN-major operands.
tb_status gemm_launch_grouped(Split split, const GemmArgs* d_problems, const int4* d_tiles, const int* d_tile_prob,
                              int num_tiles, double flops, cudaStream_t stream, int* d_sched) {
  if (num_tiles <= 0) return TB_SUCCESS;
  GemmArgs a;
  memset(&a, 0, sizeof(a));
  a.sched = d_sched;
  a.tiles = d_tiles;
  a.num_tiles = num_tiles;
  a.problems = d_problems;
  a.tile_prob = d_tile_prob;
  a.corr_scale = 1.0f / 2048.0f;
  a.kchunk = split_kchunk();
  a.err = device_error_word();
  if (split == Split::kHiLo)
    return launch_variant<GemmCfg<128, 3, true, true>, true>(a, num_tiles, stream, flops);
  return launch_variant<GemmCfg<256, 1, true, true>, true>(a, num_tiles, stream, flops);
}

// --------------------------------------------------------------------- plans
// Tiles are emitted in column-panel groups of kGroup tiles: within a group the
// walk goes down the rows, so the ~148 tiles resident at once share a few A
// row panels and kGroup B panels in L2.
static constexpr int kGroup = 8;

std::vector<int4> plan_rect(int M, int N, int bn, int kb0, int kb1) {
  std::vector<int4> t;
  const int mt = (M + kGemmBM - 1) / kGemmBM, nt = (N + bn - 1) / bn;
  t.reserve((size_t)mt * nt);
  for (int g = 0; g < nt; g += kGroup) {
    const int ge = g + kGroup < nt ? g + kGroup : nt;
    for (int i = 0; i < mt; ++i)
      for (int j = g; j < ge; ++j) t.push_back(make_int4(i * kGemmBM, j * bn, kb0, kb1));
  }
  return t;
}

std::vector<int4> plan_lower(int n, int bn, int kb0, int kb1) {
  std::vector<int4> t;
  const int mt = (n + kGemmBM - 1) / kGemmBM, nt = (n + bn - 1) / bn;
  for (int g = 0; g < nt; g += kGroup) {
    const int ge = g + kGroup < nt ? g + kGroup : nt;
    for (int i = 0; i < mt; ++i)
      for (int j = g; j < ge; ++j) {
        const int m0 = i * kGemmBM, n0 = j * bn;
        if (m0 + kGemmBM - 1 >= n0) t.push_back(make_int4(m0, n0, kb0, kb1));
      }
  }
  return t;
}

std::vector<int4> plan_upper(int n, int bn, int kb0, int kb1) {
  std::vector<int4> t;
  const int mt = (n + kGemmBM - 1) / kGemmBM, nt = (n + bn - 1) / bn;
  for (int g = 0; g < nt; g += kGroup) {
    const int ge = g + kGroup < nt ? g + kGroup : nt;
    for (int i = 0; i < mt; ++i)
      for (int j = g; j < ge; ++j) {
        const int m0 = i * kGemmBM, n0 = j * bn;
        if (n0 + bn - 1 >= m0) t.push_back(make_int4(m0, n0, kb0, kb1));
      }
  }
  return t;
}

// Device copies of tile plans, cached by content (per device). Plans are
// small (16 B per tile) and reused across calls of the same shape. The cache
// holds at most kTileCacheBytes per device; beyond that the least recently
// used lists are freed (after a device synchronisation, since launches still
// queued may read them).
namespace {
struct TileEntry {
  std::vector<int4> tiles;
  int4* d;
  uint64_t last_use;
};
struct TileCache {
  std::mutex mu;
  std::map<std::pair<int, uint64_t>, std::vector<TileEntry>> map;
  size_t bytes[64] = {};
  uint64_t clock = 0;
};
TileCache& tile_cache() {
  static TileCache c;
  return c;
}
constexpr size_t kTileCacheBytes = 64ull << 20;

// Frees least recently used lists of device `dev` until `need` more bytes
// fit under the cap (caller holds the lock).
void evict_tiles(TileCache& tc, int dev, size_t need) {
  if (dev >= 64 || tc.bytes[dev] + need <= kTileCacheBytes) return;
  cudaDeviceSynchronize();
  while (tc.bytes[dev] + need > kTileCacheBytes) {
    auto best = tc.map.end();
    size_t bi = 0;
    for (auto it = tc.map.begin(); it != tc.map.end(); ++it) {
      if (it->first.first != dev) continue;
      for (size_t i = 0; i < it->second.size(); ++i)
        if (best == tc.map.end() || it->second[i].last_use < best->second[bi].last_use) {
          best = it;
          bi = i;
        }
    }
    if (best == tc.map.end()) break;
    TileEntry& e = best->second[bi];
    cudaFree(e.d);
    tc.bytes[dev] -= e.tiles.size() * sizeof(int4);
    best->second.erase(best->second.begin() + (long)bi);
    if (best->second.empty()) tc.map.erase(best);
  }
}
}  // namespace

const int4* upload_tiles(const std::vector<int4>& tiles, cudaStream_t stream) {
  // Cached by content: a 64-bit FNV-1a hash selects the candidates, a full
  // comparison confirms.
  TileCache& tc = tile_cache();
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t bytes = tiles.size() * sizeof(int4);
  uint64_t h = 1469598103934665603ull ^ (uint64_t)bytes;
  const uint32_t* w = reinterpret_cast<const uint32_t*>(tiles.data());
  for (size_t i = 0; i < bytes / 4; ++i) h = (h ^ w[i]) * 1099511628211ull;
  std::lock_guard<std::mutex> lk(tc.mu);
  ++tc.clock;
  {
    auto it = tc.map.find({dev, h});
    if (it != tc.map.end())
      for (TileEntry& e : it->second)
        if (e.tiles.size() == tiles.size() && memcmp(e.tiles.data(), tiles.data(), bytes) == 0) {
          e.last_use = tc.clock;
          return e.d;
        }
  }
  evict_tiles(tc, dev, bytes);
  int4* d = nullptr;
  if (dev_malloc(reinterpret_cast<void**>(&d), bytes) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, tiles.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  (void)stream;
  tc.map[{dev, h}].push_back(TileEntry{tiles, d, tc.clock});
  if (dev < 64) tc.bytes[dev] += bytes;
  return d;
}

void release_tile_cache() {
  TileCache& tc = tile_cache();
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(tc.mu);
  for (auto it = tc.map.begin(); it != tc.map.end();) {
    if (it->first.first != dev) {
      ++it;
      continue;
    }
    for (TileEntry& e : it->second) cudaFree(e.d);
    it = tc.map.erase(it);
  }
  if (dev < 64) tc.bytes[dev] = 0;
}

}  // namespace tb
