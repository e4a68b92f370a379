// Persistent warp-specialised tcgen05 GEMM engine (sm_100a).
//
//   C[m0+i, n0+j] = alpha * sum_k A(m0+i, k) * B(n0+j, k) + beta * C[...]
//
// over a host-built list of 128 x BN output tiles, each with its own K-block
// range. This single kernel serves every contraction of the library: the
// flattened recursion levels of SYRK/SYR2K (lower-triangle tile lists), the
// off-diagonal updates and leaf products of TRSM, and TRMM/SYMM.
//
// Roles (192 threads, one CTA per SM):
//   warp 0      TMA producer: 64-wide K slabs of A and B into a smem ring.
//   warp 1      TMEM allocator + single-thread UMMA issuer.
//   warps 2..5  epilogue: TMEM -> registers -> alpha/beta -> C.
//   warp 6      (prefetch variants only, 224 threads) C loader: streams
//               128 x 32 chunks of C into a ring of shared-memory slots.
// The fp32 accumulator is double-buffered in TMEM (2 x 256 columns) so the
// epilogue of tile t overlaps the MMAs of tile t+1.
//
// Operands are fp16 in global memory, either MN-major (column-major storage
// with the M/N index contiguous, the layout the reference's FP32->FP16
// conversion produces) or K-major. Both map onto 128B-swizzled UMMA canonical
// layouts:
//   MN-major: TMA box {64 (MN), 64 (K)} -> 8 KB atoms; LBO = 8 KB between
//             64-wide MN atoms, SBO = 1 KB between 8-row K groups; a K step of
//             16 advances the descriptor by 2 KB.
//   K-major : TMA box {64 (K), R rows} -> R x 128 B; SBO = 1 KB between
//             8-row groups; a K step of 16 advances the descriptor by 32 B.
//
// Output: each 128 x 32 chunk of the tile is staged in shared memory
// (column-major, 512 B per column) and written with one TMA tensor store, so
// HBM sees 512-byte runs instead of one 128-byte piece per warp and column.
// When beta != 0, or when a tile crosses the lower-triangle mask, the chunk
// of C is first brought in with a TMA load and combined in shared memory
// (masked elements keep their old value). A plain per-element path remains
// for C that TMA cannot address (unaligned base or leading dimension).
//
// Split ("3-product") mode holds hi and lo copies of both operands and runs
//   acc0 += Ahi*Bhi ; acc1 += Ahi*Blo + Alo*Bhi
// with the correction in its own TMEM accumulator (Ootomo & Yokota 2022,
// the error-corrected FP16 scheme cuMpSGEMM's FP16TCEC mode uses). Every
// `kchunk` K-blocks the epilogue folds acc0 + corr_scale * acc1 into FP32
// registers with round-to-nearest adds: the tensor core's own FP32
// accumulation truncates, which would cost ~K/16 ulps.
#pragma once
#include "tb_ptx.cuh"

namespace tb {

struct GemmArgs {
  CUtensorMap mapA[2];  // [0] hi, [1] lo (split mode only)
  CUtensorMap mapB[2];
  CUtensorMap mapC;     // fp32 C, box {128, 32} (TMA epilogue only)
  CUtensorMap mapOut[2];  // fp16 side copies hi / lo over [0,out_m) x [0,out_n), box {128, 32}
  const int4* tiles;    // {m0, n0, kb_begin, kb_end}; m0/n0 relative to C
  int num_tiles;
  int a_off;  // row offset of the A operand in mapA's row coordinate
  int b_off;  // row offset of the B operand in mapB's row coordinate
  int k_off;  // K offset (elements) applied to both operands
  int M, N;   // extent of C (predication)
  float* C;
  long long ldc;
  float alpha, beta;
  int tri;   // 1: write only (i - j) >= diag (lower triangle); 2: only (j - i) >= diag (upper)
  int diag;
  float corr_scale;  // weight of the correction accumulator
  int kchunk;        // split mode: K-blocks per round-to-nearest fold
  int tma_c;         // 1: C through mapC (TMA epilogue)
  // Optional fused fp16 copies of the written result (column-major, ld_out):
  //   out_hi = fp16(v), out_lo = fp16((v - out_hi) * out_lo_scale)
  __half* out_hi;
  __half* out_lo;
  long long ld_out;
  float out_lo_scale;
  int out_m, out_n;  // side copies only for rows < out_m and columns < out_n
  int tma_out;       // 1: side copies through mapOut (requires tma_c and tri == 0)
  int c_ahead;       // CTA-pair kernel: C chunks loaded one ahead where no side copies are staged
  int* err;
  // FP8: per-(128-row block, 128-deep K block) scales of the A and B
  // operands, row-block-major with scale_ld K blocks per row block.
  const float* scale_a;
  const float* scale_b;
  int scale_ld;
  // Grouped launches: per-tile problem index into a device array of
  // GemmArgs (64-byte aligned; their tensor maps are read from global memory).
  const struct GemmArgs* problems;
  const int* tile_prob;
  // Device-side tile scheduler: nullptr = static assignment; otherwise a
  // zeroed counter from which the CTAs' producers claim tiles one at a time.
  int* sched;
  // Static assignment: nullptr = striding (CTA b takes tiles b, b + grid,
  // ...); otherwise CTA (or CTA pair) b takes tiles [ranges[b], ranges[b+1])
  // of a list the host balanced by simulating greedy claiming.
  const int* ranges;
};

// First / next tile of CTA (or CTA pair) `b` of `nb` under the static
// assignment; -1 when there is none.
__device__ __forceinline__ int static_first(const GemmArgs& a, int b) {
  if (a.ranges) return a.ranges[b] < a.ranges[b + 1] ? a.ranges[b] : -1;
  return b < a.num_tiles ? b : -1;
}
__device__ __forceinline__ int static_next(const GemmArgs& a, int b, int nb, int t) {
  if (a.ranges) return t + 1 < a.ranges[b + 1] ? t + 1 : -1;
  return t + nb < a.num_tiles ? t + nb : -1;
}

// Tile hand-off inside a CTA under the device-side scheduler: the producer
// claims a tile and queues its index (or -1, the end) in a kTileQ-deep ring;
// the MMA issuer, the four epilogue warps and (prefetch variants) the C
// loader each take the indices in order and release the slot.
constexpr int kTileQ = 4;

// The next tile of a consumer role: static striding, or the producer's
// queue (q/ph: the role's ring position). EPI: called by all 128 epilogue
// threads together, which then agree on the result.
template <bool EPI>
__device__ __forceinline__ int next_tile(const GemmArgs& args, int t, const volatile int* tq_idx, uint64_t* tq_full,
                                         uint64_t* tq_empty, int& q, uint32_t& ph, volatile int* abort_flag,
                                         int code) {
  if (!args.sched) return t < 0 ? static_first(args, blockIdx.x) : static_next(args, blockIdx.x, gridDim.x, t);
  const bool got = mbar_wait(&tq_full[q], ph, abort_flag, args.err, code);
  int v = got ? tq_idx[q] : -1;
  if constexpr (EPI) {
    if (named_bar_any(1, 128, !got)) v = -1;
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(&tq_empty[q]);
  } else {
    mbar_arrive(&tq_empty[q]);
  }
  if (++q == kTileQ) {
    q = 0;
    ph ^= 1u;
  }
  return v;
}

// The problem a tile belongs to: the launch's own arguments, or (grouped
// launches) one of the descriptors in global memory.
template <bool GROUPED>
__device__ __forceinline__ const GemmArgs& tile_problem(const GemmArgs& args, int t) {
  if constexpr (GROUPED) {
    return args.problems[args.tile_prob[t]];
  } else {
    return args;
  }
}

// PF (prefetch) variants serve launches whose tiles have few K-blocks: there
// the epilogue, not the MMA, bounds the tile, so they trade pipeline stages
// for a ring of shared-memory slots of 128 x 32 fp32 C chunks. A dedicated
// loader warp fills the ring in the epilogue's chunk order, each slot as
// soon as the stores of the chunk that used it last have read it, so the
// next tile's C is in flight while this tile's epilogue runs (for chunks the
// epilogue does not read, the loader only arrives on the slot's barrier).
// fp16 side copies get two staging buffers.
// FP8 variant: e4m3 K-major operands scaled per 128 x 128 block; the
// accumulator is folded into fp32 registers after every 128-deep K block
// with the product of the two blocks' scales.
template <int BN_, int NSPLIT_, bool A_MN_, bool B_MN_, bool PF_ = false, bool FP8_ = false>
struct GemmCfg {
  static constexpr bool FP8 = FP8_;
  static constexpr int ELEM = FP8 ? 1 : 2;       // operand bytes per element
  static constexpr int BM = 128, BN = BN_, BK = 128 / ELEM;  // one 128-byte swizzle row of K per stage
  static constexpr int KSTEPS = 4;               // MMAs per stage (K = 16 fp16 / 32 fp8 each)
  static constexpr int NSPLIT = NSPLIT_;
  static constexpr bool A_MN = A_MN_, B_MN = B_MN_;
  static constexpr bool PF = PF_;
  static constexpr bool FOLD = NSPLIT > 1 || FP8;  // accumulate in registers across TMEM rounds
  static constexpr int NOPS = (NSPLIT == 1) ? 1 : 2;  // copies per operand (hi[, lo])
  static constexpr int A_BYTES = BM * BK * ELEM;
  static constexpr int B_BYTES = BN * BK * ELEM;
  static constexpr int STAGE_BYTES = NOPS * (A_BYTES + B_BYTES);
  static constexpr int STAGES = FP8 ? 6 : PF ? (NSPLIT == 1 ? 3 : 2) : ((STAGE_BYTES <= 48 * 1024) ? 4 : 3);
  static constexpr int NACC = (NSPLIT == 1) ? 1 : 2;
  static constexpr int ACC_COLS = NACC * BN;  // TMEM columns per accumulation buffer
  static constexpr int TMEM_COLS = 2 * ACC_COLS;
  static_assert(TMEM_COLS <= 512, "TMEM budget");
  static constexpr int EPI_CHUNK_BYTES = 128 * 32 * 4;  // one staged 128 x 32 fp32 chunk
  // C-chunk staging slots (and their load barriers); PF: the loader's ring
  static constexpr int C_SLOTS = PF ? (NSPLIT == 1 ? 6 : 4) : 2;
  static constexpr int SIDE_BYTES = PF ? 2 * EPI_CHUNK_BYTES : 0;  // PF: two fp16 hi/lo side buffers
  static constexpr int EPI_BYTES = C_SLOTS * EPI_CHUNK_BYTES + SIDE_BYTES;
  static constexpr int BAR_BYTES = 512;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + EPI_BYTES + 1024 + BAR_BYTES;
  static_assert(SMEM_BYTES <= 232448, "shared memory budget");
  static constexpr uint32_t IDESC = idesc_f16(BM, BN, false, A_MN, B_MN);
  static constexpr int THREADS = PF ? 224 : 192;
};

template <bool MN, int ROWS>
__device__ __forceinline__ void load_operand(uint8_t* dst, const CUtensorMap* map, uint64_t* bar, int row0, int k) {
  if constexpr (MN) {
#pragma unroll
    for (int j = 0; j < ROWS / 64; ++j) tma_load_2d(dst + j * 8192, map, bar, row0 + 64 * j, k);
  } else {
    tma_load_2d(dst, map, bar, k, row0);
  }
}

template <bool MN>
__device__ __forceinline__ uint64_t operand_desc(uint32_t base, int kk) {
  if constexpr (MN) {
    return sdesc_sw128(base + kk * 2048, 8192, 1024);
  } else {
    return sdesc_sw128(base + kk * 32, 16, 1024);
  }
}

// Output triangle mask: tri 1 writes only (i - j) >= diag (lower), tri 2
// only (j - i) >= diag (upper); masked elements keep their old value.
// Whether a BM x BN tile at (m0, n0) reaches into the masked region.
__device__ __forceinline__ bool tile_reaches_mask(const GemmArgs& a, long long m0, long long n0, int bm, int bn) {
  return a.tri == 1 ? (m0 - (n0 + bn - 1)) < a.diag : (a.tri == 2 ? (n0 - (m0 + bm - 1)) < a.diag : false);
}

// Epilogue scalars, read into registers once per chunk. The epilogue's
// stores go through generic pointers (shared-memory slots, C, side copies)
// that the compiler cannot tell apart from the kernel's parameter memory, so
// GemmArgs fields read inside a store loop may be reloaded after every store.
struct EpiK {
  float alpha, beta, lo_scale;
  int tri, diag;
  __device__ __forceinline__ explicit EpiK(const GemmArgs& a)
      : alpha(a.alpha), beta(a.beta), lo_scale(a.out_lo_scale), tri(a.tri), diag(a.diag) {}
  // some element of the 128 x 32 chunk at (m0, n0) is masked
  __device__ __forceinline__ bool chunk_masked(long long m0, long long n0) const {
    return tri == 1 ? (m0 - (n0 + 31)) < diag : (tri == 2 ? (n0 - (m0 + 127)) < diag : false);
  }
  // The columns gj0 + [lo, hi) of row gi, out of the 32 from gj0 and below
  // `ncols` (a bound on gj), that the mask keeps: one range per row, so the
  // element loops compare small ints instead of testing every element's
  // 64-bit (i, j) against the triangle (which cost more than the stores).
  __device__ __forceinline__ void keep_range(long long gi, long long gj0, long long ncols, int& lo, int& hi) const {
    long long h = ncols - gj0, l = 0;
    if (tri == 1) h = min(h, gi - diag + 1 - gj0);  // keep gj <= gi - diag
    if (tri == 2) l = gi + diag - gj0;              // keep gj >= gi + diag
    hi = (int)max(0LL, min(32LL, h));
    lo = (int)max(0LL, min(32LL, l));
  }
};

// New values of one row's 32 staged C elements: alpha v + beta old where
// unmasked (old kept where masked), written back in place.
__device__ __forceinline__ void combine32(const EpiK& k, float* S, int row, const float* v, long long gi,
                                          long long gj0, bool any_masked, float* r) {
  if (any_masked) {
    int lo, hi;
    k.keep_range(gi, gj0, gj0 + 32, lo, hi);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const float old = S[j * 128 + row];
      r[j] = (j >= lo && j < hi) ? fmaf(k.beta, old, k.alpha * v[j]) : old;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = fmaf(k.beta, S[j * 128 + row], k.alpha * v[j]);
  }
#pragma unroll
  for (int j = 0; j < 32; ++j) S[j * 128 + row] = r[j];
}

// Scalars of the per-element store path for one tile, read into registers
// once per tile (EpiK's fields plus C, bounds and the side-copy fields; in
// grouped launches the problem descriptor lives in global memory).
struct StoreK : EpiK {
  float* C;
  long long ldc, ld_out;
  int N, out_m, out_n;
  __half* out_hi;
  __half* out_lo;
  __device__ __forceinline__ explicit StoreK(const GemmArgs& a)
      : EpiK(a), C(a.C), ldc(a.ldc), ld_out(a.ld_out), N(a.N), out_m(a.out_m), out_n(a.out_n), out_hi(a.out_hi),
        out_lo(a.out_lo) {}
};

// Fused fp16 hi[/lo] copies of 32 result values of one row.
__device__ __forceinline__ void store_fp16_copies(const StoreK& s, const float* r, long long gi, long long gj0) {
  const long long ld = s.ld_out;
  __half* hrow = s.out_hi + gi + gj0 * ld;
  __half* lrow = s.out_lo ? s.out_lo + gi + gj0 * ld : nullptr;
  int lo, hi;
  s.keep_range(gi, gj0, s.out_n, lo, hi);
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j < lo || j >= hi) continue;
    const __half h = __float2half_rn(r[j]);
    hrow[(long long)j * ld] = h;
    if (lrow) lrow[(long long)j * ld] = __float2half_rn((r[j] - __half2float(h)) * s.lo_scale);
  }
}

// Per-element path: alpha/beta update of 32 consecutive columns of one row,
// with the lower-triangle mask and bounds. With beta != 0 the 32 old values
// are loaded before any store so the loads are in flight together.
__device__ __forceinline__ void epilogue_store32(const StoreK& s, const float* v, long long gi, long long gj0) {
  const long long ldc = s.ldc;
  float* crow = s.C + gi + gj0 * ldc;
  int lo, hi;
  s.keep_range(gi, gj0, s.N, lo, hi);
  bool keep[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) keep[j] = j >= lo && j < hi;
  float r[32];
  if (s.beta != 0.0f) {
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = keep[j] ? __ldg(crow + (long long)j * ldc) : 0.f;
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = fmaf(s.beta, r[j], s.alpha * v[j]);
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = s.alpha * v[j];
  }
#pragma unroll
  for (int j = 0; j < 32; ++j)
    if (keep[j]) crow[(long long)j * ldc] = r[j];
  if (s.out_hi && gi < s.out_m) store_fp16_copies(s, r, gi, gj0);
}

// Epilogue state shared by the 4 epilogue warps (identical in all of them).
struct EpiState {
  int chunk;        // staged chunks written so far (selects the smem buffer)
  uint32_t lphase;  // per-buffer phase bit of the C-load barriers
  bool last_side;   // the previous chunk staged side copies (it used both buffers)
};

// TMA path for one 128 x 32 chunk at (m0, gj0): v[] holds this thread's row
// (32 consecutive columns). All 128 epilogue threads call it together.
// With TMA side copies (tma_out) the second staging buffer holds the fp16
// hi/lo chunk (8 KB each) and the fp32 chunk is single-buffered; otherwise
// chunks alternate between the two buffers. Problems of a grouped launch may
// differ in this, so the wait before reusing a buffer looks at the previous
// chunk's mode.
__device__ __forceinline__ void epilogue_chunk_tma(const GemmArgs& args, float* stage, uint64_t* cload, EpiState& es,
                                                   const float* v, int m0, int gj0, int row, bool need_load,
                                                   bool issuer, volatile int* abort_flag) {
  const EpiK k(args);
  const bool side_mode = args.tma_out != 0;
  const bool side = args.tma_out != 0 && gj0 < args.out_n && m0 < args.out_m;
  const bool copies = !side_mode && args.out_hi && (long long)m0 + row < args.out_m;
  const int b = side_mode ? 0 : (es.chunk & 1);
  float* S = stage + b * (128 * 32);
  __half* Hs = reinterpret_cast<__half*>(stage + 128 * 32);
  __half* Ls = Hs + 128 * 32;
  if (issuer) {
    if (side_mode || es.last_side)
      bulk_wait_read<0>();  // this chunk or the previous one uses both buffers: every earlier store has read smem
    else
      bulk_wait_read<1>();  // the store that last used buffer b has finished reading it
    if (need_load) {
      mbar_arrive_expect_tx(&cload[b], 128 * 32 * 4);
      tma_load_2d(S, &args.mapC, &cload[b], m0, gj0);
    }
  }
  named_bar_sync(1, 128);
  const long long gi = (long long)m0 + row;
  float r[32];
  if (need_load) {
    mbar_wait(&cload[b], (es.lphase >> b) & 1u, abort_flag, args.err, kDevErrTimeoutEpilogue);
    es.lphase ^= 1u << b;
    combine32(k, S, row, v, gi, gj0, k.chunk_masked(m0, gj0), r);
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      r[j] = k.alpha * v[j];
      S[j * 128 + row] = r[j];
    }
  }
  if (side) {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const __half hv = __float2half_rn(r[j]);
      Hs[j * 128 + row] = hv;
      Ls[j * 128 + row] = __float2half_rn((r[j] - __half2float(hv)) * k.lo_scale);
    }
  }
  fence_proxy_async_smem();
  named_bar_sync(1, 128);
  if (issuer) {
    tma_store_2d(&args.mapC, S, m0, gj0);
    if (side) {
      tma_store_2d(&args.mapOut[0], Hs, m0, gj0);
      if (args.out_lo) tma_store_2d(&args.mapOut[1], Ls, m0, gj0);
    }
    bulk_commit();
  }
  if (copies) store_fp16_copies(StoreK(args), r, gi, gj0);
  ++es.chunk;
  es.last_side = side_mode;
}

// Pipelined form of the TMA path for tiles that load C and stage no side
// copies: the C chunk for chunk c + 1 is requested (into the other buffer)
// before chunk c is combined, so a tile pays one load latency instead of one
// per chunk. c_issue_load requests chunk (m0, gj0) into buffer es.chunk + ahead
// once every earlier store has read its buffer; epilogue_chunk_loaded then
// combines and stores the chunk whose load was requested. Same arithmetic as
// epilogue_chunk_tma.
__device__ __forceinline__ void c_issue_load(const GemmArgs& args, float* stage, uint64_t* cload,
                                             const EpiState& es, int ahead, int m0, int gj0) {
  const int b = (es.chunk + ahead) & 1;
  bulk_wait_read<0>();  // the store that last used buffer b (and every earlier one) has read it
  mbar_arrive_expect_tx(&cload[b], 128 * 32 * 4);
  tma_load_2d(stage + b * (128 * 32), &args.mapC, &cload[b], m0, gj0);
}

__device__ __forceinline__ void epilogue_chunk_loaded(const GemmArgs& args, float* stage, uint64_t* cload,
                                                      EpiState& es, const float* v, int m0, int gj0, int row,
                                                      bool issuer, volatile int* abort_flag) {
  const EpiK k(args);
  const int b = es.chunk & 1;
  float* S = stage + b * (128 * 32);
  const long long gi = (long long)m0 + row;
  float r[32];
  mbar_wait(&cload[b], (es.lphase >> b) & 1u, abort_flag, args.err, kDevErrTimeoutEpilogue);
  es.lphase ^= 1u << b;
  combine32(k, S, row, v, gi, gj0, k.chunk_masked(m0, gj0), r);
  fence_proxy_async_smem();
  named_bar_sync(1, 128);
  if (issuer) {
    tma_store_2d(&args.mapC, S, m0, gj0);
    bulk_commit();
  }
  if (!args.tma_out && args.out_hi && gi < args.out_m) store_fp16_copies(StoreK(args), r, gi, gj0);
  ++es.chunk;
  es.last_side = false;
}

// PF epilogue, one 128 x 32 chunk (columns gj0..gj0+31) staged in the next
// slot of the loader's ring. The slot holds this chunk of C when need_load
// (the loader's TMA load completes its barrier) and is only handed over
// otherwise; the result is combined in place and stored from the slot. Before
// the issuer stores a chunk it waits until the previous chunk's stores have
// read their slot and gives that slot back to the loader. Side copies
// alternate between two fp16 buffers. All 128 epilogue threads call it
// together and keep identical state. Returns false, in every thread alike,
// when the slot's wait gave up.
struct PfState {
  int slot;        // next ring slot
  uint32_t phase;  // its barrier's phase (flips when the ring wraps)
  int prev;        // slot of the previous chunk, still to be released (-1: none)
  int side;        // side-copy chunks written so far (selects the buffer)
};

template <int RING>
__device__ __forceinline__ bool epilogue_chunk_pf(const GemmArgs& args, float* slots, __half* side_base,
                                                  uint64_t* cfull, uint64_t* cfree, PfState& pf, const float* v,
                                                  int m0, int gj0, int row, bool need_load, bool issuer,
                                                  volatile int* abort_flag) {
  const EpiK k(args);
  const bool side = args.tma_out != 0 && gj0 < args.out_n && m0 < args.out_m;
  const bool copies = !args.tma_out && args.out_hi && (long long)m0 + row < args.out_m;
  const int slot = pf.slot;
  float* S = slots + slot * (128 * 32);
  __half* Hs = side_base + (pf.side & 1) * (2 * 128 * 32);
  __half* Ls = Hs + 128 * 32;
  const bool got = mbar_wait(&cfull[slot], pf.phase, abort_flag, args.err, kDevErrTimeoutEpilogue);
  // also orders this chunk's smem writes after the issuer's previous stores
  if (named_bar_any(1, 128, !got)) return false;
  if (++pf.slot == RING) {
    pf.slot = 0;
    pf.phase ^= 1u;
  }
  const long long gi = (long long)m0 + row;
  float r[32];
  if (need_load) {
    combine32(k, S, row, v, gi, gj0, k.chunk_masked(m0, gj0), r);
  } else {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      r[j] = k.alpha * v[j];
      S[j * 128 + row] = r[j];
    }
  }
  if (side) {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const __half hv = __float2half_rn(r[j]);
      Hs[j * 128 + row] = hv;
      Ls[j * 128 + row] = __float2half_rn((r[j] - __half2float(hv)) * k.lo_scale);
    }
  }
  fence_proxy_async_smem();
  named_bar_sync(1, 128);
  if (issuer) {
    // the previous chunk's stores have read their slot (and side buffer)
    bulk_wait_read<0>();
    if (pf.prev >= 0) mbar_arrive(&cfree[pf.prev]);
    tma_store_2d(&args.mapC, S, m0, gj0);
    if (side) {
      tma_store_2d(&args.mapOut[0], Hs, m0, gj0);
      if (args.out_lo) tma_store_2d(&args.mapOut[1], Ls, m0, gj0);
    }
    bulk_commit();
  }
  pf.prev = slot;
  if (copies) store_fp16_copies(StoreK(args), r, gi, gj0);
  if (side) ++pf.side;
  return true;
}

template <class Cfg, bool GROUPED>
__global__ void __launch_bounds__(Cfg::THREADS, 1) gemm_kernel(const __grid_constant__ GemmArgs args) {
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, STAGES = Cfg::STAGES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  float* stage_c = reinterpret_cast<float*>(smem + STAGES * Cfg::STAGE_BYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * Cfg::STAGE_BYTES + Cfg::EPI_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;  // [2]
  uint64_t* tempty = tfull + 2;      // [2]
  uint64_t* drain = tempty + 2;      // [1] teardown barrier for the MMA issuer
  uint64_t* cload = drain + 1;       // [C_SLOTS] C-chunk loads of the TMA epilogue
  uint64_t* cfree = cload + Cfg::C_SLOTS;  // [C_SLOTS] PF: ring slots the epilogue gave back
  uint64_t* tq_full = cfree + Cfg::C_SLOTS;  // [kTileQ] tile hand-off (device-side scheduler)
  uint64_t* tq_empty = tq_full + kTileQ;     // [kTileQ]
  int* tq_idx = reinterpret_cast<int*>(tq_empty + kTileQ);  // [kTileQ]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tq_idx + kTileQ);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    for (int b = 0; b < Cfg::C_SLOTS; ++b) {
      mbar_init(&cload[b], 1);
      mbar_init(&cfree[b], 1);
    }
    for (int b = 0; b < kTileQ; ++b) {
      mbar_init(&tq_full[b], 1);
      mbar_init(&tq_empty[b], 1 + 4 + (Cfg::PF ? 1 : 0));  // MMA issuer, epilogue warps, C loader
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (!GROUPED && warp == 0 && lane == 0) {
    tma_prefetch_map(&args.mapA[0]);
    tma_prefetch_map(&args.mapB[0]);
    if (Cfg::NSPLIT > 1) {
      tma_prefetch_map(&args.mapA[1]);
      tma_prefetch_map(&args.mapB[1]);
    }
    if (args.tma_c) tma_prefetch_map(&args.mapC);
    if (args.tma_out) {
      tma_prefetch_map(&args.mapOut[0]);
      if (args.out_lo) tma_prefetch_map(&args.mapOut[1]);
    }
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  // the set-up above touches no global memory and may overlap the previous
  // launch's last tiles (programmatic dependent launch)
  grid_dep_wait();
  grid_dep_launch();

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      uint32_t issued_mask = 0, phase_mask = 0;  // per-stage: copy issued / its phase
      bool ok = true;
      const bool dyn = args.sched != nullptr;
      int tq = 0;
      uint32_t tq_ph = 0;
      int t = dyn ? atomicAdd(args.sched, 1) : static_first(args, blockIdx.x);
      while (ok) {
        if (t >= args.num_tiles) t = -1;
        if (dyn) {
          // hand the tile (or the end mark) to the other roles
          if (!mbar_wait(&tq_empty[tq], tq_ph ^ 1u, abort_flag, args.err, kDevErrTimeoutProducer)) {
            ok = false;
            break;
          }
          tq_idx[tq] = t;
          mbar_arrive(&tq_full[tq]);
          if (++tq == kTileQ) {
            tq = 0;
            tq_ph ^= 1u;
          }
        }
        if (t < 0) break;
        if (debug_stall_tile(args.err, t)) break;  // test hook: this tile's loads never come
        // the next claim is issued early so its latency hides
        const int t_next = dyn ? atomicAdd(args.sched, 1) : static_next(args, blockIdx.x, gridDim.x, t);
        const int4 tile = args.tiles[t];
        for (int kb = tile.z; kb < tile.w; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag, args.err, kDevErrTimeoutProducer)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[s], Cfg::STAGE_BYTES);
          uint8_t* st = smem + s * Cfg::STAGE_BYTES;
          const GemmArgs& P = tile_problem<GROUPED>(args, t);
          const int k = P.k_off + kb * BK;
#pragma unroll
          for (int h = 0; h < Cfg::NOPS; ++h) {
            load_operand<Cfg::A_MN, BM>(st + h * Cfg::A_BYTES, &P.mapA[h], &full[s], P.a_off + tile.x, k);
            load_operand<Cfg::B_MN, BN>(st + Cfg::NOPS * Cfg::A_BYTES + h * Cfg::B_BYTES, &P.mapB[h], &full[s],
                                        P.b_off + tile.y, k);
          }
          issued_mask |= 1u << s;
          phase_mask = (phase_mask & ~(1u << s)) | (ph << s);
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
        t = t_next;
      }
      if (!ok) {
        // Abort path: let every copy in flight land before the CTA exits.
        for (int i = 0; i < STAGES; ++i) {
          if (!((issued_mask >> i) & 1u)) continue;
          const uint64_t t0 = globaltimer_ns();
          while (!mbar_try_wait(&full[i], (phase_mask >> i) & 1u)) {
            if (globaltimer_ns() - t0 > 1000000000ull) {
              if (args.err) atomicCAS(args.err, 0, kDevErrTimeoutTeardown);
              break;
            }
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    // Accumulation "chunks": plain mode accumulates a tile's whole K range in
    // one TMEM buffer; split mode closes a chunk every `kchunk` K-blocks.
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int it = 0;  // chunk counter (selects TMEM buffer and phase)
      bool ok = true;
      bool any = false;
      const int kc = Cfg::FOLD ? args.kchunk : (1 << 30);
      int tq = 0;
      uint32_t tq_ph = 0;
      for (int t = next_tile<false>(args, -1, tq_idx, tq_full, tq_empty, tq, tq_ph, abort_flag, kDevErrTimeoutMma);
           t >= 0 && ok;
           t = next_tile<false>(args, t, tq_idx, tq_full, tq_empty, tq, tq_ph, abort_flag, kDevErrTimeoutMma)) {
        const int4 tile = args.tiles[t];
        for (int c0 = tile.z; c0 < tile.w && ok; c0 += kc, ++it) {
          const int c1 = (tile.w - c0 > kc) ? c0 + kc : tile.w;
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          if (!mbar_wait(&tempty[buf], tph ^ 1u, abort_flag, args.err, kDevErrTimeoutMma)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d0 = tmem_base + (uint32_t)(buf * Cfg::ACC_COLS);
          for (int kb = c0; kb < c1; ++kb) {
            if (!mbar_wait(&full[s], ph, abort_flag, args.err, kDevErrTimeoutMma)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t st = smem_u32(smem + s * Cfg::STAGE_BYTES);
            const uint32_t a_hi = st, b_hi = st + Cfg::NOPS * Cfg::A_BYTES;
#pragma unroll
            for (int kk = 0; kk < Cfg::KSTEPS; ++kk) {
              const uint32_t acc = (kb > c0 || kk > 0) ? 1u : 0u;
              const uint64_t da = operand_desc<Cfg::A_MN>(a_hi, kk);
              const uint64_t db = operand_desc<Cfg::B_MN>(b_hi, kk);
              if constexpr (Cfg::FP8)
                umma_f8(d0, da, db, Cfg::IDESC, acc);
              else
                umma_f16(d0, da, db, Cfg::IDESC, acc);
              if constexpr (Cfg::NSPLIT > 1) {
                const uint64_t da_lo = operand_desc<Cfg::A_MN>(a_hi + Cfg::A_BYTES, kk);
                const uint64_t db_lo = operand_desc<Cfg::B_MN>(b_hi + Cfg::B_BYTES, kk);
                umma_f16(d0 + BN, da, db_lo, Cfg::IDESC, acc);
                umma_f16(d0 + BN, da_lo, db, Cfg::IDESC, 1u);
              }
            }
            any = true;
            tc_commit(&empty[s]);
            if (++s == STAGES) {
              s = 0;
              ph ^= 1u;
            }
          }
          if (!ok) break;
          tc_commit(&tfull[buf]);
        }
      }
      if (!ok && any) {
        // Abort path: wait (bounded) until every issued MMA has retired.
        tc_commit(drain);
        const uint64_t t0 = globaltimer_ns();
        while (!mbar_try_wait(drain, 0)) {
          if (globaltimer_ns() - t0 > 1000000000ull) {
            if (args.err) atomicCAS(args.err, 0, kDevErrTimeoutTeardown);
            break;
          }
        }
      }
    }
    __syncwarp();
  } else if (Cfg::PF && warp == 6) {
    // ------------------------------------------------------------ C loader (PF)
    // Walks the CTA's tiles in the epilogue's chunk order; chunk n goes to
    // ring slot n % C_SLOTS once the epilogue has given back the slot's
    // previous chunk (n - C_SLOTS).
    if (lane == 0) {
      int slot = 0;
      uint32_t ph = 0;
      uint32_t armed = 0, armed_phase = 0;  // per-slot: a load was armed / its phase
      bool ok = true;
      int tq = 0;
      uint32_t tq_ph = 0;
      for (int t = next_tile<false>(args, -1, tq_idx, tq_full, tq_empty, tq, tq_ph, abort_flag,
                                    kDevErrTimeoutProducer);
           t >= 0 && ok;
           t = next_tile<false>(args, t, tq_idx, tq_full, tq_empty, tq, tq_ph, abort_flag, kDevErrTimeoutProducer)) {
        const int4 tile = args.tiles[t];
        const GemmArgs& P = tile_problem<GROUPED>(args, t);
        if (!P.tma_c) continue;
        const bool need = P.beta != 0.0f || tile_reaches_mask(P, tile.x, tile.y, BM, BN);
        for (int c0 = 0; c0 < BN && tile.y + c0 < P.N; c0 += 32) {
          if (!mbar_wait(&cfree[slot], ph ^ 1u, abort_flag, args.err, kDevErrTimeoutProducer)) {
            ok = false;
            break;
          }
          if (need) {
            mbar_arrive_expect_tx(&cload[slot], Cfg::EPI_CHUNK_BYTES);
            tma_load_2d(stage_c + slot * (128 * 32), &P.mapC, &cload[slot], tile.x, tile.y + c0);
            armed |= 1u << slot;
            armed_phase = (armed_phase & ~(1u << slot)) | (ph << slot);
          } else {
            // the slot's earlier load was consumed before the slot came back
            armed &= ~(1u << slot);
            mbar_arrive(&cload[slot]);
          }
          if (++slot == Cfg::C_SLOTS) {
            slot = 0;
            ph ^= 1u;
          }
        }
      }
      // every armed load lands before the CTA exits (immediate unless the
      // epilogue left early)
      for (int i = 0; i < Cfg::C_SLOTS; ++i) {
        if (!((armed >> i) & 1u)) continue;
        const uint64_t t0 = globaltimer_ns();
        while (!mbar_try_wait(&cload[i], (armed_phase >> i) & 1u))
          if (globaltimer_ns() - t0 > 1000000000ull) {
            if (args.err) atomicCAS(args.err, 0, kDevErrTimeoutTeardown);
            break;
          }
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue
    const int quarter = warp & 3;  // TMEM lane quarter this warp may access
    const int row = quarter * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    const bool issuer = (warp == 2 && lane == 0);
    EpiState es{0, 0u, false};
    int it = 0;
    bool ok = true;
    int tq = 0;
    uint32_t tq_ph = 0;
    if constexpr (Cfg::PF) {
      PfState pf{0, 0u, -1, 0};
      __half* side_base = reinterpret_cast<__half*>(stage_c + Cfg::C_SLOTS * (128 * 32));
      for (int t = next_tile<true>(args, -1, tq_idx, tq_full, tq_empty, tq, tq_ph, abort_flag, kDevErrTimeoutEpilogue);
           t >= 0 && ok;
           t = next_tile<true>(args, t, tq_idx, tq_full, tq_empty, tq, tq_ph, abort_flag, kDevErrTimeoutEpilogue)) {
        const int4 tile = args.tiles[t];
        const GemmArgs& P = tile_problem<GROUPED>(args, t);
        const long long gi = (long long)tile.x + row;
        const bool row_ok = gi < P.M;
        const bool tile_masked = tile_reaches_mask(P, tile.x, tile.y, BM, BN);
        const bool need_load = P.beta != 0.0f || tile_masked;
        const StoreK sk(P);
        if constexpr (!Cfg::FOLD) {
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          ++it;
          const bool got = mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue);
          if (named_bar_any(1, 128, !got)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * Cfg::ACC_COLS);
#pragma unroll 1
          for (int c0 = 0; c0 < BN; c0 += 32) {
            float v[32];
            tmem_ld32(tacc + c0, v);
            if (c0 == BN - 32) {
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive(&tempty[buf]);
            }
            if (tile.y + c0 >= P.N) continue;
            if (P.tma_c) {
              if (!epilogue_chunk_pf<Cfg::C_SLOTS>(P, stage_c, side_base, cload, cfree, pf, v, tile.x, tile.y + c0,
                                                   row, need_load, issuer, abort_flag)) {
                ok = false;
                break;
              }
            } else if (row_ok)
              epilogue_store32(sk, v, gi, (long long)tile.y + c0);
          }
        } else {
          float acc[BN];
#pragma unroll
          for (int j = 0; j < BN; ++j) acc[j] = 0.f;
          for (int c0k = tile.z; c0k < tile.w; c0k += args.kchunk) {
            const int buf = it & 1;
            const uint32_t tph = (uint32_t)(it >> 1) & 1u;
            ++it;
            const bool got = mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue);
            if (named_bar_any(1, 128, !got)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * Cfg::ACC_COLS);
#pragma unroll
            for (int c0 = 0; c0 < BN; c0 += 32) {
              float v[32], w[32];
              tmem_ld32x2(tacc + c0, tacc + BN + c0, v, w);
#pragma unroll
              for (int j = 0; j < 32; ++j) acc[c0 + j] += fmaf(args.corr_scale, w[j], v[j]);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[buf]);
          }
          if (!ok) break;
#pragma unroll
          for (int c0 = 0; c0 < BN; c0 += 32) {
            if (tile.y + c0 >= P.N) continue;
            if (P.tma_c) {
              if (!epilogue_chunk_pf<Cfg::C_SLOTS>(P, stage_c, side_base, cload, cfree, pf, acc + c0, tile.x,
                                                   tile.y + c0, row, need_load, issuer, abort_flag)) {
                ok = false;
                break;
              }
            } else if (row_ok)
              epilogue_store32(sk, acc + c0, gi, (long long)tile.y + c0);
          }
        }
      }
    } else
    for (int t = next_tile<true>(args, -1, tq_idx, tq_full, tq_empty, tq, tq_ph, abort_flag, kDevErrTimeoutEpilogue);
         t >= 0 && ok;
         t = next_tile<true>(args, t, tq_idx, tq_full, tq_empty, tq, tq_ph, abort_flag, kDevErrTimeoutEpilogue)) {
      const int4 tile = args.tiles[t];
      const GemmArgs& P = tile_problem<GROUPED>(args, t);
      const long long gi = (long long)tile.x + row;
      const bool row_ok = gi < P.M;
      // the tile crosses the masked (upper) region: min(i - j) < diag
      const bool tile_masked = tile_reaches_mask(P, tile.x, tile.y, BM, BN);
      // masked tiles with beta == 0 store their unmasked elements directly:
      // the TMA path would first have to load C to keep the masked ones
      const bool direct = tile_masked && P.beta == 0.0f;
      const StoreK sk(P);
      if constexpr (!Cfg::FOLD) {
        const int buf = it & 1;
        const uint32_t tph = (uint32_t)(it >> 1) & 1u;
        ++it;
        // one decision for all 128 epilogue threads: the chunks below hold named barriers
        if (named_bar_any(1, 128, !mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue)))
          break;
        tc_fence_after();
        const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * Cfg::ACC_COLS);
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
          float v[32];
          tmem_ld32(tacc + c0, v);
          if (c0 == BN - 32) {  // accumulator fully read: hand it back to the MMA warp
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[buf]);
          }
          if (P.tma_c && !direct) {
            if (tile.y + c0 < P.N)
              epilogue_chunk_tma(P, stage_c, cload, es, v, tile.x, tile.y + c0, row, P.beta != 0.0f || tile_masked,
                                 issuer, abort_flag);
          } else if (row_ok) {
            epilogue_store32(sk, v, gi, (long long)tile.y + c0);
          }
        }
      } else {
        float acc[BN];
#pragma unroll
        for (int j = 0; j < BN; ++j) acc[j] = 0.f;
        for (int c0k = tile.z; c0k < tile.w; c0k += args.kchunk) {
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          ++it;
          if (named_bar_any(1, 128, !mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * Cfg::ACC_COLS);
          if constexpr (Cfg::FP8) {
            // this round is K block c0k (kchunk = 1): scale by both blocks' scales
            const int kbs = (P.k_off >> 7) + c0k;
            const float sc = P.scale_a[(long long)((P.a_off + tile.x) >> 7) * P.scale_ld + kbs] *
                             P.scale_b[(long long)((P.b_off + tile.y) >> 7) * P.scale_ld + kbs];
#pragma unroll
            for (int c0 = 0; c0 < BN; c0 += 32) {
              float v[32];
              tmem_ld32(tacc + c0, v);
#pragma unroll
              for (int j = 0; j < 32; ++j) acc[c0 + j] = fmaf(sc, v[j], acc[c0 + j]);
            }
          } else {
#pragma unroll
            for (int c0 = 0; c0 < BN; c0 += 32) {
              float v[32], w[32];
              tmem_ld32x2(tacc + c0, tacc + BN + c0, v, w);
#pragma unroll
              for (int j = 0; j < 32; ++j) acc[c0 + j] += fmaf(args.corr_scale, w[j], v[j]);
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty[buf]);
        }
        if (!ok) break;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 32) {
          if (P.tma_c && !direct) {
            if (tile.y + c0 < P.N)
              epilogue_chunk_tma(P, stage_c, cload, es, acc + c0, tile.x, tile.y + c0, row,
                                 P.beta != 0.0f || tile_masked, issuer, abort_flag);
          } else if (row_ok) {
            epilogue_store32(sk, acc + c0, gi, (long long)tile.y + c0);
          }
        }
      }
    }
    if (issuer) bulk_wait<0>();  // all TMA stores complete before the CTA retires
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem_base, Cfg::TMEM_COLS);
}

// ---------------------------------------------------------------------------
// Pair variant (plain FP16): a cluster of two CTAs computes 256 x 256 output
// tiles with tcgen05.mma.cta_group::2. CTA r of the pair loads rows
// [m0 + 128r, +128) of A and rows [n0 + 128r, +128) of B (half of the tile's
// columns) into its own shared memory; the leader (r = 0) issues the 256-row
// MMA, which reads both CTAs' halves, and each CTA's TMEM receives its 128
// accumulator rows. Per SM, one 64-deep K slab moves 32 KB from L2 instead of
// the single-CTA tile's 48 KB for the same MMA work.
//   full[s]   leader only: both CTAs' loads complete_tx on it, the leader's
//             producer arms it with both CTAs' bytes;
//   empty[s]  both CTAs: the leader's commit multicasts to the pair;
//   tfull[b]  both CTAs: the leader's commit multicasts to the pair;
//   tempty[b] leader only: the 8 epilogue warps of the pair arrive remotely.
// Every wait is bounded like the single-CTA kernel's; a cluster barrier
// before TMEM is freed keeps either CTA from leaving while the pair's MMAs
// or remote arrivals may still touch it.
// DIRECT: launches that read no C and write no side copies (beta = 0, e.g.
// SYRK) store each thread's row of a chunk straight from registers (a
// warp's 32 rows of a column are one 128-byte line), which frees the
// epilogue's staging buffers for a seventh operand stage.
// NSPLIT = 3 (split precision): 256 x 128 pair tiles with hi/lo operands
// (each CTA loads 128 rows of A hi and lo and 64 rows of B hi and lo per K
// block) and two accumulators per TMEM buffer, hi*hi and hi*lo + lo*hi;
// the MMA issuer runs a tile's K range in rounds of kchunk K-blocks, one
// TMEM buffer per round, and the epilogue folds each round into FP32
// registers (acc += corr_scale * corr + main), as the single-CTA split
// kernel does. Per SM and 16-deep K step the three MMAs read 6 KB of shared
// memory each, against 8 KB for the single-CTA 128 x 128 split tile, which
// is bound by shared-memory bandwidth.
template <bool A_MN_, bool B_MN_, bool DIRECT_ = false, int NSPLIT_ = 1>
struct PairCfg {
  static constexpr int NSPLIT = NSPLIT_;
  static constexpr bool FOLD = NSPLIT > 1;
  static constexpr int NOPS = FOLD ? 2 : 1;  // copies per operand (hi[, lo])
  static constexpr int NACC = FOLD ? 2 : 1;  // accumulators per TMEM buffer
  static constexpr int BM = 128, BN = FOLD ? 128 : 256, BK = 64;  // BM: rows per CTA; BN: the pair tile's columns
  static constexpr bool A_MN = A_MN_, B_MN = B_MN_;
  static constexpr bool DIRECT = DIRECT_;
  static_assert(!(FOLD && DIRECT), "the split pair tile stages its epilogue");
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = (BN / 2) * BK * 2;
  static constexpr int STAGE_BYTES = NOPS * (A_BYTES + B_BYTES);
  static constexpr int STAGES = FOLD ? 4 : (DIRECT ? 7 : 6);
  static constexpr int ACC_COLS = NACC * BN;
  static constexpr int TMEM_COLS = 2 * ACC_COLS;
  static_assert(TMEM_COLS <= 512, "TMEM budget");
  static constexpr int EPI_BYTES = DIRECT ? 0 : 2 * 128 * 32 * 4;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + EPI_BYTES + 1024 + 256;
  static_assert(SMEM_BYTES <= 232448, "shared memory budget");
  static constexpr uint32_t IDESC = idesc_f16(2 * BM, BN, false, A_MN, B_MN);
  static constexpr int THREADS = 192;
};

template <bool MN, int ROWS>
__device__ __forceinline__ void load_operand_pair(uint8_t* dst, const CUtensorMap* map, uint32_t leader_bar, int row0,
                                                  int k) {
  if constexpr (MN) {
#pragma unroll
    for (int j = 0; j < ROWS / 64; ++j) tma_load_2d_pair(dst + j * 8192, map, leader_bar, row0 + 64 * j, k);
  } else {
    tma_load_2d_pair(dst, map, leader_bar, k, row0);
  }
}

template <class Cfg>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(192, 1)
    gemm_pair_kernel(const __grid_constant__ GemmArgs args) {
  constexpr int BN = Cfg::BN, BK = Cfg::BK, STAGES = Cfg::STAGES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  float* stage_c = reinterpret_cast<float*>(smem + STAGES * Cfg::STAGE_BYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * Cfg::STAGE_BYTES + Cfg::EPI_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;  // [2]
  uint64_t* tempty = tfull + 2;      // [2]
  uint64_t* drain = tempty + 2;      // [1]
  uint64_t* cload = drain + 1;       // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(cload + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 8);
      mbar_init(&cload[b], 1);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_map(&args.mapA[0]);
    tma_prefetch_map(&args.mapB[0]);
    if (args.tma_c) tma_prefetch_map(&args.mapC);
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_slot, Cfg::TMEM_COLS);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // the peer's barriers exist before any remote arrival
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  grid_dep_wait();  // as in gemm_kernel
  grid_dep_launch();
  const uint32_t full_leader = mapa_shared(smem_u32(full), 0);
  const uint32_t tempty_leader = mapa_shared(smem_u32(tempty), 0);

  if (warp == 0) {
    // ------------------------------------------------------------ producers (both CTAs)
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      uint32_t issued_mask = 0, phase_mask = 0;
      bool ok = true;
      for (int t = static_first(args, pair); t >= 0 && ok; t = static_next(args, pair, npairs, t)) {
        if (debug_stall_tile(args.err, t)) break;  // test hook: this tile's loads never come
        const int4 tile = args.tiles[t];
        for (int kb = tile.z; kb < tile.w; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag, args.err, kDevErrTimeoutProducer)) {
            ok = false;
            break;
          }
          if (leader) mbar_arrive_expect_tx(&full[s], 2 * Cfg::STAGE_BYTES);
          uint8_t* st = smem + s * Cfg::STAGE_BYTES;
          const int k = args.k_off + kb * BK;
          const uint32_t bar = full_leader + 8u * (uint32_t)s;
#pragma unroll
          for (int h = 0; h < Cfg::NOPS; ++h) {
            load_operand_pair<Cfg::A_MN, 128>(st + h * Cfg::A_BYTES, &args.mapA[h], bar,
                                              args.a_off + tile.x + 128 * (int)rank, k);
            load_operand_pair<Cfg::B_MN, BN / 2>(st + Cfg::NOPS * Cfg::A_BYTES + h * Cfg::B_BYTES, &args.mapB[h], bar,
                                                 args.b_off + tile.y + (BN / 2) * (int)rank, k);
          }
          issued_mask |= 1u << s;
          phase_mask = (phase_mask & ~(1u << s)) | (ph << s);
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
      if (!ok) {
        // Abort path: the leader sees its loads land on its own barriers; the
        // peer's loads report to the leader, so the peer waits a bounded time.
        if (leader) {
          for (int i = 0; i < STAGES; ++i) {
            if (!((issued_mask >> i) & 1u)) continue;
            const uint64_t t0 = globaltimer_ns();
            while (!mbar_try_wait(&full[i], (phase_mask >> i) & 1u))
              if (globaltimer_ns() - t0 > 1000000000ull) break;
          }
        } else {
          const uint64_t t0 = globaltimer_ns();
          while (globaltimer_ns() - t0 < 2000000ull) {
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer (leader)
    if (leader && lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int it = 0;
      bool ok = true, any = false;
      // a tile's K range in rounds of kchunk K-blocks (split) or one round
      const int kc = Cfg::FOLD ? args.kchunk : (1 << 30);
      for (int t = static_first(args, pair); t >= 0 && ok; t = static_next(args, pair, npairs, t)) {
        const int4 tile = args.tiles[t];
        for (int c0 = tile.z; c0 < tile.w && ok; c0 += kc, ++it) {
          const int c1 = (tile.w - c0 > kc) ? c0 + kc : tile.w;
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          if (!mbar_wait(&tempty[buf], tph ^ 1u, abort_flag, args.err, kDevErrTimeoutMma)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d0 = tmem_base + (uint32_t)(buf * Cfg::ACC_COLS);
          for (int kb = c0; kb < c1; ++kb) {
            if (!mbar_wait(&full[s], ph, abort_flag, args.err, kDevErrTimeoutMma)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a = smem_u32(smem + s * Cfg::STAGE_BYTES), b = a + Cfg::NOPS * Cfg::A_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
              const uint32_t acc = (kb > c0 || kk > 0) ? 1u : 0u;
              const uint64_t da = operand_desc<Cfg::A_MN>(a, kk), db = operand_desc<Cfg::B_MN>(b, kk);
              umma_f16_pair(d0, da, db, Cfg::IDESC, acc);
              if constexpr (Cfg::FOLD) {
                umma_f16_pair(d0 + BN, da, operand_desc<Cfg::B_MN>(b + Cfg::B_BYTES, kk), Cfg::IDESC, acc);
                umma_f16_pair(d0 + BN, operand_desc<Cfg::A_MN>(a + Cfg::A_BYTES, kk), db, Cfg::IDESC, 1u);
              }
            }
            any = true;
            tc_commit_pair(&empty[s], 3);
            if (++s == STAGES) {
              s = 0;
              ph ^= 1u;
            }
          }
          if (!ok) break;
          tc_commit_pair(&tfull[buf], 3);
        }
      }
      if (!ok && any) {
        tc_commit_pair(drain, 1);
        const uint64_t t0 = globaltimer_ns();
        while (!mbar_try_wait(drain, 0)) {
          if (globaltimer_ns() - t0 > 1000000000ull) {
            if (args.err) atomicCAS(args.err, 0, kDevErrTimeoutTeardown);
            break;
          }
        }
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue (both CTAs)
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    const bool issuer = (warp == 2 && lane == 0);
    const bool c_prefetch = args.c_ahead != 0;
    EpiState es{0, 0u, false};
    int it = 0;
    for (int t = static_first(args, pair); t >= 0; t = static_next(args, pair, npairs, t)) {
      const int4 tile = args.tiles[t];
      const int m0 = tile.x + 128 * (int)rank;
      const long long gi = (long long)m0 + row;
      const bool row_ok = gi < args.M;
      const bool tile_masked = tile_reaches_mask(args, m0, tile.y, 128, BN);
      const bool direct = tile_masked && args.beta == 0.0f;  // as in the single-CTA kernel
      const StoreK sk(args);
      // C loads one chunk ahead (the first before the accumulator wait) for
      // tiles that read C and stage no side copies in shared memory
      const long long nrem = ((long long)args.N - tile.y + 31) / 32;
      const int nval = nrem < BN / 32 ? (int)nrem : BN / 32;
      const bool ahead = !Cfg::DIRECT && c_prefetch && args.tma_c && !direct && m0 < args.M &&
                         (args.beta != 0.0f || tile_masked) &&
                         !(args.tma_out && m0 < args.out_m && tile.y < args.out_n);
      const int b0 = es.chunk & 1;
      const uint32_t ph0 = (es.lphase >> b0) & 1u;
      // one 128 x 32 chunk of this CTA's output rows: alpha * v (+ beta * C)
      auto store_chunk = [&](const float* v, int c0) {
        if (ahead) {
          if (c0 / 32 < nval) {
            if (issuer && c0 / 32 + 1 < nval) c_issue_load(args, stage_c, cload, es, 1, m0, tile.y + c0 + 32);
            epilogue_chunk_loaded(args, stage_c, cload, es, v, m0, tile.y + c0, row, issuer, abort_flag);
          }
        } else if (!Cfg::DIRECT && args.tma_c && !direct) {
          if (tile.y + c0 < args.N && m0 < args.M)
            epilogue_chunk_tma(args, stage_c, cload, es, v, m0, tile.y + c0, row, args.beta != 0.0f || tile_masked,
                               issuer, abort_flag);
        } else if (row_ok) {
          epilogue_store32(sk, v, gi, (long long)tile.y + c0);
        }
      };
      // the chunk-0 load in flight lands before the CTA leaves (bounded)
      auto drain_ahead = [&]() {
        if (ahead && issuer) {
          const uint64_t t0 = globaltimer_ns();
          while (!mbar_try_wait(&cload[b0], ph0))
            if (globaltimer_ns() - t0 > 1000000000ull) break;
        }
      };
      if (ahead && issuer) c_issue_load(args, stage_c, cload, es, 0, m0, tile.y);
      if constexpr (Cfg::FOLD) {
        float acc[BN];
#pragma unroll
        for (int j = 0; j < BN; ++j) acc[j] = 0.f;
        bool bad = false;
        for (int c0k = tile.z; c0k < tile.w; c0k += args.kchunk, ++it) {
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          if (named_bar_any(1, 128, !mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue))) {
            bad = true;
            break;
          }
          tc_fence_after();
          const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * Cfg::ACC_COLS);
#pragma unroll
          for (int c0 = 0; c0 < BN; c0 += 32) {
            float v[32], w[32];
            tmem_ld32x2(tacc + c0, tacc + BN + c0, v, w);
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[c0 + j] += fmaf(args.corr_scale, w[j], v[j]);
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive_cluster(tempty_leader + 8u * (uint32_t)buf);
        }
        if (bad) {
          drain_ahead();
          break;
        }
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 32) store_chunk(acc + c0, c0);
      } else {
        const int buf = it & 1;
        const uint32_t tph = (uint32_t)(it >> 1) & 1u;
        ++it;
        if (named_bar_any(1, 128, !mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue))) {
          drain_ahead();
          break;
        }
        tc_fence_after();
        const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * Cfg::ACC_COLS);
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
          float v[32];
          tmem_ld32(tacc + c0, v);
          if (c0 == BN - 32) {  // this CTA's half of the accumulator is read: tell the leader
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(tempty_leader + 8u * (uint32_t)buf);
          }
          store_chunk(v, c0);
        }
      }
    }
    if (issuer) bulk_wait<0>();
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // the pair's MMAs, remote arrivals and TMEM reads are over
  tc_fence_after();
  if (warp == 1) tmem_dealloc_pair(tmem_base, Cfg::TMEM_COLS);
}

}  // namespace tb
