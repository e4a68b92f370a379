// Persistent dependency-driven TRSM solve: every leaf product and every
// off-diagonal update of the recursion (reference: BLAS/tc_trsm.cu:31-80,
// tc_rtrsm_p2) in ONE launch of a tcgen05 kernel with a device-side tile
// scheduler.
//
// The recursion of tb_trsm.cu issues, per solve, one GEMM launch per leaf
// product and per update (63 launches for 32 leaves), each waiting for the
// previous one; the short ones (leaf products, K <= 1024 updates) are
// latency-bound. Here the same tiles, with the same K ranges, operands and
// epilogues (so each element sees the same products, the same FP32
// accumulation order and the same roundings), become tasks of one
// persistent kernel:
//
//  * B's independent dimension (columns for a left solve, rows for a right
//    solve) is cut into strips of one update tile; the triangular dimension
//    into the leaf blocks.
//  * Counters in global memory track progress per strip: xcnt[strip] counts
//    finished leaf tiles (leaf b of a strip can only start once leaf b-1 of
//    that strip has finished, so one count per strip orders them all), and
//    updb[block][strip] counts finished update tiles whose output lies in
//    that block.
//  * A task waits (bounded spin, acquire) for at most two counters: an
//    update tile for the leaves its K range needs (xcnt) and for the earlier
//    updates of its output tile in recursion order (updb: the FP32 sums are
//    applied in the same order as the launch sequence would); a leaf tile
//    for all updates of its block. When its output (TMA stores of B and of
//    the FP16 side copies) has landed, the tile adds one to its own counter
//    (release).
//  * Tasks are claimed in a host-planned order (an event simulation of the
//    tiles on the SMs, most urgent block first) that is topological: every
//    counter a task waits for is fed by tasks earlier in the order, so the
//    lowest unfinished task can always run and the kernel cannot deadlock,
//    whether or not all CTAs are resident.
//  * Each leaf block's FP16 hi/lo copy R_b (the leaf product's operand,
//    written by the epilogue of the last update of that block) gets its own
//    slice of one full-size buffer, since several blocks are in flight.
//
// Tiles: plain updates 128 x 256 (FP16, one accumulator), split tiles
// (leaf products, and updates of the split precision) 128 x 128 with hi/lo
// operands and a correction accumulator folded into FP32 registers every
// split_kchunk() K-blocks, as the GEMM engine does. Shared memory: 192 KB of
// operand stages (four of 48 KB for plain solves, three of 64 KB for split
// ones) and two 16 KB epilogue chunks.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <queue>
#include <string>
#include <tuple>
#include <vector>

#include "tb_gemm.cuh"
#include "tb_internal.h"

namespace tb {

namespace {

// One task: a tile of one op (a leaf product or an update) with its waits.
struct DagTask {
  int4 tile;  // {m0, n0, kb_begin, kb_end}, relative to the op's C and K offset
  int4 dep;   // {counter, target, counter, target}; counter < 0: no wait
  int4 meta;  // {op, split (0/1), counter to add 1 to when done (-1: none), 0}
};
static_assert(sizeof(DagTask) == 48, "task layout");

struct DagArgs {
  const GemmArgs* ops;  // per-op descriptors (64-byte aligned, device memory)
  const DagTask* tasks;
  int num_tasks;
  int* claim;  // zeroed: next task to claim
  int* ctr;    // zeroed progress counters
  int* err;    // device error block
  int kchunk;  // split tiles: K-blocks per round-to-nearest fold (the GEMM engine's, split_kchunk())
};

// Operand stages: plain solves (whose updates are plain 128 x 256 tiles,
// 48 KB per K-block) use four 48 KB stages, and a split leaf K-block (64 KB:
// hi and lo of both operands) spans two of them (A hi, A lo, B hi in the
// first, B lo in the second); split solves use three 64 KB stages.
constexpr int kDagABytes = 128 * 64 * 2;  // one 128-row x 64-deep FP16 operand block
constexpr int kDagRingBytes = 3 * 65536;
constexpr int kDagEpiBytes = 2 * 128 * 32 * 4;
constexpr int kDagBarBytes = 512;
constexpr int kDagSmem = kDagRingBytes + kDagEpiBytes + 1024 + kDagBarBytes;
static_assert(kDagSmem <= 232448, "shared memory budget");
static_assert(4 * 3 * kDagABytes == kDagRingBytes, "four 48 KB stages fill the ring");
constexpr int kDagThreads = 192;
constexpr int kDevErrTimeoutDependency = 5;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add(int* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Orders generic-proxy accesses (the counters) with async-proxy ones (TMA).
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Bounded wait until ctr[i] >= target (acquire).
__device__ __forceinline__ bool dep_wait(const int* ctr, int i, int target, volatile int* abort_flag, int* err) {
  if (i < 0 || ld_acquire(ctr + i) >= target) return true;
  const uint64_t t0 = globaltimer_ns();
  const uint64_t limit = wait_limit_ns(err);
  while (ld_acquire(ctr + i) < target) {
    __nanosleep(64);
    if (*abort_flag) return false;
    if (globaltimer_ns() - t0 > limit) {
      *abort_flag = 1;
      if (err) atomicCAS(err, 0, kDevErrTimeoutDependency);
      return false;
    }
  }
  return true;
}

// Brings the 128 x 32 box of a tensor at (x, y) into L2 (no shared memory).
__device__ __forceinline__ void tma_prefetch_l2(const CUtensorMap* map, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global [%0, {%1, %2}];" ::"l"(reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y)
               : "memory");
}

// Epilogue of one tile, `nch` 128 x 32 chunks of C at (m0, y0 + 32c): the
// same arithmetic per element as the GEMM engine's (alpha v + beta old, the
// fp16 hi/lo side copies), staged in two shared-memory buffers and stored by
// TMA. With beta != 0 the chunks of C are loaded two ahead: chunk c + 2 is
// loaded into the buffer of chunk c as soon as chunk c's store has read it,
// while chunk c + 1 is combined. Side copies leave through plain stores from
// each thread's registers (a warp writes 32 consecutive rows per column), so
// both buffers stay free for C; the caller fences them before it publishes
// the tile. All 128 epilogue threads call it; `vals(c, v)` yields this
// thread's 32 values of chunk c.
struct DagEpi {
  int chunk;        // chunks staged so far (selects the buffer)
  uint32_t lphase;  // per-buffer phase of the C-load barriers
};

// Chunk c of the tile: waits for its C (beta != 0), combines, writes the
// side copies, stages it and has the issuer store it (and request chunk
// c + 2 into the same buffer).
__device__ __forceinline__ void dag_chunk(const GemmArgs& P, const StoreK& sk, float* stage, uint64_t* cload,
                                          DagEpi& ep, int m0, int y0, int c, int nch, int row, long long gi,
                                          bool issuer, bool side_tile, volatile int* abort_flag, const float* v) {
  const bool need = sk.beta != 0.0f;
  const int b = ep.chunk & 1;
  float* S = stage + b * (128 * 32);
  const int gj0 = y0 + 32 * c;
  float r[32];
  if (need) {
    mbar_wait(&cload[b], (ep.lphase >> b) & 1u, abort_flag, P.err, kDevErrTimeoutEpilogue);
    ep.lphase ^= 1u << b;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      r[j] = fmaf(sk.beta, S[j * 128 + row], sk.alpha * v[j]);
      S[j * 128 + row] = r[j];
    }
  } else {
    if (issuer) bulk_wait_read<1>();  // the store that last used buffer b has read it
    named_bar_sync(1, 128);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      r[j] = sk.alpha * v[j];
      S[j * 128 + row] = r[j];
    }
  }
  if (side_tile && gi < sk.out_m && gj0 < sk.out_n) store_fp16_copies(sk, r, gi, gj0);
  fence_proxy_async_smem();
  named_bar_sync(1, 128);
  if (issuer) {
    tma_store_2d(&P.mapC, S, m0, gj0);
    bulk_commit();
    if (need && c + 2 < nch) {
      bulk_wait_read<0>();  // this chunk's store has read buffer b
      mbar_arrive_expect_tx(&cload[b], 128 * 32 * 4);
      tma_load_2d(S, &P.mapC, &cload[b], m0, gj0 + 64);
    }
  }
  ++ep.chunk;
}

// Requests the first two chunks of C of a beta != 0 tile (issuer only).
__device__ __forceinline__ void dag_first_loads(const GemmArgs& P, float* stage, uint64_t* cload, const DagEpi& ep,
                                                int m0, int y0, int nch) {
  bulk_wait_read<0>();  // earlier stores have read both buffers
  for (int c = 0; c < 2 && c < nch; ++c) {
    const int b = (ep.chunk + c) & 1;
    mbar_arrive_expect_tx(&cload[b], 128 * 32 * 4);
    tma_load_2d(stage + b * (128 * 32), &P.mapC, &cload[b], m0, y0 + 32 * c);
  }
}

template <bool A_MN, bool B_MN, int NST>
__global__ void __launch_bounds__(kDagThreads, 1) trsm_dag_kernel(const __grid_constant__ DagArgs args) {
  constexpr int SB = kDagRingBytes / NST;       // bytes per stage
  constexpr bool SPLIT2 = SB < 4 * kDagABytes;  // a split K-block spans two stages
  static_assert(SB >= 3 * kDagABytes, "a plain K-block fits one stage");
  constexpr uint32_t IDESC_PLAIN = idesc_f16(128, 256, false, A_MN, B_MN);
  constexpr uint32_t IDESC_SPLIT = idesc_f16(128, 128, false, A_MN, B_MN);
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  float* stage_c = reinterpret_cast<float*>(smem + kDagRingBytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kDagRingBytes + kDagEpiBytes);
  uint64_t* empty = full + NST;
  uint64_t* tfull = empty + NST;  // [2]
  uint64_t* tempty = tfull + 2;          // [2]
  uint64_t* drain = tempty + 2;          // [1]
  uint64_t* cload = drain + 1;           // [2]
  uint64_t* tq_full = cload + 2;         // [kTileQ]
  uint64_t* tq_empty = tq_full + kTileQ;
  int* tq_idx = reinterpret_cast<int*>(tq_empty + kTileQ);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tq_idx + kTileQ);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
      mbar_init(&cload[b], 1);
    }
    for (int b = 0; b < kTileQ; ++b) {
      mbar_init(&tq_full[b], 1);
      mbar_init(&tq_empty[b], 1 + 4);  // MMA issuer + four epilogue warps
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------------------ producer: claim, wait, load
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      uint32_t issued_mask = 0, phase_mask = 0;
      bool ok = true;
      int tq = 0;
      uint32_t tq_ph = 0;
      int t = atomicAdd(args.claim, 1);
      while (ok) {
        if (t >= args.num_tasks) t = -1;
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
        if (t < 0) break;
        if (debug_stall_tile(args.err, t)) break;  // test hook: this tile's loads never come
        const int t_next = atomicAdd(args.claim, 1);
        const DagTask task = args.tasks[t];
        if (!dep_wait(args.ctr, task.dep.x, task.dep.y, abort_flag, args.err) ||
            !dep_wait(args.ctr, task.dep.z, task.dep.w, abort_flag, args.err)) {
          ok = false;
          break;
        }
        fence_proxy_async_global();  // the data behind the counters, for the TMA loads below
        const GemmArgs& P = args.ops[task.meta.x];
        const bool split = task.meta.y != 0;
        if (P.beta != 0.0f)  // the epilogue reads this tile of C: bring it into L2 while the MMAs run
          for (int c0 = 0; c0 < (split ? 128 : 256) && task.tile.y + c0 < P.N; c0 += 32)
            tma_prefetch_l2(&P.mapC, task.tile.x, task.tile.y + c0);
        // claims the next stage: waits until it is free, records it for the abort path
        auto take = [&](int& st_idx) -> bool {
          if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag, args.err, kDevErrTimeoutProducer)) return false;
          st_idx = s;
          issued_mask |= 1u << s;
          phase_mask = (phase_mask & ~(1u << s)) | (ph << s);
          if (++s == NST) {
            s = 0;
            ph ^= 1u;
          }
          return true;
        };
        for (int kb = task.tile.z; kb < task.tile.w; ++kb) {
          const int k = P.k_off + kb * 64;
          int s1 = 0, s2 = 0;
          if (!take(s1)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + s1 * SB;
          if (split) {
            uint8_t* st_lo = st + 3 * kDagABytes;
            if (SPLIT2) {
              if (!take(s2)) {
                ok = false;
                break;
              }
              st_lo = smem + s2 * SB;
              mbar_arrive_expect_tx(&full[s1], 3 * kDagABytes);
              mbar_arrive_expect_tx(&full[s2], kDagABytes);
            } else {
              mbar_arrive_expect_tx(&full[s1], 4 * kDagABytes);
            }
            uint64_t* bar_lo = SPLIT2 ? &full[s2] : &full[s1];
            load_operand<A_MN, 128>(st, &P.mapA[0], &full[s1], P.a_off + task.tile.x, k);
            load_operand<A_MN, 128>(st + kDagABytes, &P.mapA[1], &full[s1], P.a_off + task.tile.x, k);
            load_operand<B_MN, 128>(st + 2 * kDagABytes, &P.mapB[0], &full[s1], P.b_off + task.tile.y, k);
            load_operand<B_MN, 128>(st_lo, &P.mapB[1], bar_lo, P.b_off + task.tile.y, k);
          } else {
            mbar_arrive_expect_tx(&full[s1], 3 * kDagABytes);
            load_operand<A_MN, 128>(st, &P.mapA[0], &full[s1], P.a_off + task.tile.x, k);
            load_operand<B_MN, 256>(st + kDagABytes, &P.mapB[0], &full[s1], P.b_off + task.tile.y, k);
          }
        }
        t = t_next;
      }
      if (!ok) {
        // every copy in flight lands before the CTA exits
        for (int i = 0; i < NST; ++i) {
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
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int it = 0;
      bool ok = true, any = false;
      int tq = 0;
      uint32_t tq_ph = 0;
      while (ok) {
        if (!mbar_wait(&tq_full[tq], tq_ph, abort_flag, args.err, kDevErrTimeoutMma)) break;
        const int t = tq_idx[tq];
        mbar_arrive(&tq_empty[tq]);
        if (++tq == kTileQ) {
          tq = 0;
          tq_ph ^= 1u;
        }
        if (t < 0) break;
        const DagTask task = args.tasks[t];
        const bool split = task.meta.y != 0;
        const int kc = split ? args.kchunk : (1 << 30);
        for (int c0 = task.tile.z; c0 < task.tile.w && ok; c0 += kc, ++it) {
          const int c1 = (task.tile.w - c0 > kc) ? c0 + kc : task.tile.w;
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          if (!mbar_wait(&tempty[buf], tph ^ 1u, abort_flag, args.err, kDevErrTimeoutMma)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d0 = tmem_base + (uint32_t)(buf * 256);
          // waits for the next stage's operands
          auto next_full = [&](int& st_idx) -> bool {
            if (!mbar_wait(&full[s], ph, abort_flag, args.err, kDevErrTimeoutMma)) return false;
            st_idx = s;
            if (++s == NST) {
              s = 0;
              ph ^= 1u;
            }
            return true;
          };
          for (int kb = c0; kb < c1; ++kb) {
            int s1 = 0, s2 = 0;
            if (!next_full(s1) || (split && SPLIT2 && !next_full(s2))) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t st = smem_u32(smem + s1 * SB);
            const uint32_t st_lo = (split && SPLIT2) ? smem_u32(smem + s2 * SB) : st + 3 * kDagABytes;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
              const uint32_t acc = (kb > c0 || kk > 0) ? 1u : 0u;
              const uint64_t da = operand_desc<A_MN>(st, kk);
              if (split) {
                const uint64_t db = operand_desc<B_MN>(st + 2 * kDagABytes, kk);
                const uint64_t da_lo = operand_desc<A_MN>(st + kDagABytes, kk);
                const uint64_t db_lo = operand_desc<B_MN>(st_lo, kk);
                umma_f16(d0, da, db, IDESC_SPLIT, acc);
                umma_f16(d0 + 128, da, db_lo, IDESC_SPLIT, acc);
                umma_f16(d0 + 128, da_lo, db, IDESC_SPLIT, 1u);
              } else {
                umma_f16(d0, da, operand_desc<B_MN>(st + kDagABytes, kk), IDESC_PLAIN, acc);
              }
            }
            any = true;
            tc_commit(&empty[s1]);
            if (split && SPLIT2) tc_commit(&empty[s2]);
          }
          if (!ok) break;
          tc_commit(&tfull[buf]);
        }
      }
      if (!ok && any) {
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
  } else {
    // ------------------------------------------------------------ epilogue (warps 2..5)
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    const bool issuer = (warp == 2 && lane == 0);
    DagEpi ep{0, 0u};
    int it = 0;
    int tq = 0;
    uint32_t tq_ph = 0;
    bool ok = true;
    while (ok) {
      const bool got = mbar_wait(&tq_full[tq], tq_ph, abort_flag, args.err, kDevErrTimeoutEpilogue);
      int t = got ? tq_idx[tq] : -1;
      if (named_bar_any(1, 128, !got)) t = -1;
      __syncwarp();
      if (lane == 0) mbar_arrive(&tq_empty[tq]);
      if (++tq == kTileQ) {
        tq = 0;
        tq_ph ^= 1u;
      }
      if (t < 0) break;
      const DagTask task = args.tasks[t];
      const GemmArgs& P = args.ops[task.meta.x];
      const bool split = task.meta.y != 0;
      const int bn = split ? 128 : 256;
      const int nch = min(bn, P.N - task.tile.y + 31) / 32;
      // the tile writes fp16 side copies: rows below out_m and columns below out_n of the op
      const bool side_tile = P.out_hi != nullptr && task.tile.x < P.out_m && task.tile.y < P.out_n;
      if (issuer && P.beta != 0.0f) {
        // C (this tile of B) was last written by the earlier updates of this
        // tile on other CTAs: the producer hands the tile over before its own
        // dependency wait, and the first C chunks are loaded before the
        // accumulator is ready, so the epilogue waits for them itself
        dep_wait(args.ctr, task.dep.z, task.dep.w, abort_flag, args.err);
        fence_proxy_async_global();
      }
      if (!split) {
        const int buf = it & 1;
        const uint32_t tph = (uint32_t)(it >> 1) & 1u;
        ++it;
        // the first C chunks are requested before the accumulator is ready
        const StoreK sk(P);
        const long long gi = (long long)task.tile.x + row;
        if (issuer && sk.beta != 0.0f) dag_first_loads(P, stage_c, cload, ep, task.tile.x, task.tile.y, nch);
        if (named_bar_any(1, 128, !mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue))) {
          // gave up: the C loads requested above land before the CTA exits
          if (issuer && sk.beta != 0.0f)
            for (int c = 0; c < 2 && c < nch; ++c) {
              const int b = (ep.chunk + c) & 1;
              const uint64_t t0 = globaltimer_ns();
              while (!mbar_try_wait(&cload[b], (ep.lphase >> b) & 1u))
                if (globaltimer_ns() - t0 > 1000000000ull) {
                  if (args.err) atomicCAS(args.err, 0, kDevErrTimeoutTeardown);
                  break;
                }
            }
          break;
        }
        tc_fence_after();
        const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * 256);
#pragma unroll 1
        for (int c = 0; c < nch; ++c) {
          float v[32];
          tmem_ld32(tacc + 32 * c, v);
          if (c == nch - 1) {  // the accumulator is read: hand it back to the MMA warp
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[buf]);
          }
          dag_chunk(P, sk, stage_c, cload, ep, task.tile.x, task.tile.y, c, nch, row, gi, issuer, side_tile,
                    abort_flag, v);
        }
      } else {
        float acc[128];
#pragma unroll
        for (int j = 0; j < 128; ++j) acc[j] = 0.f;
        for (int c0k = task.tile.z; c0k < task.tile.w; c0k += args.kchunk) {
          const int buf = it & 1;
          const uint32_t tph = (uint32_t)(it >> 1) & 1u;
          ++it;
          if (named_bar_any(1, 128, !mbar_wait(&tfull[buf], tph, abort_flag, args.err, kDevErrTimeoutEpilogue))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t tacc = tmem_base + lane_addr + (uint32_t)(buf * 256);
#pragma unroll
          for (int c0 = 0; c0 < 128; c0 += 32) {
            float v[32], w[32];
            tmem_ld32x2(tacc + c0, tacc + 128 + c0, v, w);
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[c0 + j] += fmaf(P.corr_scale, w[j], v[j]);
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty[buf]);
        }
        if (!ok) break;
        const StoreK sk(P);
        const long long gi = (long long)task.tile.x + row;
        if (issuer && sk.beta != 0.0f) dag_first_loads(P, stage_c, cload, ep, task.tile.x, task.tile.y, nch);
#pragma unroll
        for (int c = 0; c < 4; ++c)
          if (c < nch)
            dag_chunk(P, sk, stage_c, cload, ep, task.tile.x, task.tile.y, c, nch, row, gi, issuer, side_tile,
                      abort_flag, acc + 32 * c);
      }
      if (task.meta.z >= 0) {
        // publish: every thread's side-copy stores, then the TMA stores, have landed
        if (side_tile) __threadfence();
        named_bar_sync(1, 128);
        if (issuer) {
          bulk_wait<0>();
          fence_proxy_async_global();
          red_release_add(args.ctr + task.meta.z, 1);
        }
      }
    }
    if (issuer) bulk_wait<0>();
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem_base, 512);
}

// ---------------------------------------------------------------------------- host planning
// One GEMM of the recursion (a leaf product or an update), in recursion order.
struct DagOp {
  GemmCall call;
  bool leaf;
  int block;     // leaf: its block; update: -1
  long s, mid, e;  // update: rows/cols [mid, e) -= ... K range [s, mid); leaf: [s, e)
  bool split;
  int bn;
};

// The ordered task list of one solve shape, cached on the host.
struct DagPlan {
  std::vector<int4> packed;  // DagTask as 3 int4 each, claim order
  int num_tasks = 0;
  int num_counters = 0;
  double est_makespan = 0;  // simulated, in cost units
};

using PlanKey = std::tuple<int, long, long, int, int, int>;  // right, indep, nt, leaf, split, workers

void build_ops(TrsmCtx& c, __half* rfh, __half* rfl, long long ldrf, long s, long e, std::vector<DagOp>& ops) {
  if (e - s <= c.leaf) {
    DagOp o;
    o.leaf = true;
    o.block = (int)(s / c.leaf);
    o.s = s;
    o.mid = s;
    o.e = e;
    o.split = true;
    o.bn = 128;
    const long nbl = e - s;
    GemmCall& g = o.call;
    g.split = Split::kHiLo;
    const bool split_x = c.split == Split::kHiLo;
    const int bidx = o.block;
    if (c.right) {
      g.a_hi = {rfh + s * ldrf, c.m, nbl, ldrf, true};
      g.a_lo = {rfl + s * ldrf, c.m, nbl, ldrf, true};
      g.b_hi = {c.wh + bidx * c.wstride, nbl, nbl, c.ldw, true};
      g.b_lo = {c.wl + bidx * c.wstride, nbl, nbl, c.ldw, true};
      g.C = c.B + s * c.ldb;
      g.M = (int)c.m;
      g.N = (int)nbl;
      g.out_hi = c.xh + s * c.ldx;
      g.out_lo = split_x ? c.xl + s * c.ldx : nullptr;
    } else {
      g.a_hi = {c.wh + bidx * c.wstride, nbl, nbl, c.ldw, true};
      g.a_lo = {c.wl + bidx * c.wstride, nbl, nbl, c.ldw, true};
      g.b_hi = {rfh + s, c.n, nbl, ldrf, false};
      g.b_lo = {rfl + s, c.n, nbl, ldrf, false};
      g.C = c.B + s;
      g.M = (int)nbl;
      g.N = (int)c.n;
      g.out_hi = c.xh + s;
      g.out_lo = split_x ? c.xl + s : nullptr;
    }
    g.ldc = c.ldb;
    g.ld_out = c.ldx;
    g.alpha = 1.f;
    g.beta = 0.f;
    g.kblocks = 0;
    g.flops = (double)g.M * g.N * nbl;
    ops.push_back(o);
    return;
  }
  const long nleaves = (e - s + c.leaf - 1) / c.leaf;
  const long mid = s + ((nleaves + 1) / 2) * c.leaf;
  build_ops(c, rfh, rfl, ldrf, s, mid, ops);
  DagOp o;
  o.leaf = false;
  o.block = -1;
  o.s = s;
  o.mid = mid;
  o.e = e;
  o.split = c.split == Split::kHiLo;
  o.bn = o.split ? 128 : 256;
  GemmCall& g = o.call;
  g.split = c.split;
  const bool hilo = o.split;
  const long kk = mid - s;
  if (c.right) {
    g.a_hi = {c.xh, c.m, c.n, c.ldx, true};
    g.a_lo = {hilo ? c.xl : nullptr, c.m, c.n, c.ldx, true};
    g.b_hi = {c.ah, c.nt, c.nt, c.lda_h, true};
    g.b_lo = {hilo ? c.al : nullptr, c.nt, c.nt, c.lda_h, true};
    g.a_off = 0;
    g.b_off = (int)mid;
    g.C = c.B + mid * c.ldb;
    g.M = (int)c.m;
    g.N = (int)(e - mid);
  } else {
    g.a_hi = {c.ah, c.nt, c.nt, c.lda_h, true};
    g.a_lo = {hilo ? c.al : nullptr, c.nt, c.nt, c.lda_h, true};
    g.b_hi = {c.xh, c.n, c.m, c.ldx, false};
    g.b_lo = {hilo ? c.xl : nullptr, c.n, c.m, c.ldx, false};
    g.a_off = (int)mid;
    g.b_off = 0;
    g.C = c.B + mid;
    g.M = (int)(e - mid);
    g.N = (int)c.n;
  }
  g.k_off = (int)s;
  g.ldc = c.ldb;
  g.alpha = -1.f;
  g.beta = 1.f;
  // the next leaf [mid, mid + leaf) gets its FP16 hi/lo operand here, in its
  // own slice of the full-size copy
  const long next = std::min<long>(c.leaf, e - mid);
  g.out_hi = c.right ? rfh + mid * ldrf : rfh + mid;
  g.out_lo = c.right ? rfl + mid * ldrf : rfl + mid;
  g.ld_out = ldrf;
  if (c.right)
    g.out_n = (int)next;
  else
    g.out_m = (int)next;
  g.kblocks = 0;
  g.flops = 2.0 * g.M * g.N * kk;
  ops.push_back(o);
  build_ops(c, rfh, rfl, ldrf, mid, e, ops);
}

// Tasks of every op with their counters, then the claim order.
DagPlan make_plan(const TrsmCtx& c, const std::vector<DagOp>& ops, int workers) {
  const bool right = c.right;
  const long indep = right ? c.m : c.n;
  const int sw = right ? 128 : (c.split == Split::kHiLo ? 128 : 256);  // strip width: one update tile
  const int nstrips = (int)((indep + sw - 1) / sw);
  const int nblocks = (int)((c.nt + c.leaf - 1) / c.leaf);
  const int xc0 = 0;                      // xcnt[strip]
  const int ub0 = nstrips;                // updb[block][strip]
  auto xctr = [&](int strip) { return xc0 + strip; };
  auto uctr = [&](int block, int strip) { return ub0 + block * nstrips + strip; };
  std::vector<int> xdone((size_t)nstrips, 0);        // leaf tiles generated so far per strip
  std::vector<int> udone((size_t)nblocks * nstrips, 0);
  // leaf tiles per strip before each block (for the update waits)
  std::vector<std::vector<int>> x_before((size_t)nblocks + 1, std::vector<int>((size_t)nstrips, 0));

  struct Gen {
    DagTask t;
    int block, opi, strip;
    double cost;
  };
  std::vector<Gen> gen;
  DagPlan plan;
  for (size_t oi = 0; oi < ops.size(); ++oi) {
    const DagOp& o = ops[oi];
    const GemmCall& g = o.call;
    const int bn = o.bn;
    const int mt = (g.M + kGemmBM - 1) / kGemmBM, ntl = (g.N + bn - 1) / bn;
    const long kk = o.leaf ? (o.e - o.s) : (o.mid - o.s);
    const int kb_all = (int)((kk + kGemmBK - 1) / kGemmBK);
    std::vector<int> snap;  // update: counts of earlier update tiles per (block, strip)
    if (!o.leaf) snap = udone;
    if (o.leaf) x_before[o.block] = xdone;
    for (int i = 0; i < mt; ++i)
      for (int j = 0; j < ntl; ++j) {
        const int m0 = i * kGemmBM, n0 = j * bn;
        int kb1 = kb_all;
        if (o.leaf) {  // W lower triangular: K beyond the tile's last W row is zero
          const long lim = right ? (long)n0 + bn : (long)m0 + kGemmBM;
          kb1 = (int)((std::min<long>(lim, kk) + kGemmBK - 1) / kGemmBK);
        }
        const int strip = right ? m0 / sw : n0 / sw;
        const long bpos = right ? (o.mid + n0) : (o.mid + m0);  // first output index along the block dimension
        const int block = (int)(bpos / c.leaf);
        Gen x;
        x.t.tile = make_int4(m0, n0, 0, kb1);
        x.t.meta = make_int4((int)oi, o.split ? 1 : 0, -1, 0);
        x.t.dep = make_int4(-1, 0, -1, 0);
        if (o.leaf) {
          x.t.dep.z = uctr(block, strip);
          x.t.dep.w = udone[(size_t)block * nstrips + strip];  // all update tiles of this block (all earlier)
          x.t.meta.z = xctr(strip);
        } else {
          const int xb = (int)(o.mid / c.leaf);  // leaves [0, xb) feed this K range
          x.t.dep.x = xctr(strip);
          x.t.dep.y = 0;  // filled below, once every leaf tile is known
          x.t.dep.z = uctr(block, strip);
          x.t.dep.w = snap[(size_t)block * nstrips + strip];
          x.t.meta.z = uctr(block, strip);
          x.t.meta.w = xb;  // kept on the host only until the target is known
        }
        x.block = block;
        x.opi = (int)oi;
        x.strip = strip;
        const double mma = (double)kb1 * (o.split ? 768.0 : 512.0);
        const double epi = o.split ? 1800.0 : 3000.0;
        x.cost = std::max(mma, epi) + 400.0;
        gen.push_back(x);
      }
    // counts after this op
    for (int i = 0; i < mt; ++i)
      for (int j = 0; j < ntl; ++j) {
        const int m0 = i * kGemmBM, n0 = j * bn;
        const int strip = right ? m0 / sw : n0 / sw;
        const long bpos = right ? (o.mid + n0) : (o.mid + m0);
        const int block = (int)(bpos / c.leaf);
        if (o.leaf)
          ++xdone[strip];
        else
          ++udone[(size_t)block * nstrips + strip];
      }
  }
  x_before[nblocks] = xdone;
  for (Gen& x : gen) {
    if (x.t.dep.x >= 0) {
      x.t.dep.y = x_before[x.t.meta.w][x.strip];
      x.t.meta.w = 0;
    }
  }
  // ---- claim order: event simulation of `workers` SMs taking the ready task
  // of the most urgent block (then recursion order, then strip)
  const int nt = (int)gen.size();
  const int nctr = nstrips + nblocks * nstrips;
  std::vector<int> counter((size_t)nctr, 0);
  std::vector<int> pending((size_t)nt, 0);
  std::vector<std::vector<std::pair<int, int>>> waiters((size_t)nctr);  // (target, task)
  auto prio = [&](int i) { return std::make_tuple(gen[i].block, gen[i].opi, gen[i].strip, i); };
  using PK = std::tuple<int, int, int, int>;
  std::priority_queue<PK, std::vector<PK>, std::greater<PK>> ready;
  for (int i = 0; i < nt; ++i) {
    const int4 d = gen[i].t.dep;
    if (d.x >= 0 && d.y > 0) {
      ++pending[i];
      waiters[d.x].push_back({d.y, i});
    }
    if (d.z >= 0 && d.w > 0) {
      ++pending[i];
      waiters[d.z].push_back({d.w, i});
    }
    if (pending[i] == 0) ready.push(prio(i));
  }
  for (auto& w : waiters) std::sort(w.begin(), w.end());
  std::vector<size_t> wpos((size_t)nctr, 0);
  using Ev = std::pair<double, int>;  // (finish time, task)
  std::priority_queue<Ev, std::vector<Ev>, std::greater<Ev>> running;
  std::vector<int> order;
  order.reserve((size_t)nt);
  int free_workers = workers;
  double now = 0;
  while ((int)order.size() < nt) {
    while (free_workers > 0 && !ready.empty()) {
      const int i = std::get<3>(ready.top());
      ready.pop();
      order.push_back(i);
      running.push({now + gen[i].cost, i});
      --free_workers;
    }
    if (running.empty()) break;  // cannot happen for a valid plan
    const Ev ev = running.top();
    running.pop();
    now = ev.first;
    ++free_workers;
    const int sig = gen[ev.second].t.meta.z;
    if (sig >= 0) {
      const int v = ++counter[sig];
      auto& w = waiters[sig];
      size_t& p = wpos[sig];
      while (p < w.size() && w[p].first <= v) {
        const int j = w[p].second;
        if (--pending[j] == 0) ready.push(prio(j));
        ++p;
      }
    }
  }
  plan.est_makespan = now;
  plan.num_tasks = (int)order.size();
  plan.num_counters = nctr;
  plan.packed.reserve((size_t)nt * 3);
  for (int i : order) {
    plan.packed.push_back(gen[i].t.tile);
    plan.packed.push_back(gen[i].t.dep);
    plan.packed.push_back(gen[i].t.meta);
  }
  return plan;
}

// Host check of a plan: every index in range, every K range non-empty and
// inside its op, and the claim order topological (each wait is met by
// signals of tasks earlier in the order, which is what rules out a
// deadlock). Returns an empty string or the first problem found.
std::string check_plan(const DagPlan& plan, const std::vector<DagOp>& ops) {
  std::vector<int> signals((size_t)plan.num_counters, 0);
  char buf[256];
  for (int i = 0; i < plan.num_tasks; ++i) {
    const int4 tile = plan.packed[3 * (size_t)i], dep = plan.packed[3 * (size_t)i + 1],
               meta = plan.packed[3 * (size_t)i + 2];
    if (meta.x < 0 || meta.x >= (int)ops.size()) return "op index out of range";
    const DagOp& o = ops[meta.x];
    const long kk = o.leaf ? (o.e - o.s) : (o.mid - o.s);
    if (tile.x < 0 || tile.x >= o.call.M || tile.y < 0 || tile.y >= o.call.N || tile.x % 128 || tile.y % o.bn)
      return "tile outside its op";
    if (tile.z != 0 || tile.w <= 0 || (long)tile.w * 64 > round_up(kk, 64)) return "bad K range";
    if (meta.y != (o.split ? 1 : 0)) return "split flag differs from its op";
    for (int w = 0; w < 2; ++w) {
      const int ctr = w ? dep.z : dep.x, target = w ? dep.w : dep.y;
      if (ctr < 0) continue;
      if (ctr >= plan.num_counters) return "wait counter out of range";
      if (signals[(size_t)ctr] < target) {
        snprintf(buf, sizeof(buf), "task %d waits for counter %d >= %d, but only %d earlier tasks feed it", i, ctr,
                 target, signals[(size_t)ctr]);
        return buf;
      }
    }
    if (meta.z >= plan.num_counters) return "signal counter out of range";
    if (meta.z >= 0) ++signals[(size_t)meta.z];
  }
  return "";
}

std::mutex g_plan_mu;
std::map<PlanKey, DagPlan> g_plans;

template <bool A_MN, bool B_MN, int NST>
tb_status launch_dag(const DagArgs& a, int grid, cudaStream_t st, double flops) {
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    TB_CUDA_TRY(cudaFuncSetAttribute(trsm_dag_kernel<A_MN, B_MN, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kDagSmem));
    attr_set[dev] = true;
  }
  void* tok = prof_begin(st, kProfDag);
  trsm_dag_kernel<A_MN, B_MN, NST><<<grid, kDagThreads, kDagSmem, st>>>(a);
  TB_CUDA_TRY(cudaGetLastError());
  prof_end(tok, st, flops);
  note_launch();
  return TB_SUCCESS;
}

}  // namespace

// Off by default: on a B200 the persistent solve of m = n = 16384 (nb 512)
// took 7.8 ms against 6.3 ms for the launch-per-product recursion with its
// two streams (its small tiles pay ~20 us each of epilogue and dependency
// latency, and MMA and epilogue overlap poorly). TB_TRSM_DAG=1 in the
// environment turns it on (read once).
bool trsm_dag_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("TB_TRSM_DAG");
    on = (e && e[0] == '1') ? 1 : 0;
  }
  return on == 1;
}

bool trsm_dag_eligible(const TrsmCtx& c, const float* B, long ldb) {
  if (!trsm_dag_enabled()) return false;
  // TMA epilogue for every tile: C base 16-byte aligned, ldb a multiple of 4
  if ((reinterpret_cast<uintptr_t>(B) & 15) != 0 || (ldb % 4) != 0) return false;
  // at least two leaves (one leaf is a single product) and an order the
  // plain form solves in FP16 (smaller ones take the split path anyway)
  return c.nt > c.leaf;
}

namespace {

// The persistent solve's scratch in pool slot 3: the per-leaf operand
// copies (hi, lo), the counters (plus the claim counter) and the op
// descriptors.
struct DagScratch {
  long long ldrf;
  size_t rf_bytes, ctr_bytes, ops_bytes;
};

DagScratch dag_scratch(const TrsmCtx& c, const DagPlan& plan, size_t nops) {
  DagScratch d;
  // left: K-major, element (j, k) at [k + j * ld]; right: MN-major, element (i, k) at [i + k * ld]
  d.ldrf = c.right ? round_up(c.m, 64) : round_up(c.nt, 64);
  const long long rf_elems = d.ldrf * (c.right ? c.nt : c.n);
  d.rf_bytes = (size_t)round_up(rf_elems * 2, 256);
  d.ctr_bytes = (size_t)round_up((long long)(plan.num_counters + 1) * 4, 256);
  d.ops_bytes = (size_t)round_up((long long)(nops * sizeof(GemmArgs)), 256);
  return d;
}

const DagPlan& dag_plan(TrsmCtx& c, size_t* nops) {
  const long indep = c.right ? c.m : c.n;
  const int workers = sm_count();
  const PlanKey key{c.right ? 1 : 0, indep, c.nt, c.leaf, c.split == Split::kHiLo ? 1 : 0, workers};
  std::vector<DagOp> ops;  // shapes only: the plan does not depend on the buffers
  build_ops(c, nullptr, nullptr, c.right ? round_up(c.m, 64) : round_up(c.nt, 64), 0, c.nt, ops);
  *nops = ops.size();
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plans.find(key);
  if (it == g_plans.end()) it = g_plans.emplace(key, make_plan(c, ops, workers)).first;
  return it->second;
}

}  // namespace

tb_status trsm_dag_prepare(TrsmCtx& c, const float* B, long ldb, PrepJobs& jobs) {
  size_t nops = 0;
  const DagPlan& plan = dag_plan(c, &nops);
  const DagScratch d = dag_scratch(c, plan, nops);
  char* ws = static_cast<char*>(pool_get(2 * d.rf_bytes + d.ctr_bytes + d.ops_bytes, 3));
  if (!ws) {
    set_last_error("trsm: cannot allocate %zu bytes of scratch", 2 * d.rf_bytes + d.ctr_bytes + d.ops_bytes);
    return TB_ERROR_ALLOC;
  }
  c.rfh = reinterpret_cast<__half*>(ws);
  c.rfl = reinterpret_cast<__half*>(ws + d.rf_bytes);
  c.ldrf = d.ldrf;
  c.dag_ctr = reinterpret_cast<int*>(ws + 2 * d.rf_bytes);
  if (jobs.nconv >= 2) return TB_ERROR_NOT_SUPPORTED;
  // the first leaf's operand comes from B itself
  PrepConv& cv = jobs.conv[jobs.nconv++];
  const long nbl0 = std::min<long>(c.leaf, c.nt);
  cv.rows = c.right ? c.m : nbl0;
  cv.cols = c.right ? nbl0 : c.n;
  cv.src = B;
  cv.lds = ldb;
  cv.hi = c.rfh;
  cv.lo = c.rfl;
  cv.ldd = d.ldrf;
  cv.tri = 0;
  jobs.zero = c.dag_ctr;
  jobs.nzero = plan.num_counters + 1;
  c.dag_B = B;
  c.dag_prepped = true;
  return TB_SUCCESS;
}

tb_status trsm_solve_dag(TrsmCtx& c, const std::vector<long>& leaf_start, float* B, long ldb, long rows, long cols) {
  if (ldb < (rows > 1 ? rows : 1)) return TB_ERROR_INVALID_VALUE;
  if (rows == 0 || cols == 0) return TB_SUCCESS;
  const long prep_m = c.m, prep_n = c.n;
  c.B = B;
  c.ldb = ldb;
  if (c.right)
    c.m = rows;
  else
    c.n = cols;
  // the set-up launch prepared this solve when it knew B (same B and shape);
  // otherwise one preparation launch here
  const bool prepped = c.dag_prepped && c.dag_B == B && prep_m == c.m && prep_n == c.n;
  c.dag_prepped = false;
  if (!prepped) {
    PrepJobs jobs;
    TB_TRY(trsm_dag_prepare(c, B, ldb, jobs));
    c.dag_prepped = false;
    TB_TRY(trsm_prep_launch(jobs, c.st));
  }
  size_t nops = 0;
  const DagPlan& plan = dag_plan(c, &nops);
  const DagScratch d = dag_scratch(c, plan, nops);
  char* ws = static_cast<char*>(pool_get(2 * d.rf_bytes + d.ctr_bytes + d.ops_bytes, 3));
  if (!ws || reinterpret_cast<__half*>(ws) != c.rfh) {
    set_last_error("trsm: persistent-solve scratch moved between preparation and solve");
    return TB_ERROR_ALLOC;
  }
  GemmArgs* d_ops = reinterpret_cast<GemmArgs*>(ws + 2 * d.rf_bytes + d.ctr_bytes);
  std::vector<DagOp> ops;
  build_ops(c, c.rfh, c.rfl, c.ldrf, 0, c.nt, ops);
  std::vector<GemmArgs> hops(ops.size());
  double flops = 0;
  for (size_t i = 0; i < ops.size(); ++i) {
    TB_TRY(gemm_build_args(ops[i].call, &hops[i]));
    flops += ops[i].call.flops;
  }
  // every output (B and the FP16 side copies) must leave through TMA stores,
  // whose completion a tile waits for before it publishes its progress
  for (size_t i = 0; i < ops.size(); ++i)
    if (!hops[i].tma_c || (ops[i].call.out_hi && !hops[i].tma_out))
      return trsm_solve_launches(c, leaf_start, B, ldb, rows, cols);
  const int4* d_tasks = upload_tiles(plan.packed, c.st);
  if (!d_tasks) return TB_ERROR_ALLOC;
  TB_CUDA_TRY(cudaMemcpyAsync(d_ops, hops.data(), hops.size() * sizeof(GemmArgs), cudaMemcpyHostToDevice, c.st));
  DagArgs a;
  a.ops = d_ops;
  a.tasks = reinterpret_cast<const DagTask*>(d_tasks);
  a.num_tasks = plan.num_tasks;
  a.claim = c.dag_ctr + plan.num_counters;
  a.ctr = c.dag_ctr;
  a.err = device_error_word();
  a.kchunk = split_kchunk();
  const int grid = std::min(sm_count(), plan.num_tasks);
  // plain solves: four 48 KB stages; split solves: three 64 KB stages
  if (c.split == Split::kPlain) {
    if (c.right) return launch_dag<true, true, 4>(a, grid, c.st, flops);
    return launch_dag<true, false, 4>(a, grid, c.st, flops);
  }
  if (c.right) return launch_dag<true, true, 3>(a, grid, c.st, flops);
  return launch_dag<true, false, 3>(a, grid, c.st, flops);
}

}  // namespace tb

// Host-only check of the persistent solve's plan for a shape (no device
// memory is touched): stats = {tasks, counters, ops, simulated makespan in
// cost units}. TB_ERROR_INVALID_VALUE with the reason in tb_last_error when
// the plan is not valid.
extern "C" tb_status tb_debug_trsm_plan(char side, long m, long n, long nb, int precision, long* stats) {
  using namespace tb;
  const bool right = side == 'R' || side == 'r';
  if (!right && side != 'L' && side != 'l') return TB_ERROR_INVALID_VALUE;
  if (m <= 0 || n <= 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  TrsmCtx c;
  memset(&c, 0, sizeof(c));
  c.right = right;
  c.m = m;
  c.n = n;
  c.nt = right ? n : m;
  const Split split = precision == TB_PREC_SPLIT ? Split::kHiLo : Split::kPlain;
  c.split = (split == Split::kPlain && c.nt < 2048) ? Split::kHiLo : split;
  long leaf = round_up(std::min<long>(nb, 512), 64);
  c.leaf = (int)std::min<long>(leaf, 512);
  c.lda_h = round_up(c.nt, 64);
  c.ldx = round_up(c.m, 64);
  c.ldw = c.leaf;
  c.wstride = c.ldw * c.leaf;
  c.ldb = m;
  const long long ldrf = right ? round_up(m, 64) : round_up(c.nt, 64);
  std::vector<DagOp> ops;
  build_ops(c, nullptr, nullptr, ldrf, 0, c.nt, ops);
  const DagPlan plan = make_plan(c, ops, 148);
  const std::string why = check_plan(plan, ops);
  if (stats) {
    stats[0] = plan.num_tasks;
    stats[1] = plan.num_counters;
    stats[2] = (long)ops.size();
    stats[3] = (long)plan.est_makespan;
  }
  if (!why.empty()) {
    set_last_error("trsm plan: %s", why.c_str());
    return TB_ERROR_INVALID_VALUE;
  }
  return TB_SUCCESS;
}
