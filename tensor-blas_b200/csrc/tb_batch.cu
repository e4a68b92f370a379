// Batched uneven SYRK / TRSM instances in a few grouped launches.
//
// The reference has no batched path: a caller loops over tc_syrk / tc_trsm,
// one recursion (and, for odd sizes, one padding cudaMalloc) per instance.
// Here tb_batch_create plans every instance once — FP16 copies, tile lists,
// per-problem GEMM descriptors with their tensor maps, TRSM leaf inverses —
// and tb_batch_run enqueues:
//   1. one grouped FP32 -> FP16 conversion over all operand copies,
//   2. one grouped 32x32 FP64 diagonal-inverse launch and one grouped leaf
//      inverse (column-chain) launch for all TRSM instances,
//   3. one grouped GEMM launch per step of the TRSM recursion, the SYRK
//      instances riding on the first: every instance's recursion alternates
//      leaf product / off-diagonal update (leaf, update, leaf, ...), so step p
//      of all instances is the same kind of product and shares one launch.
// tb_batch_run allocates nothing and never synchronises, so it can be
// captured in a CUDA graph (the planning already set kernel attributes and
// the device error word).
//
// SYRK instances: C (lower) = A A^T, A n x n. TRSM instances: X A^T = B, A
// n x n lower, B n x n overwritten (the reference's tc_trsm semantics,
// BLAS/tc_trsm.cu:139-174), solved with the same recursion as tb_strsm.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "tb_gemm.cuh"
#include "tb_internal.h"

namespace tb {
namespace {

struct ConvJob {
  const float* src;
  long long rows, cols, lds;
  __half* hi;
  __half* lo;
  long long ldd;
  int tri;
  long long first;  // first block index of this job in the grouped launch
};

constexpr int kConvPerThread = 8;
constexpr int kConvPerBlock = 256 * kConvPerThread;  // elements per block of the grouped conversion

// kConvPerBlock consecutive elements (column-major order over rows x cols)
// of one job per block, so short columns of small instances do not leave
// most of a block idle. blk_job maps a block to its job (one load, where a
// search over the job table would be a chain of dependent loads per block);
// each thread issues all its loads before it converts and stores.
__global__ void __launch_bounds__(256) conv_grouped_kernel(const ConvJob* __restrict__ jobs,
                                                           const int* __restrict__ blk_job) {
  const long long b = blockIdx.x;
  const ConvJob& jb = jobs[blk_job[b]];
  const long long rows = jb.rows, total = jb.rows * jb.cols, lds = jb.lds, ldd = jb.ldd;
  const float* const src = jb.src;
  __half* const dhi = jb.hi;
  __half* const dlo = jb.lo;
  const int tri = jb.tri;
  const long long e0 = (b - jb.first) * kConvPerBlock + threadIdx.x;
  long long at[kConvPerThread];
  float f[kConvPerThread];
  // (i, j) of element e0 by one division; the thread's later elements step
  // 256 further each, which moves i on and wraps it into the next column(s)
  long long j = e0 / rows, i = e0 - j * rows;
#pragma unroll
  for (int q = 0; q < kConvPerThread; ++q) {
    const long long e = e0 + q * 256;
    if (q > 0) {
      i += 256;
      while (i >= rows) {
        i -= rows;
        ++j;
      }
    }
    const bool ok = e < total && !(tri == 2 && i < ((j >> 3) << 3));
    at[q] = ok ? i + j * ldd : -1;
    f[q] = ok ? __ldg(src + i + j * lds) : 0.f;
  }
#pragma unroll
  for (int q = 0; q < kConvPerThread; ++q) {
    if (at[q] < 0) continue;
    const __half h = __float2half_rn(f[q]);
    dhi[at[q]] = h;
    if (dlo) dlo[at[q]] = __float2half_rn((f[q] - __half2float(h)) * 2048.f);
  }
}

struct Launch {
  Split split;
  int first_problem;  // offset into the problem array
  int num_problems;
  std::vector<int4> tiles;
  std::vector<int> prob;  // global problem index per tile
  double flops = 0;
  int4* d_tiles = nullptr;
  int* d_prob = nullptr;
  int* d_sched = nullptr;  // this launch's tile counter (device-side scheduler)
};

// Grows a byte arena with 256-byte aligned slices.
struct Arena {
  size_t used = 0;
  size_t take(size_t bytes) {
    const size_t o = used;
    used += (size_t)round_up((long long)bytes, 256);
    return o;
  }
};

}  // namespace
}  // namespace tb

struct tb_batch_s {
  int device = 0;
  void* scratch = nullptr;
  void* tables = nullptr;
  tb::ConvJob* d_conv = nullptr;
  int* d_blk_job = nullptr;  // job index of each block of the grouped conversion
  int nconv = 0;
  long long conv_blocks = 0;
  tb::DiagJob* d_diag = nullptr;
  int ndiag = 0;
  long long diag_blocks = 0;
  tb::ChainJob* d_chain = nullptr;
  int nchain = 0;
  tb::GemmArgs* d_problems = nullptr;
  int* d_sched = nullptr;  // one tile counter per grouped GEMM launch
  std::vector<tb::Launch> launches;
};

namespace tb {
namespace {

// Leaf size for a TRSM instance of order n: the largest power-of-two
// multiple of 64 not above min(nb, 512, n / 2) (one leaf when n <= 64).
long leaf_for(long n, long nb) {
  long cap = std::min<long>(nb > 0 ? nb : 512, 512);
  long leaf = 64;
  while (leaf * 2 <= cap && leaf * 2 <= std::max<long>(n / 2, 64)) leaf *= 2;
  return leaf;
}

struct TrsmPlan {
  long n;
  const float* A;
  long lda;
  float* B;
  long ldb;
  long leaf;
  __half *ah, *al, *xh, *xl, *wh, *wl, *rh, *rl;
  long long lda_h, ldx, ldw, wstride, ldr;
  std::vector<long> leaf_start;
  std::vector<GemmCall> ops;  // leaf, update, leaf, ...
  std::vector<long> op_k;      // contraction length of each op
};

void trsm_ops(TrsmPlan& p, Split split, long s, long e) {
  if (e - s <= p.leaf) {
    const int bidx = (int)(std::lower_bound(p.leaf_start.begin(), p.leaf_start.end(), s) - p.leaf_start.begin());
    const long nbl = e - s;
    GemmCall g;
    g.split = Split::kHiLo;
    g.a_hi = {p.rh, p.n, nbl, p.ldr, true};
    g.a_lo = {p.rl, p.n, nbl, p.ldr, true};
    g.b_hi = {p.wh + bidx * p.wstride, nbl, nbl, p.ldw, true};
    g.b_lo = {p.wl + bidx * p.wstride, nbl, nbl, p.ldw, true};
    g.C = p.B + s * p.ldb;
    g.ldc = p.ldb;
    g.M = (int)p.n;
    g.N = (int)nbl;
    g.out_hi = p.xh + s * p.ldx;
    g.out_lo = split == Split::kHiLo ? p.xl + s * p.ldx : nullptr;
    g.ld_out = p.ldx;
    g.flops = (double)g.M * g.N * nbl;
    p.ops.push_back(g);
    p.op_k.push_back(nbl);
    return;
  }
  const long nleaves = (e - s + p.leaf - 1) / p.leaf;
  const long mid = s + ((nleaves + 1) / 2) * p.leaf;
  trsm_ops(p, split, s, mid);
  GemmCall g;
  g.split = split;
  const bool hilo = split == Split::kHiLo;
  g.a_hi = {p.xh, p.n, p.n, p.ldx, true};
  g.a_lo = {hilo ? p.xl : nullptr, p.n, p.n, p.ldx, true};
  g.b_hi = {p.ah, p.n, p.n, p.lda_h, true};
  g.b_lo = {hilo ? p.al : nullptr, p.n, p.n, p.lda_h, true};
  g.b_off = (int)mid;
  g.k_off = (int)s;
  g.C = p.B + mid * p.ldb;
  g.ldc = p.ldb;
  g.M = (int)p.n;
  g.N = (int)(e - mid);
  g.alpha = -1.f;
  g.beta = 1.f;
  g.out_hi = p.rh;
  g.out_lo = p.rl;
  g.ld_out = p.ldr;
  g.out_n = (int)std::min<long>(p.leaf, e - mid);
  g.flops = 2.0 * g.M * g.N * (double)(mid - s);
  p.ops.push_back(g);
  p.op_k.push_back(mid - s);
  trsm_ops(p, split, mid, e);
}

// Tile plan of one TRSM op with contraction length K (leaf products skip the
// zero triangle of W^T).
std::vector<int4> op_tiles(const GemmCall& g, bool leaf, long K) {
  const int bn = gemm_bn(g.split);
  std::vector<int4> plan = plan_rect(g.M, g.N, bn, 0, (int)((K + kGemmBK - 1) / kGemmBK));
  if (leaf) {
    for (int4& t : plan) {
      const long lim = (long)t.y + bn;
      const long kmax = lim < K ? lim : K;
      t.w = (int)((kmax + kGemmBK - 1) / kGemmBK);
    }
  }
  return plan;
}

}  // namespace
}  // namespace tb

extern "C" tb_status tb_batch_destroy(tb_batch_t b) {
  if (!b) return TB_SUCCESS;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  cudaFree(b->scratch);
  cudaFree(b->tables);
  cudaSetDevice(cur);
  delete b;
  return TB_SUCCESS;
}

extern "C" tb_status tb_batch_create(tb_batch_t* out, int count, const int* kind, const long* n,
                                     const float* const* A, const long* lda, float* const* BC, const long* ldbc,
                                     long nb, int precision) {
  using namespace tb;
  if (!out || count < 0 || (count > 0 && (!kind || !n || !A || !lda || !BC || !ldbc))) return TB_ERROR_INVALID_VALUE;
  if (precision != TB_PREC_PLAIN && precision != TB_PREC_SPLIT) return TB_ERROR_INVALID_VALUE;
  *out = nullptr;
  for (int i = 0; i < count; ++i) {
    if ((kind[i] != 0 && kind[i] != 1) || n[i] < 0 || lda[i] < std::max<long>(n[i], 1) ||
        ldbc[i] < std::max<long>(n[i], 1) || n[i] > 65536)
      return TB_ERROR_INVALID_VALUE;
  }
  const Split split = precision == TB_PREC_SPLIT ? Split::kHiLo : Split::kPlain;
  const bool hilo = split == Split::kHiLo;
  tb_batch_s* b = new tb_batch_s();
  cudaGetDevice(&b->device);

  // ---- scratch layout
  Arena ar;
  struct SyrkPlan {
    long n;
    const float* A;
    long lda;
    float* C;
    long ldc;
    size_t off_h, off_l;
    long long ldh;
  };
  std::vector<SyrkPlan> syrks;
  std::vector<TrsmPlan> trsms;
  struct TrsmOff {
    size_t ah, al, xh, xl, wh, wl, rh, rl, d, wg;
  };
  std::vector<TrsmOff> toff;
  for (int i = 0; i < count; ++i) {
    const long ni = n[i];
    if (ni == 0) continue;
    const long long ldh = round_up(ni, 64);
    if (kind[i] == 0) {
      SyrkPlan s{ni, A[i], lda[i], BC[i], ldbc[i], 0, 0, ldh};
      s.off_h = ar.take((size_t)ldh * ni * 2);
      s.off_l = hilo ? ar.take((size_t)ldh * ni * 2) : 0;
      syrks.push_back(s);
    } else {
      TrsmPlan p;
      p.n = ni;
      p.A = A[i];
      p.lda = lda[i];
      p.B = BC[i];
      p.ldb = ldbc[i];
      p.leaf = leaf_for(ni, nb);
      for (long s = 0; s < ni; s += p.leaf) p.leaf_start.push_back(s);
      p.lda_h = ldh;
      p.ldx = ldh;
      p.ldw = p.leaf;
      p.wstride = p.ldw * p.leaf;
      p.ldr = ldh;
      TrsmOff o;
      o.ah = ar.take((size_t)ldh * ni * 2);
      const bool thilo = hilo || ni < 2048;  // effective precision of this instance's updates
      o.al = thilo ? ar.take((size_t)ldh * ni * 2) : 0;
      o.xh = ar.take((size_t)ldh * ni * 2);
      o.xl = thilo ? ar.take((size_t)ldh * ni * 2) : 0;
      o.wh = ar.take((size_t)p.wstride * p.leaf_start.size() * 2);
      o.wl = ar.take((size_t)p.wstride * p.leaf_start.size() * 2);
      o.rh = ar.take((size_t)ldh * p.leaf * 2);
      o.rl = ar.take((size_t)ldh * p.leaf * 2);
      o.d = ar.take((size_t)((ni + 31) / 32) * 1024 * sizeof(double));
      o.wg = ar.take((size_t)p.wstride * p.leaf_start.size() * sizeof(double));
      trsms.push_back(p);
      toff.push_back(o);
    }
  }
  if (ar.used > 0 && dev_malloc(&b->scratch, ar.used) != cudaSuccess) {
    cudaGetLastError();
    delete b;
    set_last_error("tb_batch_create: cannot allocate %zu bytes of scratch", ar.used);
    return TB_ERROR_ALLOC;
  }
  char* base = static_cast<char*>(b->scratch);
  auto H = [&](size_t off) { return reinterpret_cast<__half*>(base + off); };

  // ---- conversion, inverse and GEMM problem tables
  std::vector<ConvJob> conv;
  std::vector<DiagJob> diag;
  std::vector<ChainJob> chain;
  std::vector<GemmCall> probs;  // global problem list
  std::vector<int> prob_step, prob_leaf;
  std::vector<long> prob_k;
  long long conv_nblk = 0, diag_blocks = 0;
  auto add_conv = [&](const float* src, long long rows, long long cols, long long lds, __half* hi, __half* lo,
                      long long ldd, int tri) {
    conv.push_back(ConvJob{src, rows, cols, lds, hi, lo, ldd, tri, conv_nblk});
    conv_nblk += (rows * cols + kConvPerBlock - 1) / kConvPerBlock;
  };
  for (SyrkPlan& s : syrks) {
    add_conv(s.A, s.n, s.n, s.lda, H(s.off_h), hilo ? H(s.off_l) : nullptr, s.ldh, 0);
    GemmCall g;
    g.split = split;
    g.a_hi = {H(s.off_h), s.n, s.n, s.ldh, true};
    g.a_lo = {hilo ? H(s.off_l) : nullptr, s.n, s.n, s.ldh, true};
    g.b_hi = g.a_hi;
    g.b_lo = g.a_lo;
    g.C = s.C;
    g.ldc = s.ldc;
    g.M = g.N = (int)s.n;
    g.tri = 1;
    g.flops = (double)s.n * (double)(s.n + 1) * (double)s.n;
    probs.push_back(g);
    prob_step.push_back(0);
    prob_leaf.push_back(-1);  // SYRK: lower-triangle plan
    prob_k.push_back(s.n);
  }
  for (size_t t = 0; t < trsms.size(); ++t) {
    TrsmPlan& p = trsms[t];
    const TrsmOff& o = toff[t];
    p.ah = H(o.ah);
    const bool thilo = hilo || p.n < 2048;
    p.al = thilo ? H(o.al) : nullptr;
    p.xh = H(o.xh);
    p.xl = thilo ? H(o.xl) : nullptr;
    p.wh = H(o.wh);
    p.wl = H(o.wl);
    p.rh = H(o.rh);
    p.rl = H(o.rl);
    double* D = reinterpret_cast<double*>(base + o.d);
    if (p.leaf_start.size() > 1) add_conv(p.A, p.n, p.n, p.lda, p.ah, p.al, p.lda_h, 2);
    add_conv(p.B, p.n, std::min<long>(p.leaf, p.n), p.ldb, p.rh, p.rl, p.ldr, 0);  // first leaf's R
    diag.push_back(DiagJob{p.A, (long long)p.lda, (long long)p.n, D, diag_blocks});
    diag_blocks += (p.n + 31) / 32;
    for (size_t l = 0; l < p.leaf_start.size(); ++l) {
      const long s = p.leaf_start[l];
      chain.push_back(ChainJob{p.A, (long long)p.lda, (int)s, (int)std::min<long>(p.leaf, p.n - s), D,
                               p.wh + l * p.wstride, p.wl + l * p.wstride, p.ldw,
                               reinterpret_cast<double*>(base + o.wg) + l * p.wstride});
    }
    // as tb_strsm: orders below 2048 keep the reference's FP32 accuracy
    trsm_ops(p, (split == Split::kPlain && p.n < 2048) ? Split::kHiLo : split, 0, p.n);
    for (size_t q = 0; q < p.ops.size(); ++q) {
      probs.push_back(p.ops[q]);
      prob_step.push_back((int)q);
      prob_leaf.push_back((q % 2 == 0) ? 1 : 0);
      prob_k.push_back(p.op_k[q]);
    }
  }

  // ---- device tables: problems (64-byte aligned), then jobs and tiles
  const int nprob = (int)probs.size();
  std::vector<GemmArgs> hargs(nprob);
  for (int i = 0; i < nprob; ++i) {
    tb_status st = gemm_build_args(probs[i], &hargs[i]);
    if (st != TB_SUCCESS) {
      tb_batch_destroy(b);
      return st;
    }
  }
  int nsteps = 0;
  for (int s : prob_step) nsteps = std::max(nsteps, s + 1);
  // launches: per step, one for split problems and one for plain problems
  for (int st = 0; st < nsteps; ++st) {
    for (int sp = 0; sp < 2; ++sp) {
      Launch L;
      L.split = sp ? Split::kHiLo : Split::kPlain;
      for (int i = 0; i < nprob; ++i) {
        if (prob_step[i] != st || probs[i].split != L.split) continue;
        std::vector<int4> tiles =
            prob_leaf[i] < 0 ? plan_lower(probs[i].M, gemm_bn(L.split), 0, (probs[i].M + kGemmBK - 1) / kGemmBK)
                             : op_tiles(probs[i], prob_leaf[i] == 1, prob_k[i]);
        for (const int4& tt : tiles) {
          L.tiles.push_back(tt);
          L.prob.push_back(i);
        }
        L.flops += probs[i].flops;
      }
      if (L.tiles.empty()) continue;
      // longest K range first: CTAs claim tiles in this order as they free
      // up, so the short tiles fill the tail
      std::vector<int> order(L.tiles.size());
      for (size_t q = 0; q < order.size(); ++q) order[q] = (int)q;
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return L.tiles[x].w - L.tiles[x].z > L.tiles[y].w - L.tiles[y].z;
      });
      std::vector<int4> st_tiles(order.size());
      std::vector<int> st_prob(order.size());
      for (size_t q = 0; q < order.size(); ++q) {
        st_tiles[q] = L.tiles[order[q]];
        st_prob[q] = L.prob[order[q]];
      }
      L.tiles.swap(st_tiles);
      L.prob.swap(st_prob);
      b->launches.push_back(std::move(L));
    }
  }
  Arena tab;
  const size_t o_probs = tab.take(sizeof(GemmArgs) * std::max(nprob, 1));
  const size_t o_conv = tab.take(sizeof(ConvJob) * std::max<size_t>(conv.size(), 1));
  std::vector<int> blk_job((size_t)conv_nblk);
  for (size_t q = 0; q < conv.size(); ++q) {
    const long long e = q + 1 < conv.size() ? conv[q + 1].first : conv_nblk;
    for (long long x = conv[q].first; x < e; ++x) blk_job[(size_t)x] = (int)q;
  }
  const size_t o_blk = tab.take(sizeof(int) * std::max<size_t>(blk_job.size(), 1));
  const size_t o_diag = tab.take(sizeof(DiagJob) * std::max<size_t>(diag.size(), 1));
  const size_t o_chain = tab.take(sizeof(ChainJob) * std::max<size_t>(chain.size(), 1));
  const size_t o_sched = tab.take(sizeof(int) * std::max<size_t>(b->launches.size(), 1));
  std::vector<size_t> o_tiles, o_prob;
  for (Launch& L : b->launches) {
    o_tiles.push_back(tab.take(sizeof(int4) * L.tiles.size()));
    o_prob.push_back(tab.take(sizeof(int) * L.prob.size()));
  }
  if (dev_malloc(&b->tables, tab.used) != cudaSuccess) {
    cudaGetLastError();
    tb_batch_destroy(b);
    return TB_ERROR_ALLOC;
  }
  char* tb_ = static_cast<char*>(b->tables);
  std::vector<char> host(tab.used, 0);
  memcpy(host.data() + o_probs, hargs.data(), sizeof(GemmArgs) * nprob);
  memcpy(host.data() + o_conv, conv.data(), sizeof(ConvJob) * conv.size());
  memcpy(host.data() + o_blk, blk_job.data(), sizeof(int) * blk_job.size());
  memcpy(host.data() + o_diag, diag.data(), sizeof(DiagJob) * diag.size());
  memcpy(host.data() + o_chain, chain.data(), sizeof(ChainJob) * chain.size());
  b->d_problems = reinterpret_cast<GemmArgs*>(tb_ + o_probs);
  for (size_t l = 0; l < b->launches.size(); ++l) {
    Launch& L = b->launches[l];
    memcpy(host.data() + o_tiles[l], L.tiles.data(), sizeof(int4) * L.tiles.size());
    memcpy(host.data() + o_prob[l], L.prob.data(), sizeof(int) * L.prob.size());
    L.d_tiles = reinterpret_cast<int4*>(tb_ + o_tiles[l]);
    L.d_prob = reinterpret_cast<int*>(tb_ + o_prob[l]);
    L.d_sched = reinterpret_cast<int*>(tb_ + o_sched) + l;
  }
  b->d_sched = reinterpret_cast<int*>(tb_ + o_sched);
  if (cudaMemcpy(b->tables, host.data(), tab.used, cudaMemcpyHostToDevice) != cudaSuccess) {
    tb_batch_destroy(b);
    return TB_ERROR_CUDA;
  }
  b->d_conv = reinterpret_cast<ConvJob*>(tb_ + o_conv);
  b->d_blk_job = reinterpret_cast<int*>(tb_ + o_blk);
  b->nconv = (int)conv.size();
  b->conv_blocks = conv_nblk;
  b->d_diag = reinterpret_cast<DiagJob*>(tb_ + o_diag);
  b->ndiag = (int)diag.size();
  b->diag_blocks = diag_blocks;
  b->d_chain = reinterpret_cast<ChainJob*>(tb_ + o_chain);
  b->nchain = (int)chain.size();
  // one-time set-up that must not happen inside a stream capture
  device_error_word();
  sm_count();
  TB_TRY(gemm_prepare_grouped());
  TB_TRY(trsm_prepare_grouped());
  *out = b;
  return TB_SUCCESS;
}

extern "C" tb_status tb_batch_run(tb_batch_t b) {
  using namespace tb;
  if (!b) return TB_ERROR_INVALID_VALUE;
  cudaStream_t st = current_stream();
  if (b->nconv > 0 && b->conv_blocks > 0) {
    if (b->conv_blocks > 0x7fffffffLL) return TB_ERROR_NOT_SUPPORTED;
    conv_grouped_kernel<<<(unsigned)b->conv_blocks, 256, 0, st>>>(b->d_conv, b->d_blk_job);
    TB_CUDA_TRY(cudaGetLastError());
    note_launch();
  }
  TB_TRY(trsm_inverses_grouped(b->d_diag, b->ndiag, b->diag_blocks, b->d_chain, b->nchain, st));
  // the launches' tile counters start at zero on every run (a memset node
  // when the run is captured in a graph)
  if (!b->launches.empty()) TB_CUDA_TRY(cudaMemsetAsync(b->d_sched, 0, sizeof(int) * b->launches.size(), st));
  for (Launch& L : b->launches)
    TB_TRY(gemm_launch_grouped(L.split, b->d_problems, L.d_tiles, L.d_prob, (int)L.tiles.size(), L.flops, st,
                               L.d_sched));
  return TB_SUCCESS;
}
