// TRSM driver (reference: BLAS/tc_trsm.cu:31-174, tc_cumpsgemm_trsm.cu).
//
// Method (the reference's): recursive halving of the triangular operand.
// A node [s, e) solves its left half, applies the off-diagonal update
//   right side  B[:, mid:e] -= X[:, s:mid] * A[mid:e, s:mid]^T
//   left side   B[mid:e, :] -= A[mid:e, s:mid] * X[s:mid, :]
// as one FP16-operand / FP32-accumulate tensor-core GEMM, then solves its
// right half. Leaves are diagonal blocks of nb (<= 512) columns.
//
// B200 form of the pieces:
//  * A is converted to FP16 once (lower part only), not per level.
//  * X is converted exactly once, in the epilogue of the leaf product that
//    produces it (fused hi[/lo] copies), not re-converted at every level as
//    the reference does with B1 (BLAS/tc_trsm.cu:59-66).
//  * The leaf replaces FP32 cublasStrsm with X_b = B_b * inv(A_bb)^T (or
//    inv(A_bb) * B_b): inv(A_bb) is computed in FP64 by warp-level
//    substitution on 32x32 diagonal sub-blocks plus blocked 32-wide column
//    chains in shared memory, and applied with the split-FP16 3-product
//    tensor-core GEMM, i.e. FP32-level accuracy like the reference's leaf.
//  * Split points are multiples of 64 so every TMA coordinate stays aligned.
//    For n = nb * 2^L (the configured 16384 / 512) the leaves coincide with
//    the reference's recursion exactly.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "tb_convert.cuh"
#include "tb_internal.h"

namespace tb {

namespace {

constexpr int kLeafMax = 512;  // largest diagonal block inverted explicitly

// Inverse of each 32x32 diagonal sub-block of A (rows/cols >= n padded with
// the identity). One warp per sub-block; lane c owns column c of the inverse
// and runs forward substitution in FP64 registers; rows of L are broadcast
// from shared memory. Output: D[t*1024 + i + 32*c] (column-major 32x32).
template <class T>
__device__ __forceinline__ void diag_inv32_body(long long n, const T* __restrict__ A, long long lda,
                                                double* __restrict__ D, long long t, bool unit, double (*L)[33],
                                                int c) {
  const long long base = t * 32;
  for (int i = 0; i < 32; ++i) {
    const long long gi = base + i, gj = base + c;
    double v;
    if (gi < n && gj < n)
      v = (i > c || (i == c && !unit)) ? (double)A[gi + gj * lda] : (i == c ? 1.0 : 0.0);
    else
      v = (i == c) ? 1.0 : 0.0;
    L[i][c] = v;
  }
  __syncwarp();
  double w[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    double s = (i == c) ? 1.0 : 0.0;
#pragma unroll
    for (int p = 0; p < i; ++p) s -= L[i][p] * w[p];
    w[i] = (i < c) ? 0.0 : s / L[i][i];
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) D[t * 1024 + i + 32 * c] = w[i];
}

template <class T>
__global__ void __launch_bounds__(32) diag_inv32_kernel(long long n, const T* __restrict__ A, long long lda,
                                                        double* __restrict__ D, bool unit) {
  __shared__ double L[32][33];
  diag_inv32_body<T>(n, A, lda, D, blockIdx.x, unit, L, threadIdx.x);
}

// The preparation of a TRSM in one launch: FP32 -> FP16 conversions (A's
// lower part, and for the persistent solve the first leaf block of B), the
// 32 x 32 FP64 inverses of A's diagonal (warps 0..3 of a block, one
// sub-block each) and the zeroing of an int array (the persistent solve's
// progress counters), as consecutive ranges of one 1-D grid. Each job does
// exactly what its own kernel would (same element arithmetic).
struct PrepDev {
  PrepConv conv[2];
  int conv_vec[2];
  long long conv_gx[2], conv_base[2], conv_blocks[2];
  int nconv;
  const float* A;
  long long lda, n;
  double* D;
  int unit;
  long long diag_base, diag_blocks;
  int* zero;
  long long nzero, zero_base, zero_blocks;
};

constexpr int kPrepThreads = 256;

// Launches with the diagonal-inverse job get 4 x 32 x 33 doubles of dynamic
// shared memory (the conversion-only launches none, so their blocks pack
// densely on the SMs).
constexpr int kPrepDiagSmem = 4 * 32 * 33 * (int)sizeof(double);

__global__ void __launch_bounds__(kPrepThreads) trsm_prep_kernel(const __grid_constant__ PrepDev p) {
  extern __shared__ double prep_smem[];
  double(*L)[32][33] = reinterpret_cast<double(*)[32][33]>(prep_smem);
  const long long b = blockIdx.x;
  for (int z = 0; z < p.nconv; ++z)
    if (b >= p.conv_base[z] && b < p.conv_base[z] + p.conv_blocks[z]) {
      const long long local = b - p.conv_base[z], gx = p.conv_gx[z];
      const long long gy = p.conv_blocks[z] / gx;
      const PrepConv& c = p.conv[z];
      if (p.conv_vec[z])
        conv::convert8_body(local % gx, gx, local / gx, gy, c.rows, c.cols, c.src, c.lds, c.hi, c.lo, c.ldd, 2048.f,
                            c.tri, 0);
      else
        conv::convert1_body(local % gx, gx, local / gx, gy, c.rows, c.cols, c.src, c.lds, c.hi, c.lo, c.ldd, 2048.f,
                            c.tri, 0);
      return;
    }
  if (b >= p.diag_base && b < p.diag_base + p.diag_blocks) {
    const int warp = threadIdx.x >> 5;
    if (warp >= 4) return;
    const long long t = (b - p.diag_base) * 4 + warp;
    if (t * 32 < p.n) diag_inv32_body<float>(p.n, p.A, p.lda, p.D, t, p.unit != 0, L[warp], threadIdx.x & 31);
    return;
  }
  if (b >= p.zero_base && b < p.zero_base + p.zero_blocks) {
    for (long long i = (b - p.zero_base) * kPrepThreads + threadIdx.x; i < p.nzero; i += p.zero_blocks * kPrepThreads)
      p.zero[i] = 0;
  }
}

// Grouped form: block b belongs to the job whose [first, first + count)
// range of sub-blocks holds b (jobs sorted by `first`).
__global__ void __launch_bounds__(32) diag_inv32_grouped_kernel(const DiagJob* __restrict__ jobs, int njobs) {
  int lo = 0, hi = njobs - 1;
  const long long b = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (jobs[mid].first <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  const DiagJob& jb = jobs[lo];
  __shared__ double L[32][33];
  diag_inv32_body<float>(jb.n, jb.A, jb.lda, jb.D, b - jb.first, false, L, threadIdx.x);
}

// Column chain j of the inverse of leaf block b (rows/cols [s, s+size)):
//   W[i][j] = -Dinv_i * sum_{p=j}^{i-1} L[i][p] W[p][j]   (32x32 sub-blocks)
// The growing 32-wide column panel of W is kept in global memory (FP64,
// column-major, leading dimension ldg); each 32x32 sub-block of L, each W
// block and each Dinv_i is staged (transposed) through a 32 x 32 shared tile
// with coalesced loads, and each of the 128 threads owns a 2 x 4 block of
// the 32x32 result so every shared-memory load feeds several FMAs. A CTA
// needs ~27 KB of shared memory, so several share an SM and all panels of
// all leaves run concurrently. The result is written as the FP16 hi/lo pair
// (lo scaled by 2^11) of W with leading dimension ldw, or, without hi, the
// FP64 panel is W itself; zeros above the diagonal.
constexpr int kChainThreads = 128;

template <class T>
__device__ __forceinline__ void trtri_panel_body(const T* __restrict__ A, long long lda, int s, int size,
                                                 const double* __restrict__ D, __half* __restrict__ hi,
                                                 __half* __restrict__ lo, double* __restrict__ Wg, long long ldg,
                                                 long long ldw, int j) {
  // two staging buffers: sub-block p + 1 is loaded into registers while p's
  // products run, so each step of the chain waits on one barrier and its
  // global loads overlap the FMAs
  __shared__ __align__(16) double LsT[2][32][34];  // LsT[b][k][r] = L(r, k) of a staged sub-block (or Dinv_i)
  __shared__ __align__(16) double Ts[32][36];      // Ts[k][c]
  __shared__ __align__(16) double Wb[2][32][36];   // Wb[b][k][c] = W(32p + k, 32j + c)
  const int nsub = (size + 31) / 32;
  if (j >= nsub) return;
  const int tid = threadIdx.x;
  const int r0 = 2 * (tid & 15), c0 = 4 * (tid >> 4);  // 2 x 4 output block
  const int lr = tid & 31, lc = tid >> 5;              // load role: row lr, columns lc + 4q
  const long long sub0 = (long long)s / 32;
  double* Wp = Wg + (long long)(32 * j) * ldg;  // panel column 0 = leaf column 32j
  for (int q = 0; q < 8; ++q) {
    const int c = lc + 4 * q;
    Wp[32 * j + lr + c * ldg] = D[(sub0 + j) * 1024 + lr + 32 * c];
  }
  __syncthreads();
  for (int i = j + 1; i < nsub; ++i) {
    double acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    double ra[8], rw[8];
    auto fetch = [&](int p) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int cc = lc + 4 * q;
        const int gr = 32 * i + lr, gc = 32 * p + cc;
        ra[q] = (gr < size && gc < size) ? (double)A[(long long)s + gr + ((long long)s + gc) * lda] : 0.0;
        rw[q] = __ldcg(Wp + 32 * p + lr + (long long)cc * ldg);
      }
    };
    fetch(j);
    int bsel = 0;
    for (int p = j; p < i; ++p) {
      bsel = (p - j) & 1;
      // buffer bsel was last read in step p - 2, which every thread finished
      // before the barrier of step p - 1
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int cc = lc + 4 * q;
        LsT[bsel][cc][lr] = ra[q];
        Wb[bsel][lr][cc] = rw[q];
      }
      __syncthreads();
      if (p + 1 < i) fetch(p + 1);
#pragma unroll 4
      for (int kk = 0; kk < 32; ++kk) {
        const double2 l = *reinterpret_cast<const double2*>(&LsT[bsel][kk][r0]);
        const double2 w01 = *reinterpret_cast<const double2*>(&Wb[bsel][kk][c0]);
        const double2 w23 = *reinterpret_cast<const double2*>(&Wb[bsel][kk][c0 + 2]);
        acc[0][0] = fma(l.x, w01.x, acc[0][0]);
        acc[0][1] = fma(l.x, w01.y, acc[0][1]);
        acc[0][2] = fma(l.x, w23.x, acc[0][2]);
        acc[0][3] = fma(l.x, w23.y, acc[0][3]);
        acc[1][0] = fma(l.y, w01.x, acc[1][0]);
        acc[1][1] = fma(l.y, w01.y, acc[1][1]);
        acc[1][2] = fma(l.y, w23.x, acc[1][2]);
        acc[1][3] = fma(l.y, w23.y, acc[1][3]);
      }
    }
    // Ts was last read by the previous step's tail, behind its final barrier;
    // Dinv_i goes into the staging buffer the last product step did not read
    const int dsel = bsel ^ 1;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) Ts[r0 + a][c0 + b] = acc[a][b];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int cc = lc + 4 * q;
      LsT[dsel][cc][lr] = D[(sub0 + i) * 1024 + lr + 32 * cc];
    }
    __syncthreads();
    double o[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll 4
    for (int kk = 0; kk < 32; ++kk) {
      const double2 d = *reinterpret_cast<const double2*>(&LsT[dsel][kk][r0]);
      const double2 t01 = *reinterpret_cast<const double2*>(&Ts[kk][c0]);
      const double2 t23 = *reinterpret_cast<const double2*>(&Ts[kk][c0 + 2]);
      o[0][0] = fma(-d.x, t01.x, o[0][0]);
      o[0][1] = fma(-d.x, t01.y, o[0][1]);
      o[0][2] = fma(-d.x, t23.x, o[0][2]);
      o[0][3] = fma(-d.x, t23.y, o[0][3]);
      o[1][0] = fma(-d.y, t01.x, o[1][0]);
      o[1][1] = fma(-d.y, t01.y, o[1][1]);
      o[1][2] = fma(-d.y, t23.x, o[1][2]);
      o[1][3] = fma(-d.y, t23.y, o[1][3]);
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) Wp[32 * i + r0 + a + (long long)(c0 + b) * ldg] = o[a][b];
    __syncthreads();  // the new W block is visible to the CTA before it is staged
  }
  // columns [32j, 32j+32) of W for all rows of the leaf (zeros above the diagonal)
  for (int q = 0; q < 8; ++q) {
    const int c = lc + 4 * q;
    const int gc = 32 * j + c;
    if (gc >= size) continue;
    for (int row = lr; row < size; row += 32) {
      if (!hi) {
        if (row < 32 * j) Wp[row + (long long)c * ldg] = 0.0;  // FP64 output: the panel is W itself
        continue;
      }
      const double v = row >= 32 * j ? __ldcg(Wp + row + (long long)c * ldg) : 0.0;
      const __half h = __float2half_rn((float)v);
      hi[row + (long long)gc * ldw] = h;
      lo[row + (long long)gc * ldw] = __float2half_rn((float)((v - (double)__half2float(h)) * 2048.0));
    }
  }
}

__global__ void __launch_bounds__(kChainThreads) trtri_chain_kernel(const float* __restrict__ A, long long lda,
                                                                    const int2* __restrict__ leaves,
                                                                    const double* __restrict__ D,
                                                                    __half* __restrict__ Whi, __half* __restrict__ Wlo,
                                                                    long long ldw, long long wstride,
                                                                    double* __restrict__ Wg) {
  const int2 leaf = leaves[blockIdx.y];  // {s, size}
  trtri_panel_body<float>(A, lda, leaf.x, leaf.y, D, Whi + (long long)blockIdx.y * wstride,
                          Wlo + (long long)blockIdx.y * wstride, Wg + (long long)blockIdx.y * wstride, ldw, ldw,
                          blockIdx.x);
}

// FP64 operand, FP64 inverse (the Ozaki-scheme FP64 TRSM's leaves); the
// output W itself holds the panels.
__global__ void __launch_bounds__(kChainThreads) trtri_chain_f64_kernel(const double* __restrict__ A, long long lda,
                                                                        const int2* __restrict__ leaves,
                                                                        const double* __restrict__ D,
                                                                        double* __restrict__ W, long long ldw,
                                                                        long long wstride) {
  const int2 leaf = leaves[blockIdx.y];
  trtri_panel_body<double>(A, lda, leaf.x, leaf.y, D, nullptr, nullptr, W + (long long)blockIdx.y * wstride, ldw, ldw,
                           blockIdx.x);
}

// Grouped form: one job per (instance, leaf) along blockIdx.y.
__global__ void __launch_bounds__(kChainThreads) trtri_chain_grouped_kernel(const ChainJob* __restrict__ jobs) {
  const ChainJob& jb = jobs[blockIdx.y];
  trtri_panel_body<float>(jb.A, jb.lda, jb.s, jb.size, jb.D, jb.Whi, jb.Wlo, jb.Wg, jb.ldw, jb.ldw, blockIdx.x);
}


// Leaf block [s, e): X_b = B_b * W^T (right) or W * B_b (left), W = inv(A_bb),
// as a split-FP16 product. W is lower triangular, so each output tile only
// needs the K-blocks up to its own diagonal position. The FP16 hi/lo copy of
// B_b (R) was written by the epilogue of the update that last touched B_b,
// except for the first leaf, which converts it here.
tb_status leaf_solve(TrsmCtx& c, int bidx, long s, long e) {
  const long nbl = e - s;
  GemmCall g;
  g.split = Split::kHiLo;
  const bool split_x = c.split == Split::kHiLo;
  const bool need_convert = (s == 0) && !c.r0_ready;  // the set-up launch may have converted it
  if (c.right) {
    // R = B[:, s:e] (m x nbl) -> FP16 hi/lo; X_b = R * W^T
    if (need_convert) TB_TRY(convert_f32_f16(c.m, nbl, c.B + s * c.ldb, c.ldb, c.rh, c.rl, c.ldr, 2048.f, 0, c.st));
    g.a_hi = {c.rh, c.m, nbl, c.ldr, true};
    g.a_lo = {c.rl, c.m, nbl, c.ldr, true};
    g.b_hi = {c.wh + bidx * c.wstride, nbl, nbl, c.ldw, true};
    g.b_lo = {c.wl + bidx * c.wstride, nbl, nbl, c.ldw, true};
    g.C = c.B + s * c.ldb;
    g.ldc = c.ldb;
    g.M = (int)c.m;
    g.N = (int)nbl;
    g.out_hi = c.xh + s * c.ldx;
    g.out_lo = split_x ? c.xl + s * c.ldx : nullptr;
    g.ld_out = c.ldx;
  } else {
    // R = B[s:e, :] (nbl x n) -> FP16 hi/lo (K-major operand, rows = n); X_b = W * R
    if (need_convert) TB_TRY(convert_f32_f16(nbl, c.n, c.B + s, c.ldb, c.rh, c.rl, c.ldr, 2048.f, 0, c.st));
    g.a_hi = {c.wh + bidx * c.wstride, nbl, nbl, c.ldw, true};
    g.a_lo = {c.wl + bidx * c.wstride, nbl, nbl, c.ldw, true};
    g.b_hi = {c.rh, c.n, nbl, c.ldr, false};
    g.b_lo = {c.rl, c.n, nbl, c.ldr, false};
    g.C = c.B + s;
    g.ldc = c.ldb;
    g.M = (int)nbl;
    g.N = (int)c.n;
    g.out_hi = c.xh + s;
    g.out_lo = split_x ? c.xl + s : nullptr;
    g.ld_out = c.ldx;
  }
  g.alpha = 1.f;
  g.beta = 0.f;
  g.flops = (double)g.M * g.N * nbl;  // triangular solve of the leaf: other * nbl^2 flops
  g.kblocks = (int)((nbl + kGemmBK - 1) / kGemmBK);
  const int bn = gemm_bn(g.split, g.kblocks);
  std::vector<int4> plan = plan_rect(g.M, g.N, bn, 0, g.kblocks);
  for (int4& t : plan) {  // K (= columns of W) beyond the tile's last W row is zero
    const long lim = c.right ? (long)t.y + bn : (long)t.x + kGemmBM;
    const long kmax = lim < nbl ? lim : nbl;
    t.w = (int)((kmax + kGemmBK - 1) / kGemmBK);
  }
  return gemm_launch_plan(g, plan, c.st);  // uneven K ranges: host-balanced tile ranges
}

tb_status update(TrsmCtx& c, long s, long mid, long e) {
  GemmCall g;
  g.split = c.split;
  const bool hilo = c.split == Split::kHiLo;
  const long kk = mid - s;
  if (c.right) {
    // B[:, mid:e] -= X[:, s:mid] * A[mid:e, s:mid]^T
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
    // B[mid:e, :] -= A[mid:e, s:mid] * X[s:mid, :]
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
  // The next leaf is [mid, mid + leaf): this is the last update that touches
  // it, so its FP16 hi/lo copy is written here, fused into the epilogue.
  const long next = std::min<long>(c.leaf, e - mid);
  g.out_hi = c.rh;
  g.out_lo = c.rl;
  g.ld_out = c.ldr;
  if (c.right)
    g.out_n = (int)next;
  else
    g.out_m = (int)next;
  g.flops = 2.0 * g.M * g.N * kk;
  g.kblocks = (int)((kk + kGemmBK - 1) / kGemmBK);
  const std::vector<int4> plan = plan_rect(g.M, g.N, gemm_bn(g.split, g.kblocks), 0, g.kblocks);
  return gemm_launch_plan(g, plan, c.st);
}

tb_status recurse(TrsmCtx& c, long s, long e, const std::vector<long>& leaf_start) {
  if (e - s <= c.leaf) {
    const int bidx = (int)(std::lower_bound(leaf_start.begin(), leaf_start.end(), s) - leaf_start.begin());
    return leaf_solve(c, bidx, s, e);
  }
  // split at a leaf boundary near the middle (multiple of the leaf size)
  const long nleaves = (e - s + c.leaf - 1) / c.leaf;
  const long mid = s + ((nleaves + 1) / 2) * c.leaf;
  TB_TRY(recurse(c, s, mid, leaf_start));
  TB_TRY(update(c, s, mid, e));
  return recurse(c, mid, e, leaf_start);
}

}  // namespace

tb_status trsm_prepare_grouped() { return TB_SUCCESS; }

tb_status trsm_prep_launch(const PrepJobs& j, cudaStream_t st) {
  PrepDev p;
  memset(&p, 0, sizeof(p));
  long long next = 0;
  for (int z = 0; z < j.nconv; ++z) {
    const PrepConv& c = j.conv[z];
    if (c.rows <= 0 || c.cols <= 0) continue;
    const int k = p.nconv++;
    p.conv[k] = c;
    // the grid the conversion kernels would use (tb_convert.cu)
    const bool vec = (c.rows % 8 == 0) && (c.lds % 4 == 0) && (c.ldd % 8 == 0) &&
                     (reinterpret_cast<uintptr_t>(c.src) % 16 == 0) && (reinterpret_cast<uintptr_t>(c.hi) % 16 == 0) &&
                     (c.lo == nullptr || reinterpret_cast<uintptr_t>(c.lo) % 16 == 0);
    long long gx = 0, gy = 0;
    conv::convert_grid(c.rows, c.cols, c.tri, vec, sm_count(), kPrepThreads, &gx, &gy);
    p.conv_vec[k] = vec ? 1 : 0;
    p.conv_gx[k] = gx;
    p.conv_base[k] = next;
    p.conv_blocks[k] = gx * gy;
    next += gx * gy;
  }
  if (j.D && j.n > 0) {
    p.A = j.A;
    p.lda = j.lda;
    p.n = j.n;
    p.D = j.D;
    p.unit = j.unit ? 1 : 0;
    p.diag_base = next;
    p.diag_blocks = ((j.n + 31) / 32 + 3) / 4;
    next += p.diag_blocks;
  }
  if (j.zero && j.nzero > 0) {
    p.zero = j.zero;
    p.nzero = j.nzero;
    p.zero_base = next;
    p.zero_blocks = std::min<long long>((j.nzero + kPrepThreads - 1) / kPrepThreads, 64);
    next += p.zero_blocks;
  }
  if (next == 0) return TB_SUCCESS;
  if (next > 0x7fffffffLL) return TB_ERROR_NOT_SUPPORTED;
  trsm_prep_kernel<<<(unsigned)next, kPrepThreads, p.diag_blocks > 0 ? kPrepDiagSmem : 0, st>>>(p);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

// Diagonal-block inverses of many triangular matrices in two launches.
tb_status trsm_inverses_grouped(const DiagJob* d_diag, int ndiag, long long nblocks, const ChainJob* d_chain,
                                int nchain, cudaStream_t st) {
  if (ndiag > 0 && nblocks > 0) {
    diag_inv32_grouped_kernel<<<(unsigned)nblocks, 32, 0, st>>>(d_diag, ndiag);
    TB_CUDA_TRY(cudaGetLastError());
    note_launch();
  }
  if (nchain > 0) {
    trtri_chain_grouped_kernel<<<dim3(kLeafMax / 32, (unsigned)nchain), kChainThreads, 0, st>>>(d_chain);
    TB_CUDA_TRY(cudaGetLastError());
    note_launch();
  }
  return TB_SUCCESS;
}

// FP64 inverses of the diagonal leaf blocks of an FP64 lower-triangular
// matrix (order nt): leaf b = {s_b, size_b} (s_b a multiple of 32, size_b <=
// 512) gets W_b = inv(A[s_b:, s_b:]) at W + b * wstride (ld ldw, zeros above
// the diagonal). D: (nt + 31) / 32 * 1024 doubles of scratch; d_leaves: the
// leaves in device memory.
tb_status trsm_leaf_inverses_f64(long nt, const double* A, long lda, const int2* d_leaves, int nleaf, int max_size,
                                 double* D, double* W, long long ldw, long long wstride, cudaStream_t st, bool unit) {
  const long nsub = (nt + 31) / 32;
  diag_inv32_kernel<double><<<(unsigned)nsub, 32, 0, st>>>(nt, A, lda, D, unit);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  const int max_chain = (max_size + 31) / 32;
  trtri_chain_f64_kernel<<<dim3((unsigned)max_chain, (unsigned)nleaf), kChainThreads, 0, st>>>(A, lda, d_leaves, D, W,
                                                                                              ldw, wstride);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

// Set-up shared by every right-hand side of one triangular operand: scratch
// for B blocks of at most `m` rows (right side) / `n` columns (left side),
// the FP16 copy of A's lower part and the FP64 leaf inverses as FP16 hi/lo.
// `scratch`: device memory of trsm_scratch_bytes(...) bytes, or nullptr to
// take it from the pool.
namespace {
struct TrsmLayout {
  size_t o_ah, o_al, o_xh, o_xl, o_wh, o_wl, o_rh, o_rl, o_d, o_lv, o_wg, total;
};

TrsmLayout trsm_layout(TrsmCtx& c, long nleaf) {
  const long nt = c.nt;
  const bool hilo = c.split == Split::kHiLo;
  c.lda_h = round_up(nt, 64);
  // X copy: right: m x n, MN-major rows m; left: m x n col-major, K-major (K = m rows)
  c.ldx = round_up(c.m, 64);
  c.ldw = c.leaf;
  c.wstride = c.ldw * c.leaf;
  c.ldr = c.right ? round_up(c.m, 64) : c.leaf;
  const size_t a_bytes = (size_t)c.lda_h * nt * 2;
  const size_t x_bytes = (size_t)c.ldx * c.n * 2;
  const size_t w_bytes = (size_t)c.wstride * nleaf * 2;
  const size_t r_bytes = (size_t)c.ldr * (c.right ? c.leaf : c.n) * 2;
  const size_t d_bytes = (size_t)((nt + 31) / 32) * 1024 * sizeof(double);
  const size_t l_bytes = (size_t)nleaf * sizeof(int2);
  TrsmLayout L;
  size_t off = 0;
  auto take = [&](size_t b) {
    size_t o = off;
    off += round_up((long long)b, 256);
    return o;
  };
  L.o_ah = take(a_bytes);
  L.o_al = hilo ? take(a_bytes) : 0;
  L.o_xh = take(x_bytes);
  L.o_xl = hilo ? take(x_bytes) : 0;
  L.o_wh = take(w_bytes);
  L.o_wl = take(w_bytes);
  L.o_rh = take(r_bytes);
  L.o_rl = take(r_bytes);
  L.o_d = take(d_bytes);
  L.o_lv = take(l_bytes);
  L.o_wg = take((size_t)c.wstride * nleaf * sizeof(double));  // FP64 panels of the leaf inverses
  L.total = off;
  return L;
}
}  // namespace

tb_status trsm_setup(bool right, long m, long n, const float* A, long lda, long nb, Split split, cudaStream_t st,
                     void* scratch, TrsmCtx& c, std::vector<long>& leaf_start, bool unit, float* B, long ldb) {
  if (m < 0 || n < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  const long nt = right ? n : m;
  if (lda < (nt > 1 ? nt : 1)) return TB_ERROR_INVALID_VALUE;
  c.right = right;
  c.m = m;
  c.n = n;
  c.nt = nt;
  c.B = nullptr;
  c.ldb = 0;
  // The reference's chunk planner (util/mat_size.cu:31-55) sends an order
  // below 2048 to FP32 cublasStrsm with no FP16 step at all
  // (BLAS/tc_trsm.cu:103-112); the plain form keeps that accuracy contract
  // by using the FP32-accurate split products for such orders.
  c.split = (split == Split::kPlain && nt < 2048) ? Split::kHiLo : split;
  c.st = st;
  long leaf = round_up(std::min<long>(nb, kLeafMax), 64);
  if (leaf > kLeafMax) leaf = kLeafMax;
  c.leaf = (int)leaf;
  const bool hilo = c.split == Split::kHiLo;

  leaf_start.clear();
  std::vector<int2> leaves;
  for (long s = 0; s < nt; s += leaf) {
    leaf_start.push_back(s);
    leaves.push_back(make_int2((int)s, (int)std::min<long>(leaf, nt - s)));
  }
  const long nleaf = (long)leaves.size();
  const TrsmLayout L = trsm_layout(c, nleaf);
  char* ws = static_cast<char*>(scratch ? scratch : pool_get(L.total));
  if (!ws) {
    set_last_error("trsm: cannot allocate %zu bytes of scratch", L.total);
    return TB_ERROR_ALLOC;
  }
  c.ah = reinterpret_cast<__half*>(ws + L.o_ah);
  c.al = hilo ? reinterpret_cast<__half*>(ws + L.o_al) : nullptr;
  c.xh = reinterpret_cast<__half*>(ws + L.o_xh);
  c.xl = hilo ? reinterpret_cast<__half*>(ws + L.o_xl) : nullptr;
  c.wh = reinterpret_cast<__half*>(ws + L.o_wh);
  c.wl = reinterpret_cast<__half*>(ws + L.o_wl);
  c.rh = reinterpret_cast<__half*>(ws + L.o_rh);
  c.rl = reinterpret_cast<__half*>(ws + L.o_rl);
  double* D = reinterpret_cast<double*>(ws + L.o_d);
  int2* dleaves = reinterpret_cast<int2*>(ws + L.o_lv);
  double* W64 = reinterpret_cast<double*>(ws + L.o_wg);
  TB_CUDA_TRY(cudaMemcpyAsync(dleaves, leaves.data(), nleaf * sizeof(int2), cudaMemcpyHostToDevice, st));

  // 1. on the caller's stream, one conversion launch: the FP16 copy of A's
  // lower part (only off-diagonal leaf blocks are read) and, when B is known,
  // the first leaf's operand copy (the persistent solve's, with its zeroed
  // counters, when B takes that path)
  PrepJobs conv;
  if (nleaf > 1) {
    PrepConv& cv = conv.conv[conv.nconv++];
    cv.rows = nt;
    cv.cols = nt;
    cv.src = A;
    cv.lds = lda;
    cv.hi = c.ah;
    cv.lo = c.al;
    cv.ldd = c.lda_h;
    cv.tri = 2;
  }
  c.dag_prepped = false;
  c.r0_ready = false;
  if (B && trsm_dag_eligible(c, B, ldb)) {
    TB_TRY(trsm_dag_prepare(c, B, ldb, conv));
  } else if (B) {
    PrepConv& cv = conv.conv[conv.nconv++];
    const long nbl0 = std::min<long>(leaf, nt);
    cv.rows = right ? m : nbl0;
    cv.cols = right ? nbl0 : n;
    cv.src = B;
    cv.lds = ldb;
    cv.hi = c.rh;
    cv.lo = c.rl;
    cv.ldd = c.ldr;
    c.r0_ready = true;
  }
  // 2. beside it, on an auxiliary stream: the 32 x 32 FP64 inverses of A's
  // diagonal and the leaf chains (they read only A and each other), joined
  // back into the caller's stream before the solve
  const cudaStream_t sa = aux_stream(1);
  cudaEvent_t fork = nullptr, join = nullptr;
  if (sa) {
    TB_CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    TB_CUDA_TRY(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
  }
  const cudaStream_t si = sa ? sa : st;
  tb_status rs = TB_SUCCESS;
  if (sa && (cudaEventRecord(fork, st) != cudaSuccess || cudaStreamWaitEvent(sa, fork, 0) != cudaSuccess))
    rs = TB_ERROR_CUDA;
  if (rs == TB_SUCCESS) {
    PrepJobs inv;
    inv.A = A;
    inv.lda = lda;
    inv.n = nt;
    inv.D = D;
    inv.unit = unit;
    rs = trsm_prep_launch(inv, si);
  }
  if (rs == TB_SUCCESS) {
    const int max_chain = (int)(leaf / 32);
    dim3 grid((unsigned)max_chain, (unsigned)nleaf);
    trtri_chain_kernel<<<grid, kChainThreads, 0, si>>>(A, lda, dleaves, D, c.wh, c.wl, c.ldw, c.wstride, W64);
    if (cudaGetLastError() != cudaSuccess) rs = TB_ERROR_CUDA;
    note_launch();
  }
  if (rs == TB_SUCCESS) rs = trsm_prep_launch(conv, st);
  if (sa && (cudaEventRecord(join, sa) != cudaSuccess || cudaStreamWaitEvent(st, join, 0) != cudaSuccess) &&
      rs == TB_SUCCESS)
    rs = TB_ERROR_CUDA;
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
  return rs;
}

size_t trsm_scratch_bytes(bool right, long m, long n, long nb, Split split) {
  TrsmCtx c;
  c.right = right;
  c.m = m;
  c.n = n;
  c.nt = right ? n : m;
  c.split = (split == Split::kPlain && c.nt < 2048) ? Split::kHiLo : split;
  long leaf = round_up(std::min<long>(nb, kLeafMax), 64);
  c.leaf = (int)(leaf > kLeafMax ? kLeafMax : leaf);
  return trsm_layout(c, (c.nt + c.leaf - 1) / c.leaf).total;
}

// Solves one right-hand side block with a prepared context: B is m' x n
// (right side, m' <= the set-up m) or m x n' (left side, n' <= the set-up n):
// one persistent launch for all the recursion's products where B's layout
// allows it (tb_trsm_dag.cu), else one GEMM launch per leaf and update.
tb_status trsm_solve(TrsmCtx& c, const std::vector<long>& leaf_start, float* B, long ldb, long rows, long cols) {
  if (trsm_dag_eligible(c, B, ldb)) return trsm_solve_dag(c, leaf_start, B, ldb, rows, cols);
  return trsm_solve_launches(c, leaf_start, B, ldb, rows, cols);
}

tb_status trsm_solve_launches(TrsmCtx& c, const std::vector<long>& leaf_start, float* B, long ldb, long rows,
                              long cols) {
  if (ldb < (rows > 1 ? rows : 1)) return TB_ERROR_INVALID_VALUE;
  if (rows == 0 || cols == 0) return TB_SUCCESS;
  c.B = B;
  c.ldb = ldb;
  if (c.right)
    c.m = rows;
  else
    c.n = cols;
  return recurse(c, 0, c.nt, leaf_start);
}

tb_status trsm_solve_2s(TrsmCtx& c, const std::vector<long>& leaf_start, float* B, long ldb, long rows, long cols) {
  const long span = c.right ? rows : cols;  // independent systems
  // TB_TRSM_STREAMS in the environment: how many parts of B's independent
  // dimension are solved side by side on as many streams (1 to 4; read
  // once). Default 1: with the setup's preparation launches overlapped
  // (trsm_setup), plain m = n = 16384 nb 512 took 6.13 / 6.69 / 6.87 / 6.89 ms
  // with 1 / 2 / 3 / 4 parts on a B200 (6.47 / 7.03 / 7.20 / 7.22 on another):
  // a part's short launches cost as long as the whole solve's, so splitting
  // them adds latency. Plain products only: the split form's launches carry
  // three products per tile and never gained from parts.
  static const int streams = [] {
    const char* e = getenv("TB_TRSM_STREAMS");
    const int v = e ? atoi(e) : 0;
    return (v >= 1 && v <= 4) ? v : 1;
  }();
  if (trsm_dag_eligible(c, B, ldb)) return trsm_solve_dag(c, leaf_start, B, ldb, rows, cols);
  int parts = (c.split == Split::kPlain && span >= 4096) ? streams : 1;
  cudaStream_t sq[4] = {c.st, nullptr, nullptr, nullptr};
  for (int p = 1; p < parts; ++p)
    if (!(sq[p] = aux_stream(p - 1))) parts = 1;
  if (parts == 1 || ldb < (rows > 1 ? rows : 1)) return trsm_solve_launches(c, leaf_start, B, ldb, rows, cols);
  const long w = round_up((span + parts - 1) / parts, 128);
  cudaEvent_t fork, join[4];
  TB_CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  for (auto& e : join) TB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  tb_status rs = TB_SUCCESS;
  if (cudaEventRecord(fork, c.st) != cudaSuccess) rs = TB_ERROR_CUDA;
  // the parts after the first on the auxiliary streams, the first on the
  // caller's stream; X and R scratch are laid out along the split dimension
  for (int p = parts - 1; p >= 0 && rs == TB_SUCCESS; --p) {
    const long lo = std::min(span, p * w), hi = std::min(span, (p + 1) * w);
    if (hi <= lo) continue;
    TrsmCtx cp = c;
    cp.st = sq[p];
    const long long xo = c.right ? lo : (long long)lo * c.ldx;
    const long long ro = c.right ? lo : (long long)lo * c.ldr;
    cp.xh = c.xh + xo;
    cp.xl = c.xl ? c.xl + xo : nullptr;
    cp.rh = c.rh + ro;
    cp.rl = c.rl + ro;
    if (p > 0 && cudaStreamWaitEvent(sq[p], fork, 0) != cudaSuccess) {
      rs = TB_ERROR_CUDA;
      break;
    }
    rs = c.right ? trsm_solve_launches(cp, leaf_start, B + lo, ldb, hi - lo, cols)
                 : trsm_solve_launches(cp, leaf_start, B + lo * ldb, ldb, rows, hi - lo);
    if (p > 0 && (cudaEventRecord(join[p], sq[p]) != cudaSuccess || cudaStreamWaitEvent(c.st, join[p], 0) != cudaSuccess))
      rs = TB_ERROR_CUDA;
  }
  cudaEventDestroy(fork);
  for (auto& e : join) cudaEventDestroy(e);
  return rs;
}

tb_status trsm_impl(bool right, long m, long n, const float* A, long lda, float* B, long ldb, long nb, Split split,
                    cudaStream_t st) {
  if (m < 0 || n < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  const long nt = right ? n : m;
  if (lda < (nt > 1 ? nt : 1) || ldb < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  TrsmCtx c;
  std::vector<long> leaf_start;
  TB_TRY(trsm_setup(right, m, n, A, lda, nb, split, st, nullptr, c, leaf_start, false, B, ldb));
  const tb_status rs = trsm_solve_2s(c, leaf_start, B, ldb, m, n);
  c.r0_ready = false;
  return rs;
}


// ------------------------------------------------------------------ all BLAS flag combinations
// The two solved forms (left/lower/no-trans and right/lower/trans) cover the
// other six through index maps: with J the order reversal,
//   op(A) lower in a left solve  -> L = op(A)           (A^T copied when op(A) = U^T)
//   op(A) upper in a left solve  -> J op(A) J is lower: J X = solve(J op(A) J, J B)
//   op(A) upper in a right solve -> A' = op(A)^T lower  (native when op(A) = L^T)
//   op(A) lower in a right solve -> X J (J op(A) J) = B J with J op(A) J = A'^T,
//                                   A' = J op(A)^T J lower
// The remapped lower triangle is copied once into scratch; B's rows (left)
// or columns (right) are reversed in place around the solve when J appears.
namespace {
__global__ void tri_remap_kernel(long long n, const float* __restrict__ src, long long lds, float* __restrict__ dst,
                                 long long ldd, int transpose, int reverse) {
  for (long long j = blockIdx.y; j < n; j += gridDim.y)
    for (long long i = j + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
      const long long si = reverse ? n - 1 - i : i, sj = reverse ? n - 1 - j : j;
      dst[i + j * ldd] = transpose ? src[sj + si * lds] : src[si + sj * lds];
    }
}

// Reverses the order of the rows (cols == 0) or the columns (cols == 1) of
// an m x n column-major matrix in place.
__global__ void reverse_kernel(long long m, long long n, float* __restrict__ B, long long ldb, int cols) {
  const long long pairs = cols ? n / 2 : m / 2, other = cols ? m : n;
  for (long long q = blockIdx.y; q < other; q += gridDim.y)
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < pairs;
         p += (long long)gridDim.x * blockDim.x) {
      float* x = cols ? B + q + p * ldb : B + p + q * ldb;
      float* y = cols ? B + q + (n - 1 - p) * ldb : B + (m - 1 - p) + q * ldb;
      const float t = *x;
      *x = *y;
      *y = t;
    }
}

tb_status reverse(long long m, long long n, float* B, long long ldb, bool cols, cudaStream_t st) {
  const long long pairs = cols ? n / 2 : m / 2, other = cols ? m : n;
  if (pairs == 0 || other == 0) return TB_SUCCESS;
  dim3 g((unsigned)std::min<long long>((pairs + 255) / 256, 256), (unsigned)std::min<long long>(other, 65535));
  reverse_kernel<<<g, 256, 0, st>>>(m, n, B, ldb, cols ? 1 : 0);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}
}  // namespace

// Plain solve plus one refinement sweep: X0 = plain TRSM(B); R = B - op(A) X0
// with the FP32-accurate split products (the residual is ~1e-4 of B, so its
// own error stays ~1e-7 of B); D = plain TRSM(R); X = X0 + D. The correction
// carries the plain solve's relative error (~1e-4) on a quantity ~1e-4 the
// size of X, so X reaches FP32-level accuracy.
namespace {
__global__ void add_kernel(long long m, long long n, float* __restrict__ X, long long ldx, const float* __restrict__ D,
                           long long ldd) {
  for (long long j = blockIdx.y; j < n; j += gridDim.y)
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
      X[i + j * ldx] += D[i + j * ldd];
}
}  // namespace

tb_status trsm_refine_impl(bool right, long m, long n, const float* A, long lda, float* B, long ldb, long nb,
                           cudaStream_t st) {
  if (m < 0 || n < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  const long nt = right ? n : m;
  if (lda < (nt > 1 ? nt : 1) || ldb < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  const size_t bytes = (size_t)m * n * sizeof(float);
  float* R = static_cast<float*>(pool_get(bytes, 1));
  if (!R) {
    set_last_error("trsm refine: cannot allocate %zu bytes for the residual", bytes);
    return TB_ERROR_ALLOC;
  }
  TB_CUDA_TRY(cudaMemcpy2DAsync(R, (size_t)m * 4, B, (size_t)ldb * 4, (size_t)m * 4, (size_t)n,
                                cudaMemcpyDeviceToDevice, st));
  TB_TRY(trsm_impl(right, m, n, A, lda, B, ldb, nb, Split::kPlain, st));
  // R = B0 - op(A) X0 (left: A X0; right: X0 A^T)
  TB_TRY(trmm_ex_impl(right, false, right, false, m, n, -1.f, A, lda, B, ldb, R, m, Split::kHiLo, nullptr, 0, st,
                      1.f));
  TB_TRY(trsm_impl(right, m, n, A, lda, R, m, nb, Split::kPlain, st));
  dim3 g((unsigned)std::min<long long>((m + 255) / 256, 64), (unsigned)std::min<long>(n, 65535));
  add_kernel<<<g, 256, 0, st>>>(m, n, B, ldb, R, m);
  TB_CUDA_TRY(cudaGetLastError());
  note_launch();
  return TB_SUCCESS;
}

tb_status trsm_ex_impl(bool right, bool upper, bool trans, bool unit, long m, long n, const float* A, long lda,
                       float* B, long ldb, long nb, Split split, cudaStream_t st) {
  if (m < 0 || n < 0 || nb <= 0) return TB_ERROR_INVALID_VALUE;
  const long nt = right ? n : m;
  if (lda < (nt > 1 ? nt : 1) || ldb < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  const bool op_lower = upper == trans;
  bool tr = false, rev = false;  // how A' is read from A
  if (!right) {
    tr = trans;  // (L,N): as is; (U,T): A^T; (U,N): J A J; (L,T): J A^T J
    rev = !op_lower;
  } else {
    tr = !trans;  // (L,T): as is; (U,N): A^T; (L,N): J A^T J; (U,T): J A J
    rev = op_lower;
  }
  const bool copy = tr || rev;
  const long long ldc_ = round_up(nt, 4);
  const size_t copy_bytes = copy ? (size_t)round_up(ldc_ * nt * 4, 256) : 0;
  const size_t need = copy_bytes + trsm_scratch_bytes(right, m, n, nb, split);
  char* ws = static_cast<char*>(pool_get(need));
  if (!ws) {
    set_last_error("trsm: cannot allocate %zu bytes of scratch", need);
    return TB_ERROR_ALLOC;
  }
  const float* Ause = A;
  long ldause = lda;
  if (copy) {
    float* Ac = reinterpret_cast<float*>(ws);
    dim3 g((unsigned)std::min<long long>((nt + 255) / 256, 64), (unsigned)std::min<long long>(nt, 65535));
    tri_remap_kernel<<<g, 256, 0, st>>>(nt, A, lda, Ac, ldc_, tr ? 1 : 0, rev ? 1 : 0);
    TB_CUDA_TRY(cudaGetLastError());
    note_launch();
    Ause = Ac;
    ldause = (long)ldc_;
  }
  if (rev) TB_TRY(reverse(m, n, B, ldb, right, st));
  TrsmCtx c;
  std::vector<long> leaf_start;
  TB_TRY(trsm_setup(right, m, n, Ause, ldause, nb, split, st, ws + copy_bytes, c, leaf_start, unit, B, ldb));
  TB_TRY(trsm_solve_2s(c, leaf_start, B, ldb, m, n));
  c.r0_ready = false;
  if (rev) TB_TRY(reverse(m, n, B, ldb, right, st));
  return TB_SUCCESS;
}

}  // namespace tb

extern "C" tb_status tb_strsm(char side, long m, long n, const float* A, long lda, float* B, long ldb, long nb,
                              int precision) {
  if (nb == TB_NB_AUTO) return tb::auto_strsm(side, m, n, A, lda, B, ldb, precision);
  bool right;
  if (side == 'R' || side == 'r')
    right = true;
  else if (side == 'L' || side == 'l')
    right = false;
  else
    return TB_ERROR_INVALID_VALUE;
  if (precision == TB_PREC_REFINE) return tb::trsm_refine_impl(right, m, n, A, lda, B, ldb, nb, tb::current_stream());
  if (precision != TB_PREC_PLAIN && precision != TB_PREC_SPLIT) return TB_ERROR_INVALID_VALUE;
  return tb::trsm_impl(right, m, n, A, lda, B, ldb, nb,
                       precision == TB_PREC_SPLIT ? tb::Split::kHiLo : tb::Split::kPlain, tb::current_stream());
}

extern "C" tb_status tb_strsm_ex(char side, char uplo, char transa, char diag, long m, long n, const float* A,
                                 long lda, float* B, long ldb, long nb, int precision) {
  auto flag = [](char c, char a, char b, bool* v) {
    if (c == a || c == a + ('a' - 'A')) {
      *v = false;
      return true;
    }
    if (c == b || c == b + ('a' - 'A')) {
      *v = true;
      return true;
    }
    return false;
  };
  bool right, upper, trans, unit;
  if (!flag(side, 'L', 'R', &right) || !flag(uplo, 'L', 'U', &upper) || !flag(diag, 'N', 'U', &unit))
    return TB_ERROR_INVALID_VALUE;
  if (!flag(transa, 'N', 'T', &trans) && !flag(transa, 'N', 'C', &trans)) return TB_ERROR_INVALID_VALUE;
  if (precision != TB_PREC_PLAIN && precision != TB_PREC_SPLIT) return TB_ERROR_INVALID_VALUE;
  return tb::trsm_ex_impl(right, upper, trans, unit, m, n, A, lda, B, ldb, nb,
                          precision == TB_PREC_SPLIT ? tb::Split::kHiLo : tb::Split::kPlain, tb::current_stream());
}

// ------------------------------------------------------------------ reference C++ API
#include "../../include/TensorBLAS.h"

void tc_trsm(cublasHandle_t, long int m, long int n, float* A, long int lda, float* B, long int ldb, __half*,
             long int nb) {
  tb_status s = tb::trsm_impl(true, m, n, A, lda, B, ldb, nb, tb::Split::kPlain, tb::current_stream());
  if (s != TB_SUCCESS) fprintf(stderr, "TensorBLAS tc_trsm: %s %s\n", tb_status_string(s), tb_last_error());
}

void tc_cumpsgemm_trsm(cublasHandle_t, cumpsgemm::handle_t, long int m, long int n, float* A, long int lda, float* B,
                       long int ldb, long int nb) {
  tb_status s = tb::trsm_impl(true, m, n, A, lda, B, ldb, nb, tb::Split::kHiLo, tb::current_stream());
  if (s != TB_SUCCESS) fprintf(stderr, "TensorBLAS tc_cumpsgemm_trsm: %s %s\n", tb_status_string(s), tb_last_error());
}
