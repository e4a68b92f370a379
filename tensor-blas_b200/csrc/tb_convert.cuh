// FP32 -> FP16 conversion bodies shared by the conversion kernels
// (tb_convert.cu) and the TRSM preparation kernel (tb_trsm.cu), which runs
// several conversions and the 32 x 32 inverses as block ranges of one grid.
// A body covers the matrix with blocks (bx, by) of a gx x gy grid of
// blockDim.x threads; the element arithmetic is the conversion kernels'.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

namespace tb {
namespace conv {

__device__ __forceinline__ float4 ld_stream(const float* p) {
  float4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}

__device__ __forceinline__ uint32_t pack2(__half a, __half b) {
  return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}

// Band of the triangle modes 4 / 5: a GEMM tile of at most 256 rows whose K
// range starts (upper) or ends (lower) at its own diagonal block reads the
// other triangle only within 256 of the diagonal.
constexpr long long kTriBand = 256;

// Eight converted values of one column to hi (and lo), and their copies `dup`
// elements further on.
__device__ __forceinline__ void store8(const float* f, __half* __restrict__ hi, __half* __restrict__ lo,
                                       long long off, long long dup, float lo_scale) {
  __half h[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) h[e] = __float2half_rn(f[e]);
  uint4 o;
  o.x = pack2(h[0], h[1]);
  o.y = pack2(h[2], h[3]);
  o.z = pack2(h[4], h[5]);
  o.w = pack2(h[6], h[7]);
  *reinterpret_cast<uint4*>(hi + off) = o;
  if (dup) *reinterpret_cast<uint4*>(hi + dup + off) = o;
  if (lo) {
    __half l[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) l[e] = __float2half_rn((f[e] - __half2float(h[e])) * lo_scale);
    uint4 q;
    q.x = pack2(l[0], l[1]);
    q.y = pack2(l[2], l[3]);
    q.z = pack2(l[4], l[5]);
    q.w = pack2(l[6], l[7]);
    *reinterpret_cast<uint4*>(lo + off) = q;
    if (dup) *reinterpret_cast<uint4*>(lo + dup + off) = q;
  }
}

// Vector path: rows % 8 == 0, lds % 4 == 0, ldd % 8 == 0, 16-byte aligned bases.
// Whole matrices (tri 0): a thread owns 8 rows and walks the columns by,
// by + gy, ... four at a time, with the four columns' loads (128 bytes) in
// flight together; grids of a few blocks per SM then keep enough bytes in
// flight to run at the HBM rate.
__device__ __forceinline__ void convert8_body(long long bx, long long gx, long long by, long long gy, long long rows,
                                              long long cols, const float* __restrict__ src, long long lds,
                                              __half* __restrict__ hi, __half* __restrict__ lo, long long ldd,
                                              float lo_scale, int tri, long long dup) {
  const long long rows8 = rows >> 3;
  if (tri == 2) {
    // lower part: row group v (rows 8v .. 8v + 7) has the columns j < 8v + 8.
    // A thread takes row groups t and rows8 - 1 - t, so every thread has
    // about the same number of columns, and walks them four at a time.
    const long long half = (rows8 + 1) >> 1;
    for (long long t = bx * blockDim.x + threadIdx.x; t < half; t += gx * blockDim.x) {
      for (int w = 0; w < 2; ++w) {
        const long long v = w ? rows8 - 1 - t : t;
        if (w && v == t) break;
        const long long i = v << 3, jend = min(cols, i + 8);
        long long j = by;
        for (; j + 3 * gy < jend; j += 4 * gy) {
          float4 a[4], b[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float* s = src + i + (j + u * gy) * lds;
            a[u] = ld_stream(s);
            b[u] = ld_stream(s + 4);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float f[8] = {a[u].x, a[u].y, a[u].z, a[u].w, b[u].x, b[u].y, b[u].z, b[u].w};
            store8(f, hi, lo, i + (j + u * gy) * ldd, dup, lo_scale);
          }
        }
        for (; j < jend; j += gy) {
          const float* s = src + i + j * lds;
          const float4 a = ld_stream(s), b = ld_stream(s + 4);
          const float f[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
          store8(f, hi, lo, i + j * ldd, dup, lo_scale);
        }
      }
    }
    return;
  }
  if (tri == 0) {
    for (long long v = bx * blockDim.x + threadIdx.x; v < rows8; v += gx * blockDim.x) {
      const long long i = v << 3;
      long long j = by;
      for (; j + 3 * gy < cols; j += 4 * gy) {
        float4 a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float* s = src + i + (j + u * gy) * lds;
          a[u] = ld_stream(s);
          b[u] = ld_stream(s + 4);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float f[8] = {a[u].x, a[u].y, a[u].z, a[u].w, b[u].x, b[u].y, b[u].z, b[u].w};
          store8(f, hi, lo, i + (j + u * gy) * ldd, dup, lo_scale);
        }
      }
      for (; j < cols; j += gy) {
        const float* s = src + i + j * lds;
        const float4 a = ld_stream(s), b = ld_stream(s + 4);
        const float f[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        store8(f, hi, lo, i + j * ldd, dup, lo_scale);
      }
    }
    return;
  }
  for (long long j = by; j < cols; j += gy) {
    long long v0 = bx * blockDim.x + threadIdx.x, vend = rows8;
    if (tri == 2) v0 += (j >> 3);  // rows i >= j (rounded down to 8)
    if (tri == 4) vend = min(rows8, (j / kTriBand + 1) * (kTriBand / 8));  // rows i < band end
    if (tri == 5) v0 += (j / kTriBand) * (kTriBand / 8);                   // rows i >= band start
    for (long long v = v0; v < vend; v += gx * blockDim.x) {
      const long long i = v << 3;
      const float* s = src + i + j * lds;
      const float4 a = ld_stream(s), b = ld_stream(s + 4);
      float f[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      if (tri == 1 || tri == 5) {
#pragma unroll
        for (int e = 0; e < 8; ++e)
          if (i + e < j) f[e] = 0.f;
      } else if (tri == 3 || tri == 4) {
#pragma unroll
        for (int e = 0; e < 8; ++e)
          if (i + e > j) f[e] = 0.f;
      }
      store8(f, hi, lo, i + j * ldd, dup, lo_scale);
    }
  }
}

// Grid (gx, gy) of convert8_body / convert1_body for a rows x cols operand:
// whole matrices and lower parts on the vector path take about 16 blocks of
// 256 threads per SM, each thread walking many columns; the other forms one
// column per block row.
inline void convert_grid(long long rows, long long cols, int tri, bool vec, int sms, int threads, long long* gx,
                         long long* gy) {
  long long units = vec ? rows / 8 : rows;
  if (vec && tri == 2) units = (units + 1) / 2;  // two row groups per thread
  long long x = (units + threads - 1) / threads;
  if (x > 1024) x = 1024;
  long long y = cols < 65535 ? cols : 65535;
  if (vec && (tri == 0 || tri == 2)) {
    const long long want = (16LL * sms + x - 1) / x;
    y = want < y ? want : y;
    if (y < 1) y = 1;
  }
  *gx = x;
  *gy = y;
}

// Scalar fallback for ragged or unaligned shapes.
__device__ __forceinline__ void convert1_body(long long bx, long long gx, long long by, long long gy, long long rows,
                                              long long cols, const float* __restrict__ src, long long lds,
                                              __half* __restrict__ hi, __half* __restrict__ lo, long long ldd,
                                              float lo_scale, int tri, long long dup) {
  for (long long j = by; j < cols; j += gy) {
    long long i0 = bx * blockDim.x + threadIdx.x, iend = rows;
    if (tri == 2) i0 += (j >> 3) << 3;
    if (tri == 4) iend = min(rows, (j / kTriBand + 1) * kTriBand);
    if (tri == 5) i0 += (j / kTriBand) * kTriBand;
    for (long long i = i0; i < iend; i += gx * blockDim.x) {
      float f = src[i + j * lds];
      if (((tri == 1 || tri == 5) && i < j) || ((tri == 3 || tri == 4) && i > j)) f = 0.f;
      const __half h = __float2half_rn(f);
      hi[i + j * ldd] = h;
      if (dup) hi[dup + i + j * ldd] = h;
      if (lo) {
        const __half l = __float2half_rn((f - __half2float(h)) * lo_scale);
        lo[i + j * ldd] = l;
        if (dup) lo[dup + i + j * ldd] = l;
      }
    }
  }
}

}  // namespace conv
}  // namespace tb
