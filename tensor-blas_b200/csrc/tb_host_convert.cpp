// FP32 -> FP16 conversion on the host cores (tb_host_s2h, and the
// host-memory SYRK's optional host-side conversion, TB_HOST_F16_EVERY):
// converting A's row panels before they cross PCIe halves the bytes the
// plain SYRK moves host -> device, and the device then reads the FP16 copy
// directly. The result is the IEEE-754 binary16 value nearest to
// each input, ties to even (the same as the device conversion kernels'
// __float2half_rn for every finite input, and for infinities).
//
// Columns of the panel are split over a small pool of worker threads that
// lives for the rest of the process. On x86 hosts with F16C the conversion
// uses VCVTPS2PH with round-to-nearest-even (eight values per instruction);
// elsewhere, and for the ragged end of a column, a portable bit-level
// conversion (below) gives the same results.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include "../../include/tb_capi.h"

namespace tb {
namespace {

// binary32 -> binary16, round to nearest, ties to even (IEEE 754-2008 5.4.2):
// normal results round the 13 dropped mantissa bits; results below 2^-14
// become subnormal (the value rounded to a multiple of 2^-24); overflow past
// the largest finite half (65504, i.e. at or above 65520 after rounding)
// gives infinity; NaN stays NaN (quiet).
uint16_t f32_to_f16_rn(float f) {
  uint32_t x;
  memcpy(&x, &f, 4);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u | ((ax >> 13) & 0x3ffu) : 0));
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // rounds to >= 2^16: infinity
  if (ax >= 0x38800000u) {                                    // normal half (>= 2^-14)
    const uint32_t mant = ax & 0x7fffffu;
    const uint32_t exp = (ax >> 23) - 127 + 15;
    uint32_t h = (exp << 10) | (mant >> 13);
    const uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;  // may carry into the exponent: still correct
    return (uint16_t)(sign | h);
  }
  if (ax < 0x33000000u) return (uint16_t)sign;  // below 2^-25: rounds to zero (2^-25 itself is a tie to 0)
  // subnormal half: value = m * 2^-24, m = round(ax_value * 2^24)
  const uint32_t e = ax >> 23;                          // biased exponent, 102 .. 112
  const uint32_t mant = (ax & 0x7fffffu) | 0x800000u;   // 24-bit significand
  const uint32_t shift = 126 - e;                       // 14 .. 24: value * 2^24 = mant >> shift
  uint32_t h = mant >> shift;
  const uint32_t rem = mant & ((1u << shift) - 1u), halfway = 1u << (shift - 1);
  if (rem > halfway || (rem == halfway && (h & 1u))) ++h;  // 0x400 (= 2^-14) if it rounds up to normal
  return (uint16_t)(sign | h);
}

void convert_scalar(const float* s, uint16_t* d, long n) {
  for (long i = 0; i < n; ++i) d[i] = f32_to_f16_rn(s[i]);
}

#if defined(__x86_64__)
__attribute__((target("avx,f16c"))) void convert_f16c(const float* s, uint16_t* d, long n) {
  long i = 0;
  for (; i + 8 <= n; i += 8) {
    const __m256 v = _mm256_loadu_ps(s + i);
    _mm_storeu_si128(reinterpret_cast<__m128i*>(d + i), _mm256_cvtps_ph(v, _MM_FROUND_TO_NEAREST_INT));
  }
  convert_scalar(s + i, d + i, n - i);
}
// TB_HOST_F16C=0 in the environment forces the portable path (read once).
bool has_f16c() {
  static const bool ok = [] {
    const char* e = getenv("TB_HOST_F16C");
    if (e && e[0] == '0') return false;
    return __builtin_cpu_supports("avx") && __builtin_cpu_supports("f16c");
  }();
  return ok;
}
#endif

void convert_run(const float* s, uint16_t* d, long n) {
#if defined(__x86_64__)
  if (has_f16c()) {
    convert_f16c(s, d, n);
    return;
  }
#endif
  convert_scalar(s, d, n);
}

// A fixed pool of worker threads running one job at a time: job(t, T) for
// t = 0 .. T-1, the caller taking part t = 0.
class Pool {
 public:
  static Pool& get() {
    static Pool p;
    return p;
  }
  int size() const { return (int)workers_.size() + 1; }
  void run(const std::function<void(int, int)>& job) {
    std::lock_guard<std::mutex> one(run_mu_);  // one job at a time
    const int T = size();
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &job;
      pending_ = T - 1;
      ++generation_;
    }
    cv_.notify_all();
    job(0, T);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  Pool() {
    unsigned hw = std::thread::hardware_concurrency();
    const int n = (int)std::min<unsigned>(hw > 1 ? hw : 1, 16u) - 1;
    for (int i = 0; i < n; ++i) workers_.emplace_back([this, i] { loop(i + 1); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
  }
  void loop(int t) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int, int)>* job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
        job = job_;
      }
      (*job)(t, size());
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (--pending_ == 0) done_cv_.notify_one();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_, run_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int, int)>* job_ = nullptr;
  int pending_ = 0;
  uint64_t generation_ = 0;
  bool stop_ = false;
};

}  // namespace

// rows x cols column-major FP32 (leading dimension lds) -> FP16 (ldd), on the
// host's cores.
void host_f32_to_f16(const float* src, long lds, long rows, long cols, uint16_t* dst, long ldd) {
  if (rows <= 0 || cols <= 0) return;
  Pool& pool = Pool::get();
  if ((double)rows * cols < 262144.0 || pool.size() == 1) {
    for (long j = 0; j < cols; ++j) convert_run(src + j * lds, dst + j * ldd, rows);
    return;
  }
  pool.run([&](int t, int T) {
    const long c0 = cols * t / T, c1 = cols * (t + 1) / T;
    for (long j = c0; j < c1; ++j) convert_run(src + j * lds, dst + j * ldd, rows);
  });
}

}  // namespace tb

extern "C" tb_status tb_host_s2h(long m, long n, const float* as, long ldas, void* ah, long ldah) {
  if (m < 0 || n < 0 || ldas < (m > 1 ? m : 1) || ldah < (m > 1 ? m : 1)) return TB_ERROR_INVALID_VALUE;
  if (m == 0 || n == 0) return TB_SUCCESS;
  if (!as || !ah) return TB_ERROR_INVALID_VALUE;
  tb::host_f32_to_f16(as, ldas, m, n, static_cast<uint16_t*>(ah), ldah);
  return TB_SUCCESS;
}
