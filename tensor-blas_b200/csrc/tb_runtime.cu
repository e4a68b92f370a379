// Library runtime: status strings, per-thread error text, the current stream,
// the per-device scratch pool and the device error word used by the bounded
// waits of the persistent kernels.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "tb_internal.h"

namespace tb {

namespace {
thread_local char g_last_error[512] = "";
cudaStream_t g_stream = nullptr;

constexpr int kMaxDevices = 64;
struct DeviceState {
  void* pool[kPoolSlots] = {};
  size_t pool_bytes[kPoolSlots] = {};
  int* err = nullptr;
  int sms = 0;
  cudaStream_t aux = nullptr;
};
DeviceState g_dev[kMaxDevices];
std::mutex g_mu;

DeviceState* state() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) return nullptr;
  return &g_dev[d];
}
}  // namespace

// ------------------------------------------------------------------ accounting
namespace {
std::atomic<unsigned long long> g_launches{0};
struct ProfRec {
  cudaEvent_t a, b;
  double flops;
};
bool g_prof_on = false;
std::vector<ProfRec> g_prof_live;     // recorded since tb_profile_begin
std::vector<cudaEvent_t> g_ev_free;  // recycled events
cudaEvent_t ev_get() {
  if (!g_ev_free.empty()) {
    cudaEvent_t e = g_ev_free.back();
    g_ev_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

void note_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

bool profiling() { return g_prof_on; }

void* prof_begin(cudaStream_t st) {
  if (!g_prof_on) return nullptr;
  ProfRec r;
  r.a = ev_get();
  r.b = ev_get();
  r.flops = 0;
  cudaEventRecord(r.a, st);
  g_prof_live.push_back(r);
  return reinterpret_cast<void*>(g_prof_live.size());
}

void prof_end(void* token, cudaStream_t st, double flops) {
  if (!token) return;
  ProfRec& r = g_prof_live[reinterpret_cast<size_t>(token) - 1];
  cudaEventRecord(r.b, st);
  r.flops = flops;
}

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

tb_status cuda_status(cudaError_t e) {
  set_last_error("CUDA error %d: %s", (int)e, cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return TB_ERROR_ALLOC;
  return TB_ERROR_CUDA;
}

cudaStream_t current_stream() { return g_stream; }

cudaStream_t aux_stream() {
  DeviceState* s = state();
  if (!s) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!s->aux && cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    s->aux = nullptr;
  }
  return s->aux;
}

int sm_count() {
  DeviceState* s = state();
  if (!s) return 148;
  if (s->sms == 0) {
    int d = 0, n = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
    s->sms = n > 0 ? n : 148;
  }
  return s->sms;
}

void* pool_get(size_t bytes, int slot) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState* s = state();
  if (!s || slot < 0 || slot >= kPoolSlots) return nullptr;
  if (bytes == 0) bytes = 256;
  if (s->pool_bytes[slot] >= bytes) return s->pool[slot];
  if (s->pool[slot]) {
    cudaDeviceSynchronize();  // work queued on the old buffer must finish
    cudaFree(s->pool[slot]);
    s->pool[slot] = nullptr;
    s->pool_bytes[slot] = 0;
  }
  size_t want = (size_t)round_up((long long)bytes, 1 << 20);
  if (cudaMalloc(&s->pool[slot], want) != cudaSuccess) {
    cudaGetLastError();
    s->pool[slot] = nullptr;
    return nullptr;
  }
  s->pool_bytes[slot] = want;
  return s->pool[slot];
}

int* device_error_word() {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState* s = state();
  if (!s) return nullptr;
  if (!s->err) {
    if (cudaMalloc(&s->err, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    cudaMemset(s->err, 0, sizeof(int));
  }
  return s->err;
}

tb_status check_device_error(cudaStream_t stream) {
  int* w = device_error_word();
  TB_CUDA_TRY(cudaStreamSynchronize(stream));
  if (!w) return TB_SUCCESS;
  int h = 0;
  TB_CUDA_TRY(cudaMemcpy(&h, w, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) {
    cudaMemset(w, 0, sizeof(int));
    set_last_error("device-side bounded wait timed out (code %d)", h);
    return TB_ERROR_TIMEOUT;
  }
  return TB_SUCCESS;
}

}  // namespace tb

extern "C" {

tb_status tb_set_stream(void* stream) {
  tb::g_stream = static_cast<cudaStream_t>(stream);
  return TB_SUCCESS;
}

void* tb_get_stream(void) { return tb::g_stream; }

const char* tb_status_string(tb_status s) {
  switch (s) {
    case TB_SUCCESS: return "TB_SUCCESS";
    case TB_ERROR_INVALID_VALUE: return "TB_ERROR_INVALID_VALUE";
    case TB_ERROR_ALLOC: return "TB_ERROR_ALLOC";
    case TB_ERROR_CUDA: return "TB_ERROR_CUDA";
    case TB_ERROR_TIMEOUT: return "TB_ERROR_TIMEOUT";
    case TB_ERROR_NOT_SUPPORTED: return "TB_ERROR_NOT_SUPPORTED";
  }
  return "TB_UNKNOWN_STATUS";
}

const char* tb_last_error(void) { return tb::g_last_error; }

tb_status tb_synchronize(void) { return tb::check_device_error(tb::g_stream); }

int tb_version(void) { return 100; }

unsigned long long tb_launch_count(void) { return tb::g_launches.load(); }

tb_status tb_profile_begin(void) {
  tb::g_prof_live.clear();
  tb::g_prof_on = true;
  return TB_SUCCESS;
}

tb_status tb_profile_end(double* gemm_ms, double* gemm_flops, long* gemm_launches) {
  tb::g_prof_on = false;
  double fl = 0;
  long cnt = 0;
  tb_status st = TB_SUCCESS;
  // launch intervals relative to the first launch's start event; launches on
  // different streams may overlap, so the device time is their union
  std::vector<std::pair<double, double>> iv;
  const cudaEvent_t ref = tb::g_prof_live.empty() ? nullptr : tb::g_prof_live.front().a;
  for (auto& r : tb::g_prof_live)
    if (cudaEventSynchronize(r.b) != cudaSuccess) st = TB_ERROR_CUDA;
  for (auto& r : tb::g_prof_live) {
    float t0 = 0, t1 = 0;
    if (cudaEventElapsedTime(&t0, ref, r.a) == cudaSuccess && cudaEventElapsedTime(&t1, ref, r.b) == cudaSuccess) {
      iv.push_back({t0, t1});
      fl += r.flops;
      ++cnt;
    }
  }
  for (auto& r : tb::g_prof_live) {
    tb::g_ev_free.push_back(r.a);
    tb::g_ev_free.push_back(r.b);
  }
  tb::g_prof_live.clear();
  std::sort(iv.begin(), iv.end());
  double ms = 0, cur0 = 0, cur1 = -1e300;
  for (const auto& x : iv) {
    if (x.first > cur1) {
      if (cur1 > cur0) ms += cur1 - cur0;
      cur0 = x.first;
      cur1 = x.second;
    } else if (x.second > cur1) {
      cur1 = x.second;
    }
  }
  if (cur1 > cur0) ms += cur1 - cur0;
  if (gemm_ms) *gemm_ms = ms;
  if (gemm_flops) *gemm_flops = fl;
  if (gemm_launches) *gemm_launches = cnt;
  return st;
}

}  // extern "C"
