// Library runtime: status strings, per-thread error text, the current stream,
// the per-device scratch pool and the device error word used by the bounded
// waits of the persistent kernels.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "tb_internal.h"

namespace tb {

namespace {
thread_local char g_last_error[512] = "";
cudaStream_t g_stream = nullptr;

constexpr int kMaxDevices = 64;
struct DeviceState {
  void* pool = nullptr;
  size_t pool_bytes = 0;
  int* err = nullptr;
  int sms = 0;
};
DeviceState g_dev[kMaxDevices];
std::mutex g_mu;

DeviceState* state() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) return nullptr;
  return &g_dev[d];
}
}  // namespace

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

void* pool_get(size_t bytes) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState* s = state();
  if (!s) return nullptr;
  if (bytes == 0) bytes = 256;
  if (s->pool_bytes >= bytes) return s->pool;
  if (s->pool) {
    cudaDeviceSynchronize();  // work queued on the old buffer must finish
    cudaFree(s->pool);
    s->pool = nullptr;
    s->pool_bytes = 0;
  }
  size_t want = (size_t)round_up((long long)bytes, 1 << 20);
  if (cudaMalloc(&s->pool, want) != cudaSuccess) {
    cudaGetLastError();
    s->pool = nullptr;
    return nullptr;
  }
  s->pool_bytes = want;
  return s->pool;
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

}  // extern "C"
