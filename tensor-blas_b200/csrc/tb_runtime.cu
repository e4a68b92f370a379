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
  int* err = nullptr;        // the library's device error block (kErrBlockInts ints)
  int* extra_err = nullptr;  // a second block of this device (the allocation-free entry point's)
  int sms = 0;
  cudaStream_t aux[kAuxStreams] = {};
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
  double flops, bytes;
  int kind;  // ProfKind
};
// Per kind, for the last tb_profile_end: the union of the launches'
// intervals (ms), their flops and their number.
double g_prof_kind_ms[kProfKinds], g_prof_kind_flops[kProfKinds], g_prof_kind_bytes[kProfKinds];
long g_prof_kind_n[kProfKinds];
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

namespace {
std::atomic<unsigned long long> g_allocs{0};
}  // namespace

cudaError_t dev_malloc(void** p, size_t bytes) {
  g_allocs.fetch_add(1, std::memory_order_relaxed);
  return cudaMalloc(p, bytes);
}

bool profiling() { return g_prof_on; }

void* prof_begin(cudaStream_t st, ProfKind kind) {
  if (!g_prof_on) return nullptr;
  ProfRec r;
  r.a = ev_get();
  r.b = ev_get();
  r.flops = 0;
  r.bytes = 0;
  r.kind = (int)kind;
  cudaEventRecord(r.a, st);
  g_prof_live.push_back(r);
  return reinterpret_cast<void*>(g_prof_live.size());
}

void prof_end(void* token, cudaStream_t st, double flops, double bytes) {
  if (!token) return;
  ProfRec& r = g_prof_live[reinterpret_cast<size_t>(token) - 1];
  cudaEventRecord(r.b, st);
  r.flops = flops;
  r.bytes = bytes;
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

cudaStream_t aux_stream(int i) {
  DeviceState* s = state();
  if (!s || i < 0 || i >= kAuxStreams) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!s->aux[i] && cudaStreamCreateWithFlags(&s->aux[i], cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    s->aux[i] = nullptr;
  }
  return s->aux[i];
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
  if (dev_malloc(&s->pool[slot], want) != cudaSuccess) {
    cudaGetLastError();
    s->pool[slot] = nullptr;
    return nullptr;
  }
  s->pool_bytes[slot] = want;
  return s->pool[slot];
}

size_t pool_capacity(int slot) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState* s = state();
  return (s && slot >= 0 && slot < kPoolSlots) ? s->pool_bytes[slot] : 0;
}

size_t free_device_bytes() {
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return f;
}

void release_pool() {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState* s = state();
  if (!s) return;
  for (int i = 0; i < kPoolSlots; ++i) {
    if (s->pool[i]) cudaFree(s->pool[i]);
    s->pool[i] = nullptr;
    s->pool_bytes[i] = 0;
  }
}

int* device_error_word() {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState* s = state();
  if (!s) return nullptr;
  if (!s->err) {
    if (dev_malloc(reinterpret_cast<void**>(&s->err), kErrBlockInts * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      s->err = nullptr;
      return nullptr;
    }
    cudaMemset(s->err, 0, kErrBlockInts * sizeof(int));
  }
  return s->err;
}

void register_error_block(int* block) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState* s = state();
  if (s) s->extra_err = block;
}

// The error blocks of the current device that exist (none is created here).
static int error_blocks(int* out[2]) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState* s = state();
  int n = 0;
  if (s && s->err) out[n++] = s->err;
  if (s && s->extra_err) out[n++] = s->extra_err;
  return n;
}

tb_status check_device_error(cudaStream_t stream) {
  TB_CUDA_TRY(cudaStreamSynchronize(stream));
  int* blocks[2];
  const int nb = error_blocks(blocks);
  int code = 0;
  for (int i = 0; i < nb; ++i) {
    int h = 0;
    TB_CUDA_TRY(cudaMemcpy(&h, blocks[i], sizeof(int), cudaMemcpyDeviceToHost));
    if (h != 0) {
      TB_CUDA_TRY(cudaMemset(blocks[i], 0, sizeof(int)));
      if (!code) code = h;
    }
  }
  if (code) {
    set_last_error("device-side bounded wait timed out (code %d)", code);
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

unsigned long long tb_alloc_count(void) { return tb::g_allocs.load(); }

tb_status tb_release_scratch(void) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return tb::cuda_status(e);
  tb::release_pool();
  tb::release_tile_cache();
  tb::release_host_staging();
  return TB_SUCCESS;
}

tb_status tb_debug_stall(long tile, unsigned long long wait_ns) {
  if (tile < -1) return TB_ERROR_INVALID_VALUE;
  // words 1-3 of every error block of this device (word 0, the code, is kept)
  int* pool_block = tb::device_error_word();
  if (!pool_block) return TB_ERROR_ALLOC;
  int* blocks[2];
  const int nb = tb::error_blocks(blocks);
  int words[3] = {(int)(tile + 1), (int)(wait_ns & 0xffffffffull), (int)(wait_ns >> 32)};
  for (int i = 0; i < nb; ++i) TB_CUDA_TRY(cudaMemcpy(blocks[i] + 1, words, sizeof(words), cudaMemcpyHostToDevice));
  return TB_SUCCESS;
}

unsigned long long tb_launch_count(void) { return tb::g_launches.load(); }

tb_status tb_profile_begin(void) {
  tb::g_prof_live.clear();
  tb::g_prof_on = true;
  return TB_SUCCESS;
}

}  // extern "C"

namespace tb {
namespace {
// Total length of the union of intervals (launches on several streams may
// overlap; the device time is counted once).
double union_ms(std::vector<std::pair<double, double>> iv) {
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
  return ms;
}
}  // namespace
}  // namespace tb

extern "C" {
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
  for (int k = 0; k < tb::kProfKinds; ++k) {
    tb::g_prof_kind_ms[k] = tb::g_prof_kind_flops[k] = tb::g_prof_kind_bytes[k] = 0;
    tb::g_prof_kind_n[k] = 0;
  }
  std::vector<std::pair<double, double>> kind_iv[tb::kProfKinds];
  for (auto& r : tb::g_prof_live) {
    float t0 = 0, t1 = 0;
    if (cudaEventElapsedTime(&t0, ref, r.a) == cudaSuccess && cudaEventElapsedTime(&t1, ref, r.b) == cudaSuccess) {
      iv.push_back({t0, t1});
      kind_iv[r.kind].push_back({t0, t1});
      fl += r.flops;
      ++cnt;
      tb::g_prof_kind_flops[r.kind] += r.flops;
      tb::g_prof_kind_bytes[r.kind] += r.bytes;
      ++tb::g_prof_kind_n[r.kind];
    }
  }
  for (auto& r : tb::g_prof_live) {
    tb::g_ev_free.push_back(r.a);
    tb::g_ev_free.push_back(r.b);
  }
  tb::g_prof_live.clear();
  const double ms = tb::union_ms(iv);
  for (int k = 0; k < tb::kProfKinds; ++k) tb::g_prof_kind_ms[k] = tb::union_ms(kind_iv[k]);
  if (gemm_ms) *gemm_ms = ms;
  if (gemm_flops) *gemm_flops = fl;
  if (gemm_launches) *gemm_launches = cnt;
  return st;
}

tb_status tb_profile_kernel(int kind, double* ms, double* flops, double* bytes, long* launches) {
  if (kind < 0 || kind >= tb::kProfKinds) {
    tb::set_last_error("tb_profile_kernel: kind %d out of range", kind);
    return TB_ERROR_INVALID_VALUE;
  }
  if (ms) *ms = tb::g_prof_kind_ms[kind];
  if (flops) *flops = tb::g_prof_kind_flops[kind];
  if (bytes) *bytes = tb::g_prof_kind_bytes[kind];
  if (launches) *launches = tb::g_prof_kind_n[kind];
  return TB_SUCCESS;
}

}  // extern "C"
