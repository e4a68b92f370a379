// Autotuner: picks nb and the GEMM engine per (routine, flags, sizes,
// precision) when a caller passes nb = TB_NB_AUTO.
//
// Candidates are timed once, on scratch outputs of the caller's shapes
// (zero-filled: values do not change the tensor-core timing), with CUDA
// events on the caller's stream; the fastest is kept in an in-memory cache
// per device and, when a cache file is set (TB_AUTOTUNE_CACHE in the
// environment or tb_autotune_set_file), in a JSON file that is rewritten
// through a temporary file and a rename, so a reader never sees half of it.
// Keys start with the device name, compute capability and driver version,
// so one file can serve several machines.
//
// Knobs: the GEMM engine, i.e. the tile shape and cluster size of the large
// plain launches (1: 256 x 256 tiles on CTA pairs, 0: single-CTA 128 x 256
// tiles, 2: single-CTA 128 x 128 tiles, twice as many tiles as 0 for
// problems whose wider tiles leave SMs idle; split launches use 128-wide
// tiles either way, so 2 is a candidate for plain precision only); for TRSM
// the leaf size nb (128,
// 256, 512), which sets the recursion's leaf inverses and the number of
// update launches (SYRK, SYR2K and TRMM do not use nb); and for plain 'N'
// SYRKs whose triangle has fewer 128 x 256 tiles than the GPU has SMs (small
// n, long k) the split-K count (2 to 16 parts of K in one grouped launch plus
// a reduction), which fills the SMs the one-pass launch leaves idle.
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "tb_internal.h"

namespace tb {
namespace {

std::mutex g_mu;
std::map<std::string, TuneChoice> g_cache;
std::string g_file;
bool g_file_init = false;

// The key prefix of the current device, built once per device: the device
// properties query takes milliseconds of host time, and every NB_AUTO call
// builds a key.
std::string device_tag() {
  static std::mutex mu;
  static std::map<int, std::string> tags;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return "nodevice";
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = tags.find(dev);
    if (it != tags.end()) return it->second;
  }
  int drv = 0;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
    cudaGetLastError();
    return "nodevice";
  }
  cudaDriverGetVersion(&drv);
  char buf[384];
  snprintf(buf, sizeof(buf), "%s/sm_%d%d/drv%d", p.name, p.major, p.minor, drv);
  for (char* c = buf; *c; ++c)
    if (*c == '"' || *c == '\\' || *c == '|') *c = '_';
  std::lock_guard<std::mutex> lk(mu);
  tags[dev] = buf;
  return buf;
}

// caller holds g_mu
void load_locked() {
  if (g_file.empty()) return;
  FILE* f = fopen(g_file.c_str(), "r");
  if (!f) return;
  char line[1024];
  while (fgets(line, sizeof(line), f)) {
    char key[512];
    TuneChoice c{};
    if (sscanf(line, " {\"key\": \"%511[^\"]\", \"nb\": %ld, \"engine\": %d, \"splitk\": %d, \"ms\": %lf}", key,
               &c.nb, &c.engine, &c.splitk, &c.ms) == 5 ||
        sscanf(line, " {\"key\": \"%511[^\"]\", \"nb\": %ld, \"engine\": %d, \"ms\": %lf}", key, &c.nb, &c.engine,
               &c.ms) == 4) {
      if (c.splitk < 1) c.splitk = 1;
      g_cache[key] = c;
    }
  }
  fclose(f);
}

// caller holds g_mu
tb_status save_locked() {
  if (g_file.empty()) return TB_SUCCESS;
  const std::string tmp = g_file + ".tmp." + std::to_string((long)getpid());
  FILE* f = fopen(tmp.c_str(), "w");
  if (!f) {
    set_last_error("autotune: cannot write %s", tmp.c_str());
    return TB_ERROR_INVALID_VALUE;
  }
  fprintf(f, "{\n \"format\": \"tensorblas-autotune-1\",\n \"entries\": [\n");
  size_t i = 0;
  for (const auto& kv : g_cache)
    fprintf(f, "  {\"key\": \"%s\", \"nb\": %ld, \"engine\": %d, \"splitk\": %d, \"ms\": %.6f}%s\n",
            kv.first.c_str(), kv.second.nb, kv.second.engine, kv.second.splitk, kv.second.ms,
            ++i < g_cache.size() ? "," : "");
  fprintf(f, " ]\n}\n");
  const bool ok = fflush(f) == 0 && fsync(fileno(f)) == 0;
  fclose(f);
  if (!ok || rename(tmp.c_str(), g_file.c_str()) != 0) {
    remove(tmp.c_str());
    set_last_error("autotune: cannot replace %s", g_file.c_str());
    return TB_ERROR_INVALID_VALUE;
  }
  return TB_SUCCESS;
}

// caller holds g_mu
void init_file_locked() {
  if (g_file_init) return;
  g_file_init = true;
  const char* e = getenv("TB_AUTOTUNE_CACHE");
  if (e && *e) {
    g_file = e;
    load_locked();
  }
}

}  // namespace

std::string tune_key(const char* routine, const char* flags, long a, long b, int precision) {
  return device_tag() + "|" + routine + "|" + flags + "|" + std::to_string(a) + "|" + std::to_string(b) + "|" +
         std::to_string(precision);
}

tb_status autotune(const std::string& key, const std::vector<TuneChoice>& candidates,
                   const std::function<tb_status(const TuneChoice&)>& trial, cudaStream_t st, TuneChoice* out) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    init_file_locked();
    auto it = g_cache.find(key);
    if (it != g_cache.end()) {
      *out = it->second;
      return TB_SUCCESS;
    }
  }
  cudaEvent_t e0, e1;
  TB_CUDA_TRY(cudaEventCreate(&e0));
  TB_CUDA_TRY(cudaEventCreate(&e1));
  TuneChoice best{0, 0, -1.0};
  tb_status status = TB_SUCCESS;
  for (const TuneChoice& c : candidates) {
    EngineScope scope(c.engine);
    SplitKScope sk(c.splitk);
    status = trial(c);  // warm-up: plans, scratch growth, tile uploads
    if (status != TB_SUCCESS) break;
    double ms = 1e30;
    for (int r = 0; r < 2 && status == TB_SUCCESS; ++r) {
      cudaEventRecord(e0, st);
      status = trial(c);
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) status = TB_ERROR_CUDA;
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      ms = t < ms ? t : ms;
    }
    if (status != TB_SUCCESS) break;
    if (best.ms < 0 || ms < best.ms) {
      best = c;
      best.ms = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status != TB_SUCCESS) return status;
  TB_TRY(check_device_error(st));
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache[key] = best;
  *out = best;
  return save_locked();
}

}  // namespace tb

using namespace tb;

extern "C" tb_status tb_autotune_set_file(const char* path) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_file_init = true;
  g_file = path ? path : "";
  load_locked();
  return TB_SUCCESS;
}

extern "C" tb_status tb_autotune_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache.clear();
  return TB_SUCCESS;
}

extern "C" int tb_autotune_entries(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  return (int)g_cache.size();
}

extern "C" tb_status tb_autotune_put(const char* routine, const char* flags, long a, long b, int precision, long nb,
                                     int engine, double ms) {
  if (!routine || !flags || nb <= 0 || engine < 0 || engine > kEngineNarrow) return TB_ERROR_INVALID_VALUE;
  const std::string key = tune_key(routine, flags, a, b, precision);
  std::lock_guard<std::mutex> lk(g_mu);
  init_file_locked();
  g_cache[key] = TuneChoice{nb, engine, ms};
  return save_locked();
}

extern "C" tb_status tb_autotune_put_ex(const char* routine, const char* flags, long a, long b, int precision, long nb,
                                        int engine, int splitk, double ms) {
  if (!routine || !flags || nb <= 0 || engine < 0 || engine > kEngineNarrow || splitk < 1 || splitk > 64)
    return TB_ERROR_INVALID_VALUE;
  const std::string key = tune_key(routine, flags, a, b, precision);
  std::lock_guard<std::mutex> lk(g_mu);
  init_file_locked();
  TuneChoice c{nb, engine, ms};
  c.splitk = splitk;
  g_cache[key] = c;
  return save_locked();
}

extern "C" tb_status tb_autotune_get_ex(const char* routine, const char* flags, long a, long b, int precision,
                                        long* nb, int* engine, int* splitk) {
  if (!splitk) return TB_ERROR_INVALID_VALUE;
  const tb_status s = tb_autotune_get(routine, flags, a, b, precision, nb, engine);
  if (s != TB_SUCCESS) return s;
  const std::string key = tune_key(routine, flags, a, b, precision);
  std::lock_guard<std::mutex> lk(g_mu);
  *splitk = g_cache[key].splitk;
  return TB_SUCCESS;
}

extern "C" tb_status tb_autotune_get(const char* routine, const char* flags, long a, long b, int precision, long* nb,
                                     int* engine) {
  if (!routine || !flags || !nb || !engine) return TB_ERROR_INVALID_VALUE;
  const std::string key = tune_key(routine, flags, a, b, precision);
  std::lock_guard<std::mutex> lk(g_mu);
  init_file_locked();
  auto it = g_cache.find(key);
  if (it == g_cache.end()) return TB_ERROR_NOT_SUPPORTED;
  *nb = it->second.nb;
  *engine = it->second.engine;
  return TB_SUCCESS;
}

// ---------------------------------------------------------------- nb = TB_NB_AUTO
namespace tb {
namespace {

// Zero-filled device scratch for the trials' outputs, allocated on first use.
struct TuneScratch {
  size_t bytes;
  float* p = nullptr;
  explicit TuneScratch(size_t b) : bytes(b) {}
  ~TuneScratch() {
    if (p) cudaFree(p);
  }
  tb_status get(cudaStream_t st, float** out) {
    if (!p) {
      if (dev_malloc(reinterpret_cast<void**>(&p), bytes) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        set_last_error("autotune: cannot allocate %zu bytes of trial output", bytes);
        return TB_ERROR_ALLOC;
      }
      TB_CUDA_TRY(cudaMemsetAsync(p, 0, bytes, st));
    }
    *out = p;
    return TB_SUCCESS;
  }
};

// Engine candidates of a routine without nb: the pair and single-CTA
// engines, and for plain precision the narrow single-CTA tiles.
std::vector<TuneChoice> engines(int precision) {
  std::vector<TuneChoice> c = {{256, 1, 0}, {256, 0, 0}};
  if (precision == TB_PREC_PLAIN) c.push_back(TuneChoice{256, kEngineNarrow, 0});
  return c;
}

}  // namespace

tb_status auto_ssyrk(char uplo, char trans, long n, long k, float alpha, const float* A, long lda, float beta,
                     float* C, long ldc, int precision) {
  if (n <= 0 || k <= 0 || ldc < n || precision == TB_PREC_FP8)
    return tb_ssyrk(uplo, trans, n, k, alpha, A, lda, beta, C, ldc, 256, precision);
  const cudaStream_t st = current_stream();
  TuneScratch s((size_t)ldc * n * sizeof(float));
  const char flags[3] = {uplo, trans, 0};
  std::vector<TuneChoice> cands = engines(precision);
  const bool tr = trans == 'T' || trans == 't' || trans == 'C' || trans == 'c';
  const long kb = (k + kGemmBK - 1) / kGemmBK;
  if (precision == TB_PREC_PLAIN && !tr && n <= kSplitKMaxN && kb > kGemmPfMaxKb) {
    // split-K candidates while the one-pass triangle leaves SMs idle
    const bool up = uplo == 'U' || uplo == 'u';
    const long tiles = (long)(up ? plan_upper((int)n, 256, 0, 1) : plan_lower((int)n, 256, 0, 1)).size();
    for (int sk : {2, 4, 8, 16})
      if (tiles < sm_count() && tiles * sk <= 4L * sm_count() && sk <= kb / 4) {
        TuneChoice c{256, 0, 0};
        c.splitk = sk;
        cands.push_back(c);
      }
  }
  TuneChoice ch;
  TB_TRY(autotune(tune_key("ssyrk", flags, n, k, precision), cands,
                  [&](const TuneChoice& c) {
                    float* Cs = nullptr;
                    TB_TRY(s.get(st, &Cs));
                    return tb_ssyrk(uplo, trans, n, k, alpha, A, lda, beta, Cs, ldc, c.nb, precision);
                  },
                  st, &ch));
  EngineScope scope(ch.engine);
  SplitKScope sk(ch.splitk);
  return tb_ssyrk(uplo, trans, n, k, alpha, A, lda, beta, C, ldc, ch.nb, precision);
}

tb_status auto_strsm(char side, long m, long n, const float* A, long lda, float* B, long ldb, int precision) {
  if (m <= 0 || n <= 0 || ldb < m) return tb_strsm(side, m, n, A, lda, B, ldb, 512, precision);
  const cudaStream_t st = current_stream();
  TuneScratch s((size_t)ldb * n * sizeof(float));
  const char flags[2] = {side, 0};
  std::vector<TuneChoice> cands;
  for (long nb : {512L, 256L, 128L})
    for (int e : {1, 0, kEngineNarrow})
      if (e != kEngineNarrow || precision == TB_PREC_PLAIN) cands.push_back(TuneChoice{nb, e, 0});
  TuneChoice ch;
  TB_TRY(autotune(tune_key("strsm", flags, m, n, precision), cands,
                  [&](const TuneChoice& c) {
                    float* Bs = nullptr;
                    TB_TRY(s.get(st, &Bs));
                    return tb_strsm(side, m, n, A, lda, Bs, ldb, c.nb, precision);
                  },
                  st, &ch));
  EngineScope scope(ch.engine);
  return tb_strsm(side, m, n, A, lda, B, ldb, ch.nb, precision);
}

tb_status auto_ssyr2k(char uplo, char trans, long n, long k, float alpha, const float* A, long lda, const float* B,
                      long ldb, float beta, float* C, long ldc, int precision) {
  if (n <= 0 || k <= 0 || ldc < n || precision == TB_PREC_FP8)
    return tb_ssyr2k(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 256, precision);
  const cudaStream_t st = current_stream();
  TuneScratch s((size_t)ldc * n * sizeof(float));
  const char flags[3] = {uplo, trans, 0};
  TuneChoice ch;
  TB_TRY(autotune(tune_key("ssyr2k", flags, n, k, precision), engines(precision),
                  [&](const TuneChoice& c) {
                    float* Cs = nullptr;
                    TB_TRY(s.get(st, &Cs));
                    return tb_ssyr2k(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, Cs, ldc, c.nb, precision);
                  },
                  st, &ch));
  EngineScope scope(ch.engine);
  return tb_ssyr2k(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C, ldc, ch.nb, precision);
}

tb_status auto_strmm(char uplo, long m, long n, float alpha, const float* A, long lda, const float* B, long ldb,
                     float* C, long ldc, int precision) {
  if (m <= 0 || n <= 0 || ldc < m || precision == TB_PREC_FP8)
    return tb_strmm(uplo, m, n, alpha, A, lda, B, ldb, C, ldc, 256, precision);
  const cudaStream_t st = current_stream();
  TuneScratch s((size_t)ldc * n * sizeof(float));
  const char flags[2] = {uplo, 0};
  TuneChoice ch;
  TB_TRY(autotune(tune_key("strmm", flags, m, n, precision), engines(precision),
                  [&](const TuneChoice& c) {
                    float* Cs = nullptr;
                    TB_TRY(s.get(st, &Cs));
                    return tb_strmm(uplo, m, n, alpha, A, lda, B, ldb, Cs, ldc, c.nb, precision);
                  },
                  st, &ch));
  EngineScope scope(ch.engine);
  return tb_strmm(uplo, m, n, alpha, A, lda, B, ldb, C, ldc, ch.nb, precision);
}

}  // namespace tb
