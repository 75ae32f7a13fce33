// Runtime plumbing of the nec2c CUDA backend: per-thread error text, the
// stream work is enqueued on, device buffers and a launch counter.
#include <stdlib.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <atomic>
#include <thread>
#include "common.cuh"
#include "device_api.h"
#include "runtime.cuh"

static thread_local char g_error[512];
static thread_local cudaStream_t g_stream = nullptr;
static thread_local const int *g_gate = nullptr;
static std::atomic<unsigned long long> g_launches{0};

extern "C" void n2c_set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}
extern "C" const char *n2d_last_error(void) { return g_error; }
extern "C" void n2d_set_stream(void *s) { g_stream = (cudaStream_t)s; }
extern "C" void *n2d_get_stream(void) { return (void *)g_stream; }
cudaStream_t n2c_stream() { return g_stream; }
extern "C" void n2d_set_gate(const int *gate_dev) { g_gate = gate_dev; }
const int *n2c_gate() { return g_gate; }
void n2c_count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
extern "C" unsigned long long n2d_launch_count(void) { return g_launches.load(); }

bool n2c_pdl_enabled() {
  static const bool on = [] {
    const char *v = getenv("NEC2C_CUDA_PDL");
    return !(v && v[0] == '0');
  }();
  return on;
}

int n2c_check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    n2c_set_error("%s launch failed: %s", what, cudaGetErrorString(e));
    return 0;
  }
  n2c_count_launch(1);
  return 1;
}

extern "C" int n2d_sync(void) {
  cudaError_t e = cudaStreamSynchronize(g_stream);
  if (e != cudaSuccess) { n2c_set_error("stream synchronize: %s", cudaGetErrorString(e)); return 0; }
  return 1;
}
extern "C" void *n2d_alloc(size_t bytes) {
  void *p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) { n2c_set_error("cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e)); return nullptr; }
  return p;
}
extern "C" void n2d_free(void *p) { if (p) cudaFree(p); }
// Stream-ordered allocation on this thread's stream from the device's default
// pool, which keeps freed memory for reuse (no device-wide synchronisation,
// unlike cudaFree): for per-call scratch of work that runs concurrently on
// several streams.
extern "C" void *n2d_alloc_async(size_t bytes) {
  static thread_local int pool_dev = -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  if (pool_dev != dev) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      unsigned long long keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    pool_dev = dev;
  }
  void *p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMallocAsync(&p, bytes, g_stream);
  if (e != cudaSuccess) { n2c_set_error("cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e)); return nullptr; }
  return p;
}
extern "C" void n2d_free_async(void *p) { if (p) cudaFreeAsync(p, g_stream); }
// This thread's own non-blocking stream (created once per thread and device)
// for hosts that run several solves concurrently.
extern "C" void *n2d_stream_create(void) {
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    n2c_set_error("stream creation failed");
    return nullptr;
  }
  return (void *)s;
}
extern "C" void n2d_stream_destroy(void *s) { if (s) cudaStreamDestroy((cudaStream_t)s); }
extern "C" int n2d_mem_info(size_t *free_bytes, size_t *total_bytes) {
  N2C_CHECK(cudaMemGetInfo(free_bytes, total_bytes));
  return 1;
}
// ------------------------------------------------------------- host copies
// Pageable host memory above STAGE_MIN bytes moves through two pinned staging
// buffers so that the host memcpy of one chunk overlaps the DMA of the other.
// Pinned (page-locked or registered) host memory is copied directly.
static const size_t STAGE_CHUNK = 8u << 20, STAGE_MIN = 1u << 20;

// Host rows copied by several threads (a single thread moves pageable memory
// at a fraction of the host's bandwidth): half the host cores, at most 8,
// shared among the copies in progress on all threads (several streams'
// workers copy at once), rows split evenly; small copies stay on the calling
// thread.
static std::atomic<int> g_copies{0};
static void copy_rows(char *dst, size_t dp, const char *src, size_t sp, size_t width, size_t rows) {
  const size_t bytes = width * rows;
  const int active = g_copies.fetch_add(1) + 1;
  unsigned hw = std::thread::hardware_concurrency() / 2 / (unsigned)active;
  unsigned nt = hw < 1 ? 1 : (hw > 8 ? 8 : hw);
  if (bytes < (4u << 20) || rows < 2 * nt) nt = 1;
  auto part = [=](unsigned i) {
    const size_t r0 = rows * i / nt, r1 = rows * (i + 1) / nt;
    if (dp == width && sp == width) memcpy(dst + r0 * width, src + r0 * width, (r1 - r0) * width);
    else for (size_t r = r0; r < r1; ++r) memcpy(dst + r * dp, src + r * sp, width);
  };
  if (nt == 1) {
    part(0);
  } else {
    std::thread th[8];
    for (unsigned i = 1; i < nt; ++i) th[i] = std::thread(part, i);
    part(0);
    for (unsigned i = 1; i < nt; ++i) th[i].join();
  }
  g_copies.fetch_sub(1);
}
struct Stage {
  void *buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool ok = false;
  // Released when the owning thread exits (worker threads of a server);
  // errors after the process has torn CUDA down are ignored.
  ~Stage() {
    for (int i = 0; i < 2; ++i) {
      if (ev[i]) cudaEventDestroy(ev[i]);
      if (buf[i]) cudaFreeHost(buf[i]);
    }
    cudaGetLastError();
  }
};
static thread_local Stage g_stage;

static bool stage_ready() {
  Stage &s = g_stage;
  if (s.ok) return true;
  for (int i = 0; i < 2; ++i) {
    if (cudaHostAlloc(&s.buf[i], STAGE_CHUNK, cudaHostAllocDefault) != cudaSuccess) { cudaGetLastError(); return false; }
    if (cudaEventCreateWithFlags(&s.ev[i], cudaEventDisableTiming) != cudaSuccess) { cudaGetLastError(); return false; }
  }
  s.ok = true;
  return true;
}

static bool is_pinned(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) { cudaGetLastError(); return false; }
  return at.type == cudaMemoryTypeHost;
}

// Rows of `width` bytes: host rows at pitch hp, device rows at pitch dp.
static int staged_h2d(void *dst, size_t dp, const void *src, size_t hp, size_t width, size_t rows) {
  Stage &s = g_stage;
  const size_t per = STAGE_CHUNK / width;         // rows per chunk (>= 1: width <= chunk)
  int k = 0;
  for (size_t r0 = 0; r0 < rows; r0 += per, k ^= 1) {
    const size_t nr = rows - r0 < per ? rows - r0 : per;
    N2C_CHECK(cudaEventSynchronize(s.ev[k]));
    char *b = (char *)s.buf[k];
    copy_rows(b, width, (const char *)src + r0 * hp, hp, width, nr);
    N2C_CHECK(cudaMemcpy2DAsync((char *)dst + r0 * dp, dp, b, width, width, nr, cudaMemcpyHostToDevice, g_stream));
    N2C_CHECK(cudaEventRecord(s.ev[k], g_stream));
  }
  return 1;
}

static int staged_d2h(void *dst, size_t hp, const void *src, size_t dp, size_t width, size_t rows) {
  Stage &s = g_stage;
  const size_t per = STAGE_CHUNK / width;
  const size_t chunks = (rows + per - 1) / per;
  auto issue = [&](size_t c) -> int {
    const size_t r0 = c * per, nr = rows - r0 < per ? rows - r0 : per;
    N2C_CHECK(cudaMemcpy2DAsync(s.buf[c & 1], width, (const char *)src + r0 * dp, dp, width, nr,
                                cudaMemcpyDeviceToHost, g_stream));
    N2C_CHECK(cudaEventRecord(s.ev[c & 1], g_stream));
    return 1;
  };
  if (!issue(0)) return 0;
  for (size_t c = 0; c < chunks; ++c) {
    if (c + 1 < chunks && !issue(c + 1)) return 0;
    N2C_CHECK(cudaEventSynchronize(s.ev[c & 1]));
    const size_t r0 = c * per, nr = rows - r0 < per ? rows - r0 : per;
    copy_rows((char *)dst + r0 * hp, hp, (const char *)s.buf[c & 1], width, width, nr);
  }
  return 1;
}

extern "C" int n2d_upload(void *dst, const void *src, size_t bytes) {
  if (!bytes) return 1;
  if (bytes >= STAGE_MIN && !is_pinned(src) && stage_ready()) {
    const size_t w = 64 * 1024, rows = bytes / w, tail = bytes - rows * w;
    if (rows && !staged_h2d(dst, w, src, w, w, rows)) return 0;
    if (tail) N2C_CHECK(cudaMemcpyAsync((char *)dst + rows * w, (const char *)src + rows * w, tail,
                                        cudaMemcpyHostToDevice, g_stream));
    N2C_CHECK(cudaStreamSynchronize(g_stream));   // the caller may reuse src
    return 1;
  }
  N2C_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, g_stream));
  return 1;
}
extern "C" int n2d_download(void *dst, const void *src, size_t bytes) {
  if (!bytes) return 1;
  if (bytes >= STAGE_MIN && !is_pinned(dst) && stage_ready()) {
    const size_t w = 64 * 1024, rows = bytes / w, tail = bytes - rows * w;
    if (rows && !staged_d2h(dst, w, src, w, w, rows)) return 0;
    if (tail) N2C_CHECK(cudaMemcpyAsync((char *)dst + rows * w, (const char *)src + rows * w, tail,
                                        cudaMemcpyDeviceToHost, g_stream));
    N2C_CHECK(cudaStreamSynchronize(g_stream));
    return 1;
  }
  N2C_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, g_stream));
  N2C_CHECK(cudaStreamSynchronize(g_stream));
  return 1;
}
extern "C" int n2d_memset(void *dst, int v, size_t bytes) {
  if (!bytes) return 1;
  N2C_CHECK(cudaMemsetAsync(dst, v, bytes, g_stream));
  return 1;
}
extern "C" int n2d_copy_d2d(void *dst, const void *src, size_t bytes) {
  if (!bytes) return 1;
  N2C_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, g_stream));
  return 1;
}

extern "C" int n2d_upload2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                            size_t rows) {
  if (!width || !rows) return 1;
  if (width * rows >= STAGE_MIN && width <= STAGE_CHUNK && !is_pinned(src) && stage_ready()) {
    if (!staged_h2d(dst, dpitch, src, spitch, width, rows)) return 0;
    N2C_CHECK(cudaStreamSynchronize(g_stream));
    return 1;
  }
  N2C_CHECK(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyHostToDevice, g_stream));
  return 1;
}
extern "C" int n2d_download2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                              size_t rows) {
  if (!width || !rows) return 1;
  if (width * rows >= STAGE_MIN && width <= STAGE_CHUNK && !is_pinned(dst) && stage_ready()) {
    if (!staged_d2h(dst, dpitch, src, spitch, width, rows)) return 0;
    N2C_CHECK(cudaStreamSynchronize(g_stream));
    return 1;
  }
  N2C_CHECK(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDeviceToHost, g_stream));
  N2C_CHECK(cudaStreamSynchronize(g_stream));
  return 1;
}
extern "C" int n2d_set_device(int device) {
  N2C_CHECK(cudaSetDevice(device));
  return 1;
}

extern "C" int n2d_device_ok(void) {
  int count = 0, dev = 0, major = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
    cudaGetLastError();
    n2c_set_error("no CUDA device available");
    return 0;
  }
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) { n2c_set_error("device compute capability %d.x is not sm_100", major); return 0; }
  return 1;
}

int n2c_sm_count() {
  static const int sms = [] {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
  }();
  return sms;
}
