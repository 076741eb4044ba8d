// api.cu - status reporting, device info and small C ABI helpers.
#include <stdarg.h>
#include <mutex>
#include <vector>
#include "common.cuh"

namespace mb {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

mb_status fail(mb_status st, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return st;
}

mb_status cuda_fail(cudaError_t e, const char *what) {
  set_error("%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? MB_ERR_OOM : MB_ERR_CUDA;
}

const DevInfo &dev_info() {
  static std::mutex mu;
  static std::vector<DevInfo> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if ((int)cache.size() <= dev) cache.resize(dev + 1);
  DevInfo &d = cache[dev];
  if (d.device != dev) {
    d.device = dev;
    cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&d.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&d.max_threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    if (d.sms <= 0) d.sms = 148;
  }
  return d;
}

cudaMemPool_t scratch_pool() {
  static std::mutex mu;
  static std::vector<cudaMemPool_t> pools;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

uint32_t *device_error_word() {
  static std::mutex mu;
  static std::vector<uint32_t *> words;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if ((int)words.size() <= dev) words.resize(dev + 1, nullptr);
  if (!words[dev]) {
    uint32_t *p = nullptr;
    if (cudaMalloc(&p, 4 * sizeof(uint32_t)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, 4 * sizeof(uint32_t));
    words[dev] = p;
  }
  return words[dev];
}

mb_status check_device_error(cudaStream_t s) {
  uint32_t *w = device_error_word();
  if (!w) return fail(MB_ERR_OOM, "device error word allocation failed");
  uint32_t h[4] = {0, 0, 0, 0};
  MB_CUDA(cudaMemcpyAsync(h, w, sizeof(h), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  if (h[0] != 0) {
    cudaMemsetAsync(w, 0, 4 * sizeof(uint32_t), s);
    cudaStreamSynchronize(s);
    return fail(MB_ERR_TIMEOUT, "a bounded device wait ran out (code %u, block %u)", h[1], h[2]);
  }
  return MB_OK;
}

}  // namespace mb

extern "C" {

const char *mb_last_error(void) { return mb::g_err; }

const char *mb_version(void) { return "merle_b200 0.1 (sm_100a)"; }

uint64_t mb_bitmap_words(uint64_t nrows) { return (nrows + 31) / 32; }

uint64_t mb_bitmap_stride(uint64_t nrows) { return mb::round_up((nrows + 31) / 32, 32); }

int mb_vprg_is_nochk(const mb_vprg *p) {
  if (!p) return 1;
  for (uint32_t i = 0; i < p->ncols && i < MB_MAXCOLS; ++i)
    if (p->cols[i].leftmost || p->cols[i].rightmost) return 0;
  return 1;
}

}  // extern "C"
