// Status codes, device queries and per-stream reduction scratch.
#include <algorithm>
#include <climits>
#include <cstdio>

#include "sb2_internal.cuh"

namespace sb2 {

std::atomic<long long> g_wait_limit_us{2000000};

int map_cuda_error(cudaError_t e) {
  if (e == cudaSuccess) return SB2_OK;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the sticky-free allocation error
    return SB2_ERR_NO_MEMORY;
  }
  return SB2_ERR_CUDA;
}

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

int num_sms(int device) {
  static std::mutex mu;
  static std::map<int, int> cache;
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(device);
  if (it != cache.end()) return it->second;
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0)
    v = 148;
  cache[device] = v;
  return v;
}

// Solver workspaces are allocated per call in stream order.  They come from
// a pool owned by the library that keeps up to kPoolKeepBytes of freed memory
// mapped for the next call; the device's default pool would unmap freed
// blocks at each synchronization, and the next solve would pay for mapping
// them again (milliseconds for a few hundred MB).
static constexpr unsigned long long kPoolKeepBytes = 8ull << 30;

cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t s) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  const int dev = current_device();
  cudaMemPool_t pool;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = pools.find(dev);
    if (it == pools.end()) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      cudaError_t e = cudaMemPoolCreate(&pool, &props);
      if (e != cudaSuccess) return e;
      unsigned long long keep = kPoolKeepBytes;
      e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) {
        cudaMemPoolDestroy(pool);
        return e;
      }
      pools[dev] = pool;
    } else {
      pool = it->second;
    }
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

// Arrays handed to the caller from the pool (sb2_coo_to_csr's outputs):
// sb2_device_free gives them back to the pool instead of the driver, which
// saves the unmapping (and the next call's mapping) of large buffers.
static std::mutex g_owned_mu;
static std::map<void*, int> g_owned;  // pointer -> device

cudaError_t pool_malloc_owned(void** p, size_t bytes, cudaStream_t s) {
  cudaError_t e = pool_malloc(p, bytes, s);
  if (e == cudaSuccess) {
    std::lock_guard<std::mutex> g(g_owned_mu);
    g_owned[*p] = current_device();
  }
  return e;
}

bool release_owned(void* p, cudaError_t* err) {
  int dev;
  {
    std::lock_guard<std::mutex> g(g_owned_mu);
    auto it = g_owned.find(p);
    if (it == g_owned.end()) return false;
    dev = it->second;
    g_owned.erase(it);
  }
  // cudaFree's guarantee: no work on the device still uses p
  int prev = current_device();
  cudaSetDevice(dev);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaFreeAsync(p, 0);
  cudaSetDevice(prev);
  *err = e;
  return true;
}

int get_red_scratch(cudaStream_t s, RedScratch** out) {
  static std::mutex mu;
  static std::map<std::pair<int, cudaStream_t>, RedScratch*> table;
  const int dev = current_device();
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(dev, s);
  auto it = table.find(key);
  if (it != table.end()) {
    *out = it->second;
    return SB2_OK;
  }
  RedScratch* r = new RedScratch();
  cudaError_t e = cudaMalloc(&r->partials, sizeof(double) * kRedMaxBlocks * 4);
  if (e == cudaSuccess) e = cudaMalloc(&r->counter, sizeof(unsigned) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&r->result, sizeof(double) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&r->status, sizeof(int) * 4);
  if (e == cudaSuccess) e = cudaMemset(r->status, 0, sizeof(int) * 4);
  if (e == cudaSuccess) e = cudaMemset(r->counter, 0, sizeof(unsigned) * 4);
  if (e != cudaSuccess) {
    cudaFree(r->partials);
    cudaFree(r->counter);
    cudaFree(r->result);
    cudaFree(r->status);
    delete r;
    return map_cuda_error(e);
  }
  table[key] = r;
  *out = r;
  return SB2_OK;
}

}  // namespace sb2

extern "C" {

const char* sb2_status_string(int status) {
  switch (status) {
    case SB2_OK: return "ok";
    case SB2_ERR_INVALID_VALUE: return "invalid value (sizes, null or overlapping pointers)";
    case SB2_ERR_NO_MEMORY: return "device or host allocation failed";
    case SB2_ERR_CUDA: return "CUDA runtime error";
    case SB2_ERR_TIMEOUT: return "a bounded device-side wait ran out";
    case SB2_ERR_INVALID_CSR: return "CSR invariants violated";
    case SB2_ERR_NOT_SUPPORTED: return "option combination not supported";
    case SB2_ERR_HOST: return "host-side failure";
    default: return "unknown status";
  }
}

int sb2_version(void) { return 10000; }

int sb2_device_alloc(size_t bytes, void** out) try {
  if (!out) return SB2_ERR_INVALID_VALUE;
  *out = nullptr;
  if (bytes == 0) return SB2_OK;
  return sb2::map_cuda_error(cudaMalloc(out, bytes));
} SB2_CATCH

int sb2_device_free(void* p) try {
  if (!p) return SB2_OK;
  cudaError_t e;
  if (sb2::release_owned(p, &e)) return sb2::map_cuda_error(e);
  return sb2::map_cuda_error(cudaFree(p));
} SB2_CATCH

int sb2_memcpy(void* dst, const void* src, size_t bytes, void* stream) try {
  if (bytes == 0) return SB2_OK;
  if (!dst || !src) return SB2_ERR_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return sb2::map_cuda_error(e);
} SB2_CATCH

int sb2_stream_sync(void* stream) try {
  return sb2::map_cuda_error(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
} SB2_CATCH

int sb2_set_wait_limit_ms(int ms) try {
  const long long old_us = sb2::g_wait_limit_us;
  if (ms > 0) sb2::g_wait_limit_us = (long long)ms * 1000;
  return (int)std::min<long long>((old_us + 999) / 1000, INT_MAX);
} SB2_CATCH

int sb2_spmv_status(void* stream, int* status) try {
  if (!status) return SB2_ERR_INVALID_VALUE;
  sb2::RedScratch* rs = nullptr;
  const int st = sb2::get_red_scratch(static_cast<cudaStream_t>(stream), &rs);
  if (st != SB2_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  SB2_CUDA_TRY(cudaMemcpyAsync(status, rs->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaMemsetAsync(rs->status, 0, sizeof(int), s));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  return SB2_OK;
} SB2_CATCH

int sb2_set_wait_limit_us(int us) try {
  const long long old_us = sb2::g_wait_limit_us;
  if (us > 0) sb2::g_wait_limit_us = us;
  return (int)std::min<long long>(old_us, INT_MAX);
} SB2_CATCH

}  // extern "C"
