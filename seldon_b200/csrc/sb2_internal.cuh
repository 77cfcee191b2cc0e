// Internal declarations shared by the libseldon_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "seldon_b200.h"

namespace sb2 {

// ----------------------------------------------------------------- tracing

// An NVTX range around a C entry point: a profiler's timeline shows each
// library call by name.  NVTX v3 is header-only and costs a few nanoseconds
// when no tool is attached.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};
#define SB2_TRACE(name) ::sb2::TraceRange sb2_trace_range_(name)

// ----------------------------------------------------------------- status

#define SB2_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t e_ = (expr);                                 \
    if (e_ != cudaSuccess) return ::sb2::map_cuda_error(e_); \
  } while (0)

#define SB2_TRY(expr)          \
  do {                         \
    int s_ = (expr);           \
    if (s_ != SB2_OK) return s_; \
  } while (0)

int map_cuda_error(cudaError_t e);

// Closes every C entry point's function-try-block: no C++ exception leaves
// the C ABI (a ctypes, cgo or JNI caller cannot catch one).
#define SB2_CATCH                          \
  catch (const std::bad_alloc&) {          \
    return SB2_ERR_NO_MEMORY;              \
  }                                        \
  catch (...) {                            \
    return SB2_ERR_HOST;                   \
  }

// ----------------------------------------------------------------- tuning

// SpMV row-block partition.  A block is either a run of consecutive rows whose
// nonzeros (<= kNnzCap) are streamed once through shared memory, or a single
// long row handled by the whole CTA.
constexpr int kSpmvThreads = 256;
constexpr int kNnzCap = 2048;      // nonzeros staged per stream block
constexpr int kRowCap = 1024;      // rows per stream block
constexpr int kLongRow = 512;      // rows longer than this get a CTA each
constexpr int kThreadRowMax = 24;  // longest row for thread-per-row reduction

enum BlockKind : unsigned char { kBlkThread = 0, kBlkWarp = 1, kBlkLong = 2 };

// Device arrays are padded so 16-byte vector loads of ind/val never leave
// the allocation: capacity rounded up to 4 plus one spare group.
inline long long padded_nnz(long long nnz) { return ((nnz + 3) / 4) * 4 + 4; }

// ----------------------------------------------------------------- matrix

struct Partition {
  int nblk = 0;
  int* d_blk = nullptr;             // [nblk+1] first row of each block
  unsigned char* d_kind = nullptr;  // [nblk]
  int4* d_desc = nullptr;           // [nblk] {r0, r1 | kind << 30, k0, k1} (TMA partition)
};

// Row pointers are padded the same way: the bulk copies of a block's row
// pointers start and end on 16-byte boundaries.
inline long long padded_rows(long long rows) { return ((rows + 1 + 3) / 4) * 4 + 4; }

// Binned sliced-ELLPACK copy of an operator (see sell.cuh).  nslice < 0:
// not applicable (more than 2^26 rows).
struct SellArrays {
  int nslice = -1;             // slices of 128 rows (4 per lane)
  long long* d_sptr = nullptr; // first group of each slice
  uint2* d_qinfo = nullptr;    // per lane: row0 (or scattered flag), 4 lengths
  int4* d_qrows = nullptr;     // per lane row ids, only when some lane is scattered
  int* d_scol = nullptr;
  double* d_sval = nullptr;
  float* d_sval32 = nullptr;  // FP32 copy (lazy, mixed precision)
  int nwarp = 0, ncta = 0;
  int* d_wrows = nullptr;
  int* d_crows = nullptr;
  long long padded = 0;       // stored entries incl. padding
  bool sorted = false;
  long long* d_pos = nullptr; // SELL position of each CSR entry of the thread
                              // bin, -1 for entries of the warp/CTA bins
};

struct CsrArrays {
  int rows = 0, cols = 0;
  long long nnz = 0;
  int* d_ptr = nullptr;     // [padded_rows]
  int* d_ind = nullptr;     // [padded_nnz]
  double* d_val = nullptr;  // [padded_nnz]
  Partition part;           // plain kernel: row blocks incl. long rows
  Partition tma;            // pipelined kernel (nblk == -1: not applicable)
  SellArrays sell;          // binned quad-row SELL (default product)
  int max_row = 0;          // longest row
};

}  // namespace sb2

struct sb2_csr {
  int device = 0;
  int m = 0, n = 0;
  int nnz_stored = 0;  // as given (upper part for symmetric)
  long long nnz = 0;   // nonzeros of the full operator
  int sym = 0;
  sb2::CsrArrays full;    // the operator (symmetric input expanded)
  sb2::CsrArrays upper;   // stored upper part (symmetric only; SOR semantics)
  sb2::CsrArrays trans;   // A^T (built on first transposed product)
  double* d_diag = nullptr;  // A(i,i) by Seldon's lookup rule (lazy)
  float* d_val32 = nullptr;  // FP32 copy of full.d_val (lazy)
  float* d_diag32 = nullptr; // FP32 copy of d_diag (lazy)
  std::mutex mu;             // guards the lazy members
  // cluster-resident CG plan (lazy; cl_ranks < 0: not planned yet, 0: no fit)
  int cl_ranks = -1, cl_rpc = 0, cl_nnz_max = 0, cl_cap = 0;
  // staging vectors of the host-buffer entry points (lazy, reused)
  double* d_hx = nullptr;
  double* d_hy = nullptr;
  std::mutex host_mu;        // one host-buffer product at a time per matrix
  // pipelined host-buffer batches (lazy): two buffers per side, copy streams
  double* d_bx[2] = {nullptr, nullptr};
  double* d_by[2] = {nullptr, nullptr};
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t e_in[2] = {nullptr, nullptr}, e_kern[2] = {nullptr, nullptr},
              e_out[2] = {nullptr, nullptr};
};

namespace sb2 {

// ----------------------------------------------------------------- helpers

int upload_csr(int rows, int cols, const int* ptr, const int* ind,
               const double* val, CsrArrays* out);
void free_csr(CsrArrays* a);
int build_partition_host(const int* ptr, int rows, Partition* out);
int build_tma_partition_host(const int* ptr, int rows, Partition* out);
int build_sell_host(const int* ptr, const int* ind, const double* val, int rows, SellArrays* out);
void free_sell(SellArrays* s);
int ensure_transpose(const sb2_csr* A);
int ensure_diag(const sb2_csr* A);
int precond_kind(const sb2_precond* M);
const sb2_csr* precond_matrix(const sb2_precond* M);
int precond_n(const sb2_precond* M);  // order of the system M applies to

// Per-(device, stream) scratch for reductions: kRedSlots partial sums and a
// completion counter that the last CTA resets to zero.
constexpr int kRedMaxBlocks = 1184;
struct RedScratch {
  double* partials = nullptr;  // [kRedMaxBlocks * 4]
  unsigned* counter = nullptr;
  double* result = nullptr;    // [8] device results of host-returning calls
  int* status = nullptr;       // bounded-wait status of kernels on this stream
};
int get_red_scratch(cudaStream_t s, RedScratch** out);

int current_device();
int num_sms(int device);
// Stream-ordered workspace allocation from the library's own memory pool
// (freed with cudaFreeAsync).
cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t s);
// The same for arrays handed to the caller: sb2_device_free returns them to
// the pool (release_owned is false for any other pointer).
cudaError_t pool_malloc_owned(void** p, size_t bytes, cudaStream_t s);
bool release_owned(void* p, cudaError_t* err);

// Launch y = beta*y + alpha*A*x (overwrite: y = alpha*A*x) on a CSR operator.
int launch_spmv(const CsrArrays& a, double alpha, const double* x, double beta,
                double* y, bool overwrite, cudaStream_t s);

// Limit of the persistent solvers' bounded grid-barrier waits, microseconds.
extern std::atomic<long long> g_wait_limit_us;
inline unsigned long long barrier_wait_ns() { return (unsigned long long)g_wait_limit_us.load() * 1000ull; }
// The TMA product's ring waits (bulk copies in flight) never use less than 1 s.
inline unsigned long long ring_wait_ns() {
  const unsigned long long ns = barrier_wait_ns();
  return ns < 1000000000ull ? 1000000000ull : ns;
}

// ----------------------------------------------------------------- device code

#ifdef __CUDACC__

// Products and sums rounded separately (no FMA contraction), matching the
// reference loops compiled without contraction.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
  // Fixed tree: lane 0 ends with ((v0+v16)+(v8+v24))... for every call.
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = add_rn(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Deterministic block sum; the result is valid in thread 0 only.  `red` must
// hold NT/32 elements of shared memory.
template <int NT, typename T>
__device__ __forceinline__ T block_sum(T v, T* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < NT / 32) ? red[lane] : T(0);
    v = warp_sum(v);
  }
  __syncthreads();
  return v;
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned atom_add_acqrel_u32(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;"
               : "=r"(old)
               : "l"(p), "r"(v)
               : "memory");
  return old;
}

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialization may start while the previous kernel of its stream finishes:
// pdl_wait() blocks until that kernel has completed and its writes are
// visible (a no-op without the launch attribute); pdl_release() lets the
// next kernel of the stream be scheduled once every CTA of this grid has
// called it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Streaming loads of the matrix (read once per product: evict first).
__device__ __forceinline__ int4 ld_stream_int4(const int* p) {
  return __ldcs(reinterpret_cast<const int4*>(p));
}
__device__ __forceinline__ void ld_stream_val4(const double* p, double v[4]) {
  double2 a = __ldcs(reinterpret_cast<const double2*>(p));
  double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ld_stream_val4(const float* p, float v[4]) {
  float4 a = __ldcs(reinterpret_cast<const float4*>(p));
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}

// 16-byte vector accesses of 4 consecutive entries (p 16-byte aligned).
template <typename T>
__device__ __forceinline__ void vld4_cs(const T* p, T (&o)[4]) {
  if constexpr (sizeof(T) == 8) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  } else {
    const float4 a = __ldcs(reinterpret_cast<const float4*>(p));
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
  }
}

template <typename T>
__device__ __forceinline__ void vld4_ldg(const T* p, T (&o)[4]) {
  if constexpr (sizeof(T) == 8) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  } else {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
  }
}

template <typename T>
__device__ __forceinline__ void vld4_cg(const T* p, T (&o)[4]) {
  if constexpr (sizeof(T) == 8) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  } else {
    const float4 a = __ldcg(reinterpret_cast<const float4*>(p));
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
  }
}

template <typename T>
__device__ __forceinline__ void vld4_ca(const T* p, T (&o)[4]) {
  if constexpr (sizeof(T) == 8) {
    const double2 a = __ldca(reinterpret_cast<const double2*>(p));
    const double2 b = __ldca(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  } else {
    const float4 a = __ldca(reinterpret_cast<const float4*>(p));
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
  }
}

template <typename T>
__device__ __forceinline__ void vst4(T* p, const T (&v)[4]) {
  if constexpr (sizeof(T) == 8) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
  } else {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
}

template <typename T>
__device__ __forceinline__ bool is_aligned16(const T* p) {
  return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

// The four columns c.x..c.w are c.x, c.x+1, c.x+2, c.x+3 and x + c.x is
// 16-byte aligned: one vector load fetches the four x values.
template <typename XT>
__device__ __forceinline__ bool quad_contiguous(const XT* x, const int4& c) {
  return c.y == c.x + 1 && c.z == c.x + 2 && c.w == c.x + 3 && is_aligned16(x + c.x);
}

#endif  // __CUDACC__

}  // namespace sb2
