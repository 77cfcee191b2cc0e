// Batched solves: thousands of independent, unevenly sized sparse systems in
// one persistent launch.
//
// The batch is a block-diagonal CSR operator with the row ranges of its
// systems.  CTAs of a persistent grid take systems from an atomic queue,
// largest first (the order is fixed when the batch is created), and run a
// whole solve per system: all reductions are CTA-wide (__syncthreads), so no
// CTA ever waits for another one.  Each system keeps its working set (its
// rows of the operator in FP32 and FP64 and its vectors) warm in L2 while the
// CTA iterates on it.
//
// Solver per system (identity preconditioner):
//   mode 0 -- FP32 conjugate gradients with reliable updates: the FP32
//             correction is added to the FP64 solution and the FP32 residual
//             replaced by the FP64 residual b - A x whenever it has dropped by
//             `update_ratio` or predicts convergence; stop on the FP64
//             relative residual < tol (Iterative.cxx:272-319 rule).
//   mode 1 -- plain FP64 CG (Cg.cxx:45-116), the reference point.
// The call does not synchronize with the host unless a summary is asked for,
// so the whole batch solve can be captured in a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <numeric>
#include <vector>

#include <cooperative_groups.h>

#include "sb2_internal.cuh"

struct sb2_batch {
  int device = 0;
  int nsys = 0, m = 0;
  long long nnz = 0;
  int* d_sys_row = nullptr;  // [nsys+1]
  int* d_order = nullptr;    // systems by decreasing size
  int* d_ptr = nullptr;      // [m+1] global CSR
  void* d_ind = nullptr;     // local column (row offset of the system subtracted):
                             // uint16 when every system has <= 65536 rows, else int32
  bool ind16 = false;
  double* d_val = nullptr;
  float* d_val32 = nullptr;
  // scratch: FP64 residual; mode 0: FP32 r, p (two), q, d; mode 1: FP64 p
  // (two), q in the same space
  double* d_r64 = nullptr;
  float* d_w32 = nullptr;
  unsigned* d_queue = nullptr;
  // plan (autotuned): CTA size, and the largest system a single warp solves
  int threads = 256;
  int warp_max = 0;
  int cluster = 0;       // CTAs of a cluster plan (0: none)
  int cluster_min = 0;   // systems of more rows are solved by a whole cluster
  int max_rows = 0;
  unsigned long long histo_key = 0;  // size histogram, for the tuned-plan cache
};

namespace sb2 {

struct BatchArgs {
  int nsys;
  const int* sys_row;
  const int* order;
  const int* ptr;
  const void* ind;
  const double* val;
  const float* val32;
  const double* b;
  double* x;
  double* r64;
  float* w32;  // 6 * m floats
  int m;
  unsigned* queue;
  double tol;
  double ratio;
  int max_iter;
  int mode;
  int init_guess_null;
  int warp_max;     // systems of at most this many rows: one warp each
  int cluster_min;  // cluster launches: systems of more rows take the whole cluster
  int* iters;       // per system (may be null)
  double* relres;   // per system (may be null)
};

// The threads that solve one system: a whole CTA, or one warp.  sums()
// reduces K per-thread values into every thread in a fixed order (a shuffle
// tree per warp, then the warps in order); the CTA form takes one
// __syncthreads, alternating between two buffers so that the next reduction
// may start while slow threads still read this one.
template <int NT>
struct CtaGroup {
  // values other threads of the group wrote (the product's gathers): the
  // SM's L1 holds the CTA's own stores
  template <typename T>
  static __device__ __forceinline__ T ld(const T* p) { return *p; }
  double* red;  // shared: 2 buffers x 2 values x NT/32 warps
  int ph;
  static constexpr int kSize = NT;
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int stride() const { return NT; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  template <int K, typename T>
  __device__ __forceinline__ void sums(T (&v)[K]) {
    constexpr int W = NT / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double* buf = red + ph * 2 * W;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const T t = warp_sum(v[k]);
      if (lane == 0) buf[k * W + w] = (double)t;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) {
      T acc = T(0);
      for (int q = 0; q < W; q++) acc = add_rn(acc, (T)buf[k * W + q]);
      v[k] = acc;
    }
    ph ^= 1;
  }
  template <typename T>
  __device__ __forceinline__ T sum(T v) {
    T o[1] = {v};
    sums<1>(o);
    return o[0];
  }
};

struct WarpGroup {
  static constexpr int kSize = 32;
  template <typename T>
  static __device__ __forceinline__ T ld(const T* p) { return *p; }
  __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
  __device__ __forceinline__ int stride() const { return 32; }
  __device__ __forceinline__ void sync() const { __syncwarp(); }
  // __syncwarp orders the lanes' memory accesses around the reduction
  // (shuffles alone do not), as __syncthreads does for the CTA form
  template <int K, typename T>
  __device__ __forceinline__ void sums(T (&v)[K]) {
    __syncwarp();
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = __shfl_sync(0xffffffffu, warp_sum(v[k]), 0);
  }
  template <typename T>
  __device__ __forceinline__ T sum(T v) {
    __syncwarp();
    return __shfl_sync(0xffffffffu, warp_sum(v), 0);
  }
};

// A whole thread-block cluster of NT-thread CTAs on one system (the largest
// systems of a cluster plan).  Rows go to threads by cluster rank.  sums():
// a shuffle tree per warp, the warps in order into the CTA's partial (in its
// shared memory), a cluster barrier, then the partials of ranks 0..C-1 in
// rank order, read through distributed shared memory.  Partials alternate
// between two buffers, so one cluster barrier per reduction suffices: no
// CTA can write a buffer again before every CTA has passed the next
// reduction's barrier, after its reads of this one.  The product's gathers
// read other CTAs' rows from L2: another SM's L1 may hold an older copy.
template <int NT>
struct ClusterGroup {
  double* red;    // shared: 2 buffers x 2 values x NT/32 warps
  double* cpart;  // shared: 2 buffers x 2 values (this CTA's partials)
  double* gath;   // shared: 2 values x 16 ranks (partials gathered)
  int ph;
  int nrank;
  int crank;
  __device__ __forceinline__ int rank() const { return crank * NT + (int)threadIdx.x; }
  __device__ __forceinline__ int stride() const { return nrank * NT; }
  __device__ __forceinline__ void sync() const { cooperative_groups::this_cluster().sync(); }
  template <typename T>
  static __device__ __forceinline__ T ld(const T* p) { return __ldcg(p); }
  template <int K, typename T>
  __device__ __forceinline__ void sums(T (&v)[K]) {
    constexpr int W = NT / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double* buf = red + ph * 2 * W;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const T t = warp_sum(v[k]);
      if (lane == 0) buf[k * W + w] = (double)t;
    }
    __syncthreads();
    if (threadIdx.x < K) {
      T acc = T(0);
      for (int q = 0; q < W; q++) acc = add_rn(acc, (T)buf[threadIdx.x * W + q]);
      cpart[ph * 2 + threadIdx.x] = (double)acc;
    }
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    cl.sync();
    if ((int)threadIdx.x < K * nrank) {
      const int k = threadIdx.x / nrank, r = threadIdx.x % nrank;
      gath[k * 16 + r] = *cl.map_shared_rank(cpart + ph * 2 + k, r);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) {
      T acc = T(0);
      for (int r = 0; r < nrank; r++) acc = add_rn(acc, (T)gath[k * 16 + r]);
      v[k] = acc;
    }
    ph ^= 1;
  }
  template <typename T>
  __device__ __forceinline__ T sum(T v) {
    T o[1] = {v};
    sums<1>(o);
    return o[0];
  }
};

// r64 = b - A x over one system (FP64, entries in stored order); returns
// ||r64||^2 in every thread of the group.  x must be complete (synced).
template <class G, typename IT>
__device__ double fp64_residual(G& g, const BatchArgs& a, int r0, int n, const double* xs) {
  const IT* __restrict__ ind = static_cast<const IT*>(a.ind);
  double acc = 0.0;
  for (int i = g.rank(); i < n; i += g.stride()) {
    const int k0 = __ldg(a.ptr + r0 + i), k1 = __ldg(a.ptr + r0 + i + 1);
    double t = 0.0;
    for (int k = k0; k < k1; k++) t = add_rn(t, mul_rn(__ldg(a.val + k), G::ld(xs + __ldg(ind + k))));
    const double v = add_rn(__ldg(a.b + r0 + i), -t);
    a.r64[r0 + i] = v;
    acc = add_rn(acc, mul_rn(v, v));
  }
  return g.sum(acc);
}

// p = first ? r : beta*p + zc*r on the group's rows (Mlt(beta, p); Add(zc, r, p)).
template <class G, typename T>
__device__ __forceinline__ void direction(G& g, int n, const T* __restrict__ r, T* __restrict__ p,
                                          bool first, T beta, T zc) {
  for (int i = g.rank(); i < n; i += g.stride())
    p[i] = first ? r[i] : add_rn(mul_rn(p[i], beta), mul_rn(zc, r[i]));
}

// q = A p over one system (entries in stored order) with (p, q), summed over
// the group (its reduction orders the writes of q before any later read).
template <class G, typename IT, typename VT, typename T>
__device__ __forceinline__ T product_dot(G& g, const BatchArgs& a, const VT* __restrict__ val,
                                         int r0, int n, const T* __restrict__ p,
                                         T* __restrict__ q) {
  const IT* __restrict__ ind = static_cast<const IT*>(a.ind);
  T pq = T(0);
  for (int i = g.rank(); i < n; i += g.stride()) {
    const int k0 = __ldg(a.ptr + r0 + i), k1 = __ldg(a.ptr + r0 + i + 1);
    T t = T(0);
    for (int k = k0; k < k1; k++) t = add_rn(t, mul_rn(T(__ldg(val + k)), G::ld(p + __ldg(ind + k))));
    q[i] = t;
    pq = add_rn(pq, mul_rn(p[i], t));
  }
  return g.sum(pq);
}

// Plain FP64 CG (Cg.cxx:45-116, identity preconditioner).
template <class G, typename IT>
__device__ void solve_fp64(G& g, const BatchArgs& a, int s, int r0, int n, double nb) {
  double* x = a.x + r0;
  double* r = a.r64 + r0;
  double* p = reinterpret_cast<double*>(a.w32) + r0;
  double* q = reinterpret_cast<double*>(a.w32) + 2 * (size_t)a.m + r0;
  double rr;
  if (a.init_guess_null) {
    double acc = 0.0;
    for (int i = g.rank(); i < n; i += g.stride()) {
      x[i] = 0.0;
      const double bi = __ldg(a.b + r0 + i);
      r[i] = bi;
      acc = add_rn(acc, mul_rn(bi, bi));
    }
    rr = g.sum(acc);
  } else {
    rr = fp64_residual<G, IT>(g, a, r0, n, x);
  }
  const double facteur = 1.0 / nb;
  double rho = rr, rho_1 = 1.0, res = facteur * sqrt(rr), beta = 0.0;
  int it = 0;
  while (!(res < a.tol) && it < a.max_iter) {
    if (rho == 0.0) break;
    direction(g, n, r, p, it == 0, beta, 1.0);
    g.sync();
    const double delta = product_dot<G, IT, double, double>(g, a, a.val, r0, n, p, q);
    if (delta == 0.0) break;
    const double alpha = rho / delta;
    double acc = 0.0;
    for (int i = g.rank(); i < n; i += g.stride()) {
      x[i] = add_rn(x[i], mul_rn(alpha, p[i]));
      const double ri = add_rn(r[i], mul_rn(-alpha, q[i]));
      r[i] = ri;
      acc = add_rn(acc, mul_rn(ri, ri));
    }
    rr = g.sum(acc);
    rho_1 = rho;
    rho = rr;
    beta = rho / rho_1;
    res = facteur * sqrt(rr);
    it++;
  }
  if (g.rank() == 0) {
    if (a.iters) a.iters[s] = it;
    if (a.relres) a.relres[s] = res;
  }
}

// FP32 CG with FP64 reliable updates.
template <class G, typename IT>
__device__ void solve_mixed(G& g, const BatchArgs& a, int s, int r0, int n, double nb) {
  double* x = a.x + r0;
  float* r = a.w32 + r0;
  float* p = a.w32 + (size_t)a.m + r0;
  float* q = a.w32 + 3 * (size_t)a.m + r0;
  float* d = a.w32 + 4 * (size_t)a.m + r0;
  if (a.init_guess_null)
    for (int i = g.rank(); i < n; i += g.stride()) x[i] = 0.0;
  g.sync();
  double rr64 = fp64_residual<G, IT>(g, a, r0, n, x);
  double res = sqrt(rr64) / nb;
  int it = 0;
  if (res < a.tol) {
    if (g.rank() == 0) {
      if (a.iters) a.iters[s] = 0;
      if (a.relres) a.relres[s] = res;
    }
    return;
  }
  const float fnb = (float)nb;
  float acc = 0.0f;
  for (int i = g.rank(); i < n; i += g.stride()) {
    const float ri = (float)a.r64[r0 + i];
    r[i] = ri;
    d[i] = 0.0f;
    acc = add_rn(acc, mul_rn(ri, ri));
  }
  float rho = g.sum(acc), rho_1 = 1.0f, zc = 1.0f, beta = 0.0f;
  float rmax = sqrtf(rho);
  bool first = true;
  for (;;) {
    direction(g, n, r, p, first, beta, zc);
    g.sync();
    const float delta = product_dot<G, IT, float, float>(g, a, a.val32, r0, n, p, q);
    first = false;
    zc = 1.0f;
    if (delta == 0.0f) break;
    const float alpha = rho / delta;
    acc = 0.0f;
    for (int i = g.rank(); i < n; i += g.stride()) {
      d[i] = add_rn(d[i], mul_rn(alpha, p[i]));
      const float ri = add_rn(r[i], mul_rn(-alpha, q[i]));
      r[i] = ri;
      acc = add_rn(acc, mul_rn(ri, ri));
    }
    const float rr = g.sum(acc);
    it++;
    const float rn = sqrtf(rr);
    const bool correct = (rn / fnb < (float)a.tol) || (rn < (float)a.ratio * rmax) ||
                         it >= a.max_iter;
    if (!correct) {
      rho_1 = rho;
      rho = rr;
      beta = rho / rho_1;
      continue;
    }
    // FP64 correction: x += d, d = 0, r64 = b - A x
    for (int i = g.rank(); i < n; i += g.stride()) {
      x[i] = add_rn(x[i], (double)d[i]);
      d[i] = 0.0f;
    }
    g.sync();
    rr64 = fp64_residual<G, IT>(g, a, r0, n, x);
    res = sqrt(rr64) / nb;
    if (res < a.tol || it >= a.max_iter) break;
    // replace the FP32 residual; keep the direction, minus its component
    // along the new residual
    float v2[2] = {0.0f, 0.0f};
    for (int i = g.rank(); i < n; i += g.stride()) {
      const float ri = (float)a.r64[r0 + i];
      r[i] = ri;
      v2[0] = add_rn(v2[0], mul_rn(ri, ri));
      v2[1] = add_rn(v2[1], mul_rn(ri, p[i]));
    }
    g.sums(v2);
    rmax = sqrtf(v2[0]);
    rho_1 = rho;
    rho = v2[0];
    if (rho == 0.0f) break;
    beta = rho / rho_1;
    zc = 1.0f - beta * (v2[1] / rho);
  }
  if (g.rank() == 0) {
    if (a.iters) a.iters[s] = it;
    if (a.relres) a.relres[s] = res;
  }
}

template <class G, typename IT>
__device__ void solve_system(G& g, const BatchArgs& a, int s) {
  const int r0 = __ldg(a.sys_row + s), n = __ldg(a.sys_row + s + 1) - r0;
  double acc = 0.0;
  for (int i = g.rank(); i < n; i += g.stride()) {
    const double bi = __ldg(a.b + r0 + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  const double nb = sqrt(g.sum(acc));
  if (nb == 0.0) {  // zero right-hand side: x untouched (Iterative.cxx:240-241)
    if (g.rank() == 0) {
      if (a.iters) a.iters[s] = 0;
      if (a.relres) a.relres[s] = 0.0;
    }
    return;
  }
  if (a.mode == 1)
    solve_fp64<G, IT>(g, a, s, r0, n, nb);
  else
    solve_mixed<G, IT>(g, a, s, r0, n, nb);
}

// One persistent launch.  CTAs take systems from the queue (largest first)
// and solve each with all their threads; the first system of at most
// warp_max rows that a CTA takes switches it to warps: from then on (every
// later system is as small or smaller) each warp takes and solves systems on
// its own, with shuffle reductions and no CTA barrier.  In a cluster launch
// (CLUSTER) the clusters first take the systems of more than cluster_min
// rows, one system per cluster; the first smaller system a cluster takes
// goes to its rank-0 CTA, and from then on its CTAs take systems alone.
template <int NT, typename IT, bool WARPS, bool CLUSTER>
__global__ void __launch_bounds__(NT, 1536 / NT) batch_kernel(BatchArgs a) {
  __shared__ int s_sys;
  __shared__ double s_red[2 * 2 * (NT / 32)];
  CtaGroup<NT> cg{s_red, 0};
  int carry = -1;  // a system taken in the cluster phase that this CTA solves alone
  if constexpr (CLUSTER) {
    __shared__ double s_cpart[4];
    __shared__ double s_gath[2 * 16];
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    ClusterGroup<NT> clg{s_red, s_cpart, s_gath, 0, (int)cl.num_blocks(), (int)cl.block_rank()};
    for (;;) {
      if (clg.crank == 0 && threadIdx.x == 0) {
        const unsigned k = atomicAdd(a.queue, 1u);
        const int t = (k < (unsigned)a.nsys) ? __ldg(a.order + k) : -1;
        for (int r = 0; r < clg.nrank; r++) *cl.map_shared_rank(&s_sys, r) = t;
      }
      cl.sync();
      const int s = s_sys;
      cl.sync();  // every CTA has read s_sys before rank 0 writes it again
      if (s < 0) return;
      if (__ldg(a.sys_row + s + 1) - __ldg(a.sys_row + s) <= a.cluster_min) {
        if (clg.crank == 0) carry = s;
        break;
      }
      solve_system<ClusterGroup<NT>, IT>(clg, a, s);
    }
  }
  int small = -1;
  for (;;) {
    int s = carry;
    carry = -1;
    if (s < 0) {
      if (threadIdx.x == 0) {
        const unsigned k = atomicAdd(a.queue, 1u);
        s_sys = (k < (unsigned)a.nsys) ? __ldg(a.order + k) : -1;
      }
      __syncthreads();
      s = s_sys;
      __syncthreads();
      if (s < 0) return;
    }
    if (WARPS && __ldg(a.sys_row + s + 1) - __ldg(a.sys_row + s) <= a.warp_max) {
      small = s;
      break;
    }
    solve_system<CtaGroup<NT>, IT>(cg, a, s);
    __syncthreads();
  }
  if constexpr (WARPS) {
  WarpGroup wg;
  const int lane = threadIdx.x & 31;
  int s = (threadIdx.x >> 5) == 0 ? small : -2;
  for (;;) {
    if (s == -2) {
      int t = -1;
      if (lane == 0) {
        const unsigned k = atomicAdd(a.queue, 1u);
        t = (k < (unsigned)a.nsys) ? __ldg(a.order + k) : -1;
      }
      s = __shfl_sync(0xffffffffu, t, 0);
    }
    if (s < 0) return;
    solve_system<WarpGroup, IT>(wg, a, s);
    __syncwarp();
    s = -2;
  }
  }
}

// Clusters of `cluster` CTAs that one GPU holds at once for this kernel
// (0: the launch cannot be scheduled).
template <int NT, typename IT, bool WARPS>
static int cluster_grid(int cluster) {
  auto* k = batch_kernel<NT, IT, WARPS, true>;
  if (cluster > 8 &&
      cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster);
  cfg.blockDim = dim3(NT);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

template <int NT, typename IT, bool WARPS>
static int launch_batch(const BatchArgs& a, int cluster, cudaStream_t s) {
  if (cluster >= 2) {
    const int nc = cluster_grid<NT, IT, WARPS>(cluster);
    if (nc < 1) return SB2_ERR_NOT_SUPPORTED;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nc * cluster);
    cfg.blockDim = dim3(NT);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SB2_CUDA_TRY(cudaLaunchKernelEx(&cfg, batch_kernel<NT, IT, WARPS, true>, a));
    return SB2_OK;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<NT, IT, WARPS, false>,
                                                    NT, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int grid = std::min(a.nsys, per_sm * num_sms(current_device()));
  batch_kernel<NT, IT, WARPS, false><<<std::max(grid, 1), NT, 0, s>>>(a);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

// the kernel without the warp path (warp_max == 0) keeps fewer registers
template <typename IT, bool WARPS>
static int launch_batch_w(const BatchArgs& a, int threads, int cluster, cudaStream_t s) {
  switch (threads) {
    case 128: return launch_batch<128, IT, WARPS>(a, cluster, s);
    case 512: return launch_batch<512, IT, WARPS>(a, cluster, s);
    default: return launch_batch<256, IT, WARPS>(a, cluster, s);
  }
}

template <typename IT>
static int launch_batch_t(const BatchArgs& a, int threads, int cluster, cudaStream_t s) {
  return a.warp_max > 0 ? launch_batch_w<IT, true>(a, threads, cluster, s)
                        : launch_batch_w<IT, false>(a, threads, cluster, s);
}

static int batch_run(const sb2_batch* B, double* x, const double* b, const sb2_batch_params* prm,
                     int* iters, double* relres, int threads, int warp_max, int cluster,
                     int cluster_min, cudaStream_t s) {
  BatchArgs a{B->nsys, B->d_sys_row, B->d_order, B->d_ptr, B->d_ind, B->d_val, B->d_val32,
              b, x, B->d_r64, B->d_w32, B->m, B->d_queue, prm->tol, prm->update_ratio,
              prm->max_iter, prm->mode, prm->init_guess_null, warp_max, cluster_min, iters,
              relres};
  SB2_CUDA_TRY(cudaMemsetAsync(B->d_queue, 0, sizeof(unsigned), s));
  return B->ind16 ? launch_batch_t<unsigned short>(a, threads, cluster, s)
                  : launch_batch_t<int>(a, threads, cluster, s);
}

__global__ void batch_ind16(long long n, const int* __restrict__ a, unsigned short* __restrict__ b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (unsigned short)a[i];
}

__global__ void batch_to_float(long long n, const double* __restrict__ a, float* __restrict__ b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// Key of the tuned-plan cache: the count of systems in each power-of-two
// row-count class (and the number of systems), hashed.
static unsigned long long size_histogram_key(int nsys, const int* sys_row) {
  int cnt[33] = {0};
  for (int s = 0; s < nsys; s++) {
    unsigned v = (unsigned)(sys_row[s + 1] - sys_row[s]);
    int c = 0;
    while (v) {
      v >>= 1;
      c++;
    }
    cnt[c]++;
  }
  unsigned long long h = 1469598103934665603ull ^ (unsigned long long)nsys;
  for (int c = 0; c < 33; c++) {
    h ^= (unsigned long long)cnt[c] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    h *= 1099511628211ull;
  }
  return h;
}

struct BatchPlan {
  int threads, warp_max, cluster, cluster_min;
};
// Plans chosen by sb2_batch_autotune, per (size histogram, mode): a later
// batch with the same histogram takes its plan without timing.
static std::mutex g_plan_mu;
static std::map<std::pair<unsigned long long, int>, BatchPlan> g_plans;

}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_batch_create(int nsys, const int* sys_row, const int* ptr, const int* ind,
                     const double* val, sb2_batch** out) try {
  if (!out || nsys < 0 || !sys_row || !ptr) return SB2_ERR_INVALID_VALUE;
  *out = nullptr;
  // validation, each pass reading only what the previous one proved in
  // range: monotone system ranges from 0, then monotone row pointers from 0,
  // then every entry inside its own system
  if (sys_row[0] != 0) return SB2_ERR_INVALID_CSR;
  int maxrows = 0;
  for (int s = 0; s < nsys; s++) {
    if (sys_row[s + 1] < sys_row[s]) return SB2_ERR_INVALID_CSR;
    maxrows = std::max(maxrows, sys_row[s + 1] - sys_row[s]);
  }
  const int m = sys_row[nsys];
  if (ptr[0] != 0) return SB2_ERR_INVALID_CSR;
  for (int i = 0; i < m; i++)
    if (ptr[i + 1] < ptr[i]) return SB2_ERR_INVALID_CSR;
  const long long nnz = ptr[m];
  if (nnz > 0 && (!ind || !val)) return SB2_ERR_INVALID_VALUE;
  std::vector<int> local(std::max<long long>(nnz, 1));
  for (int s = 0; s < nsys; s++) {
    const int a = sys_row[s], e = sys_row[s + 1];
    for (int i = a; i < e; i++)
      for (int k = ptr[i]; k < ptr[i + 1]; k++) {
        if (ind[k] < a || ind[k] >= e) return SB2_ERR_INVALID_CSR;
        local[k] = ind[k] - a;
      }
  }
  std::vector<int> order(nsys);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
    return (sys_row[p + 1] - sys_row[p]) > (sys_row[q + 1] - sys_row[q]);
  });
  sb2_batch* B = new sb2_batch();
  B->device = current_device();
  B->nsys = nsys;
  B->m = m;
  B->nnz = nnz;
  B->max_rows = maxrows;
  B->histo_key = size_histogram_key(nsys, sys_row);
  cudaError_t e = cudaMalloc(&B->d_sys_row, sizeof(int) * (nsys + 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_order, sizeof(int) * std::max(nsys, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_ptr, sizeof(int) * (m + 1));
  B->ind16 = (maxrows <= 65536);
  if (e == cudaSuccess) e = cudaMalloc(&B->d_ind, (B->ind16 ? sizeof(unsigned short) : sizeof(int)) *
                                                      std::max<long long>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_val, sizeof(double) * std::max<long long>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_val32, sizeof(float) * std::max<long long>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_r64, sizeof(double) * std::max(m, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_w32, sizeof(float) * 6 * (size_t)std::max(m, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_queue, sizeof(unsigned) * 4);
  if (e == cudaSuccess) e = cudaMemcpy(B->d_sys_row, sys_row, sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nsys) e = cudaMemcpy(B->d_order, order.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B->d_ptr, ptr, sizeof(int) * (m + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz && !B->ind16)
    e = cudaMemcpy(B->d_ind, local.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz && B->ind16) {
    // 2-byte local columns: stage the 4-byte ones and narrow them on the device
    int* tmp = nullptr;
    e = cudaMalloc(&tmp, sizeof(int) * nnz);
    if (e == cudaSuccess) e = cudaMemcpy(tmp, local.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      batch_ind16<<<num_sms(B->device) * 8, 256>>>(nnz, tmp, static_cast<unsigned short*>(B->d_ind));
      e = cudaDeviceSynchronize();
    }
    cudaFree(tmp);
  }
  if (e == cudaSuccess && nnz) e = cudaMemcpy(B->d_val, val, sizeof(double) * nnz, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz) {
    batch_to_float<<<num_sms(B->device) * 8, 256>>>(nnz, B->d_val, B->d_val32);
    e = cudaDeviceSynchronize();
  }
  if (e != cudaSuccess) {
    sb2_batch_destroy(B);
    return map_cuda_error(e);
  }
  *out = B;
  return SB2_OK;
} SB2_CATCH

int sb2_batch_destroy(sb2_batch* B) try {
  if (!B) return SB2_OK;
  cudaFree(B->d_sys_row);
  cudaFree(B->d_order);
  cudaFree(B->d_ptr);
  cudaFree(B->d_ind);
  cudaFree(B->d_val);
  cudaFree(B->d_val32);
  cudaFree(B->d_r64);
  cudaFree(B->d_w32);
  cudaFree(B->d_queue);
  delete B;
  return SB2_OK;
} SB2_CATCH

int sb2_batch_solve(const sb2_batch* B, double* x, const double* b, const sb2_batch_params* prm,
                    int* d_iters, double* d_relres, sb2_batch_result* result, void* stream) try {
  SB2_TRACE("sb2_batch_solve");
  if (!B || !prm || (B->m > 0 && (!x || !b)) || x == b) return SB2_ERR_INVALID_VALUE;
  if (prm->mode < 0 || prm->mode > 1) return SB2_ERR_INVALID_VALUE;
  cudaStream_t s = (cudaStream_t)stream;
  if (B->nsys == 0) {
    if (result) *result = sb2_batch_result{};
    return SB2_OK;
  }
  SB2_TRY(batch_run(B, x, b, prm, d_iters, d_relres, B->threads, B->warp_max, B->cluster,
                    B->cluster_min, s));
  if (!result) return SB2_OK;
  // host summary (synchronizes): per-system counts and residuals
  std::vector<int> it(B->nsys);
  std::vector<double> rr(B->nsys);
  int* di = d_iters;
  double* dr = d_relres;
  if (!di || !dr) return SB2_ERR_INVALID_VALUE;  // the summary is built from them
  SB2_CUDA_TRY(cudaMemcpyAsync(it.data(), di, sizeof(int) * B->nsys, cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaMemcpyAsync(rr.data(), dr, sizeof(double) * B->nsys, cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  sb2_batch_result R{};
  for (int k = 0; k < B->nsys; k++) {
    R.total_iter += it[k];
    R.max_iter = std::max(R.max_iter, it[k]);
    R.max_rel_residual = std::max(R.max_rel_residual, rr[k]);
    if (rr[k] < prm->tol) R.converged++;
  }
  *result = R;
  return SB2_OK;
} SB2_CATCH

int sb2_batch_set_threads(sb2_batch* B, int threads) try {
  if (!B || (threads != 128 && threads != 256 && threads != 512)) return SB2_ERR_INVALID_VALUE;
  B->threads = threads;
  return SB2_OK;
} SB2_CATCH

int sb2_batch_get_threads(const sb2_batch* B) { return B ? B->threads : 0; }

int sb2_batch_set_plan(sb2_batch* B, int threads, int warp_max) try {
  if (!B || (threads != 128 && threads != 256 && threads != 512) || warp_max < 0)
    return SB2_ERR_INVALID_VALUE;
  B->threads = threads;
  B->warp_max = warp_max;
  B->cluster = 0;
  B->cluster_min = 0;
  return SB2_OK;
} SB2_CATCH

int sb2_batch_set_cluster_plan(sb2_batch* B, int cluster, int cluster_min) try {
  if (!B || (cluster != 0 && cluster != 2 && cluster != 4 && cluster != 8 && cluster != 16) ||
      cluster_min < 0)
    return SB2_ERR_INVALID_VALUE;
  B->cluster = cluster;
  B->cluster_min = cluster ? cluster_min : 0;
  return SB2_OK;
} SB2_CATCH

int sb2_batch_get_cluster_plan(const sb2_batch* B, int* cluster, int* cluster_min) try {
  if (!B || !cluster || !cluster_min) return SB2_ERR_INVALID_VALUE;
  *cluster = B->cluster;
  *cluster_min = B->cluster_min;
  return SB2_OK;
} SB2_CATCH

int sb2_batch_get_plan(const sb2_batch* B, int* threads, int* warp_max) try {
  if (!B || !threads || !warp_max) return SB2_ERR_INVALID_VALUE;
  *threads = B->threads;
  *warp_max = B->warp_max;
  return SB2_OK;
} SB2_CATCH

}  // extern "C"

extern "C" int sb2_batch_autotune(sb2_batch* B, double* x, const double* b,
                                  const sb2_batch_params* prm, void* stream) try {
  if (!B || !prm) return SB2_ERR_INVALID_VALUE;
  if (B->nsys == 0) return SB2_OK;
  const std::pair<unsigned long long, int> key{B->histo_key, prm->mode};
  {
    std::lock_guard<std::mutex> g(sb2::g_plan_mu);
    auto it = sb2::g_plans.find(key);
    if (it != sb2::g_plans.end()) {
      B->threads = it->second.threads;
      B->warp_max = it->second.warp_max;
      B->cluster = it->second.cluster;
      B->cluster_min = it->second.cluster_min;
      return SB2_OK;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  SB2_CUDA_TRY(cudaEventCreate(&e0));
  SB2_CUDA_TRY(cudaEventCreate(&e1));
  float best = 1e30f;
  sb2::BatchPlan bp{B->threads, B->warp_max, B->cluster, B->cluster_min};
  int st = SB2_OK;
  // one untimed run, one timed run of the same solve; a cluster plan the
  // GPU cannot schedule is skipped
  auto trial = [&](const sb2::BatchPlan& p) {
    int r = sb2::batch_run(B, x, b, prm, nullptr, nullptr, p.threads, p.warp_max, p.cluster,
                           p.cluster_min, s);
    if (r == SB2_ERR_NOT_SUPPORTED) return SB2_OK;
    if (r != SB2_OK) return r;
    cudaEventRecord(e0, s);
    r = sb2::batch_run(B, x, b, prm, nullptr, nullptr, p.threads, p.warp_max, p.cluster,
                       p.cluster_min, s);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) r = SB2_ERR_CUDA;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r == SB2_OK && ms < best) {
      best = ms;
      bp = p;
    }
    return r;
  };
  // CTA sizes x the largest system one warp solves (0: none)
  const int cand_t[3] = {128, 256, 512};
  const int cand_w[3] = {0, 256, 1024};
  for (int ci = 0; ci < 9 && st == SB2_OK; ci++) {
    const int t = cand_t[ci / 3], w = cand_w[ci % 3];
    if (w > 0 && ci % 3 > 0 && cand_w[ci % 3 - 1] >= B->max_rows) continue;  // same plan as a smaller w
    st = trial(sb2::BatchPlan{t, w, 0, 0});
  }
  // then clusters of 4 or 16 CTAs for the systems above half or an eighth of
  // the largest, on the best plan's CTA size and warp systems
  const sb2::BatchPlan base = bp;
  const int cand_c[2] = {4, 16};
  const int cand_m[2] = {B->max_rows / 2, B->max_rows / 8};
  for (int ci = 0; ci < 4 && st == SB2_OK; ci++)
    st = trial(sb2::BatchPlan{base.threads, base.warp_max, cand_c[ci / 2], cand_m[ci % 2]});
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st == SB2_OK) {
    B->threads = bp.threads;
    B->warp_max = bp.warp_max;
    B->cluster = bp.cluster;
    B->cluster_min = bp.cluster_min;
    std::lock_guard<std::mutex> g(sb2::g_plan_mu);
    sb2::g_plans[key] = bp;
  }
  return st;
} SB2_CATCH
