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
#include <numeric>
#include <vector>

#include "sb2_internal.cuh"

struct sb2_batch {
  int device = 0;
  int nsys = 0, m = 0;
  long long nnz = 0;
  int* d_sys_row = nullptr;  // [nsys+1]
  int* d_order = nullptr;    // systems by decreasing size
  int* d_ptr = nullptr;      // [m+1] global CSR
  int* d_ind = nullptr;      // local column (row offset of the system subtracted)
  double* d_val = nullptr;
  float* d_val32 = nullptr;
  // scratch: FP64 residual, FP32 r, p, q, d
  double* d_r64 = nullptr;
  float* d_w32 = nullptr;
  unsigned* d_queue = nullptr;
  int threads = 256;         // CTA size (autotuned)
  int max_rows = 0;
};

namespace sb2 {

struct BatchArgs {
  int nsys;
  const int* sys_row;
  const int* order;
  const int* ptr;
  const int* ind;
  const double* val;
  const float* val32;
  const double* b;
  double* x;
  double* r64;
  float* w32;  // 4 * m floats: r, p, q, d
  int m;
  unsigned* queue;
  double tol;
  double ratio;
  int max_iter;
  int mode;
  int init_guess_null;
  int* iters;       // per system (may be null)
  double* relres;   // per system (may be null)
};

template <int NT, typename T>
__device__ __forceinline__ T cta_sum(T v, T* red) {
  v = block_sum<NT>(v, red);
  __shared__ T s_bcast;
  if (threadIdx.x == 0) s_bcast = v;
  __syncthreads();
  const T out = s_bcast;
  __syncthreads();
  return out;
}

// y_i = sum_j A_ij x_j over the rows [r0, r1) of one system, thread per row,
// entries in stored order.
template <typename VT, typename XT, typename AT>
__device__ __forceinline__ AT row_dot(const int* __restrict__ ptr, const int* __restrict__ ind,
                                      const VT* __restrict__ val, const XT* __restrict__ x,
                                      int i) {
  const int a = __ldg(ptr + i), e = __ldg(ptr + i + 1);
  AT t = AT(0);
  for (int k = a; k < e; k++) t = add_rn(t, mul_rn(AT(__ldg(val + k)), AT(x[__ldg(ind + k)])));
  return t;
}

// r64 = b - A x (FP64, x in local indexing at xs), returns ||r64||^2.
template <int NT>
__device__ double fp64_residual(const BatchArgs& a, int r0, int n, const double* xs,
                                double* red) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) {
    const double t = row_dot<double, double, double>(a.ptr + r0, a.ind, a.val, xs, i);
    const double v = add_rn(__ldg(a.b + r0 + i), -t);
    a.r64[r0 + i] = v;
    acc = add_rn(acc, mul_rn(v, v));
  }
  __syncthreads();
  return cta_sum<NT>(acc, red);
}

template <int NT>
__device__ void solve_fp64(const BatchArgs& a, int s, int r0, int n, double nb) {
  __shared__ double red[NT / 32];
  double* x = a.x + r0;
  double* r = a.r64 + r0;
  // FP64 work vectors in the FP32 scratch: p and q take two floats each
  double* p = reinterpret_cast<double*>(a.w32) + r0;
  double* q = reinterpret_cast<double*>(a.w32 + a.m * 2) + r0;
  double rr;
  if (a.init_guess_null) {
    for (int i = threadIdx.x; i < n; i += NT) {
      x[i] = 0.0;
      r[i] = __ldg(a.b + r0 + i);
    }
    rr = nb * nb;
    __syncthreads();
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) acc = add_rn(acc, mul_rn(r[i], r[i]));
    rr = cta_sum<NT>(acc, red);
  } else {
    rr = fp64_residual<NT>(a, r0, n, x, red);
  }
  const double facteur = 1.0 / nb;
  double rho = rr, rho_1 = 1.0, res = facteur * sqrt(rr);
  int it = 0;
  while (!(res < a.tol) && it < a.max_iter) {
    if (rho == 0.0) break;
    const double beta = rho / rho_1;
    for (int i = threadIdx.x; i < n; i += NT) p[i] = (it == 0) ? r[i] : add_rn(mul_rn(p[i], beta), r[i]);
    __syncthreads();
    double pq = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
      const double t = row_dot<double, double, double>(a.ptr + r0, a.ind, a.val, p, i);
      q[i] = t;
      pq = add_rn(pq, mul_rn(p[i], t));
    }
    const double delta = cta_sum<NT>(pq, red);
    if (delta == 0.0) break;
    const double alpha = rho / delta;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
      x[i] = add_rn(x[i], mul_rn(alpha, p[i]));
      const double ri = add_rn(r[i], mul_rn(-alpha, q[i]));
      r[i] = ri;
      acc = add_rn(acc, mul_rn(ri, ri));
    }
    rr = cta_sum<NT>(acc, red);
    rho_1 = rho;
    rho = rr;
    res = facteur * sqrt(rr);
    it++;
  }
  if (threadIdx.x == 0) {
    if (a.iters) a.iters[s] = it;
    if (a.relres) a.relres[s] = res;
  }
}

template <int NT>
__device__ void solve_mixed(const BatchArgs& a, int s, int r0, int n, double nb) {
  __shared__ double red64[NT / 32];
  __shared__ float red32[NT / 32];
  double* x = a.x + r0;
  float* r = a.w32 + r0;
  float* p = a.w32 + a.m + r0;
  float* q = a.w32 + 2 * (size_t)a.m + r0;
  float* d = a.w32 + 3 * (size_t)a.m + r0;
  if (a.init_guess_null)
    for (int i = threadIdx.x; i < n; i += NT) x[i] = 0.0;
  __syncthreads();
  double rr64 = fp64_residual<NT>(a, r0, n, x, red64);
  double res = sqrt(rr64) / nb;
  int it = 0;
  if (res < a.tol) {
    if (threadIdx.x == 0) {
      if (a.iters) a.iters[s] = 0;
      if (a.relres) a.relres[s] = res;
    }
    return;
  }
  const float fnb = (float)nb;
  for (int i = threadIdx.x; i < n; i += NT) {
    r[i] = (float)a.r64[r0 + i];
    d[i] = 0.0f;
  }
  __syncthreads();
  float acc = 0.0f;
  for (int i = threadIdx.x; i < n; i += NT) acc = add_rn(acc, mul_rn(r[i], r[i]));
  float rho = cta_sum<NT>(acc, red32), rho_1 = 1.0f, zc = 1.0f;
  float rmax = sqrtf(rho);
  bool first = true;
  for (;;) {
    const float beta = first ? 0.0f : rho / rho_1;
    for (int i = threadIdx.x; i < n; i += NT)
      p[i] = first ? r[i] : add_rn(mul_rn(p[i], beta), mul_rn(zc, r[i]));
    __syncthreads();
    first = false;
    zc = 1.0f;
    float pq = 0.0f;
    for (int i = threadIdx.x; i < n; i += NT) {
      const float t = row_dot<float, float, float>(a.ptr + r0, a.ind, a.val32, p, i);
      q[i] = t;
      pq = add_rn(pq, mul_rn(p[i], t));
    }
    const float delta = cta_sum<NT>(pq, red32);
    if (delta == 0.0f) break;
    const float alpha = rho / delta;
    acc = 0.0f;
    for (int i = threadIdx.x; i < n; i += NT) {
      d[i] = add_rn(d[i], mul_rn(alpha, p[i]));
      const float ri = add_rn(r[i], mul_rn(-alpha, q[i]));
      r[i] = ri;
      acc = add_rn(acc, mul_rn(ri, ri));
    }
    const float rr = cta_sum<NT>(acc, red32);
    it++;
    const float rn = sqrtf(rr);
    const bool correct = (rn / fnb < (float)a.tol) || (rn < (float)a.ratio * rmax) ||
                         it >= a.max_iter;
    if (!correct) {
      rho_1 = rho;
      rho = rr;
      continue;
    }
    // FP64 correction: x += d, d = 0, r64 = b - A x
    for (int i = threadIdx.x; i < n; i += NT) {
      x[i] = add_rn(x[i], (double)d[i]);
      d[i] = 0.0f;
    }
    __syncthreads();
    rr64 = fp64_residual<NT>(a, r0, n, x, red64);
    res = sqrt(rr64) / nb;
    if (res < a.tol || it >= a.max_iter) break;
    // replace the FP32 residual; keep the direction, minus its component
    // along the new residual
    float r2 = 0.0f, rp = 0.0f;
    for (int i = threadIdx.x; i < n; i += NT) {
      const float ri = (float)a.r64[r0 + i];
      r[i] = ri;
      r2 = add_rn(r2, mul_rn(ri, ri));
      rp = add_rn(rp, mul_rn(ri, p[i]));
    }
    r2 = cta_sum<NT>(r2, red32);
    rp = cta_sum<NT>(rp, red32);
    rmax = sqrtf(r2);
    rho_1 = rho;
    rho = r2;
    if (rho == 0.0f) break;
    zc = 1.0f - (rho / rho_1) * (rp / rho);
  }
  if (threadIdx.x == 0) {
    if (a.iters) a.iters[s] = it;
    if (a.relres) a.relres[s] = res;
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) batch_kernel(BatchArgs a) {
  __shared__ int s_sys;
  __shared__ double red[NT / 32];
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned k = atomicAdd(a.queue, 1u);
      s_sys = (k < (unsigned)a.nsys) ? __ldg(a.order + k) : -1;
    }
    __syncthreads();
    const int s = s_sys;
    __syncthreads();
    if (s < 0) return;
    const int r0 = __ldg(a.sys_row + s), n = __ldg(a.sys_row + s + 1) - r0;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
      const double bi = __ldg(a.b + r0 + i);
      acc = add_rn(acc, mul_rn(bi, bi));
    }
    const double nb = sqrt(cta_sum<NT>(acc, red));
    if (nb == 0.0) {  // zero right-hand side: x untouched (Iterative.cxx:240-241)
      if (threadIdx.x == 0) {
        if (a.iters) a.iters[s] = 0;
        if (a.relres) a.relres[s] = 0.0;
      }
      continue;
    }
    if (a.mode == 1)
      solve_fp64<NT>(a, s, r0, n, nb);
    else
      solve_mixed<NT>(a, s, r0, n, nb);
    __syncthreads();
  }
}

template <int NT>
static int launch_batch(const BatchArgs& a, cudaStream_t s) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<NT>, NT, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int grid = std::min(a.nsys, per_sm * num_sms(current_device()));
  batch_kernel<NT><<<std::max(grid, 1), NT, 0, s>>>(a);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

static int batch_run(const sb2_batch* B, double* x, const double* b, const sb2_batch_params* prm,
                     int* iters, double* relres, int threads, cudaStream_t s) {
  BatchArgs a{B->nsys, B->d_sys_row, B->d_order, B->d_ptr, B->d_ind, B->d_val, B->d_val32,
              b, x, B->d_r64, B->d_w32, B->m, B->d_queue, prm->tol, prm->update_ratio,
              prm->max_iter, prm->mode, prm->init_guess_null, iters, relres};
  SB2_CUDA_TRY(cudaMemsetAsync(B->d_queue, 0, sizeof(unsigned), s));
  switch (threads) {
    case 128: return launch_batch<128>(a, s);
    case 512: return launch_batch<512>(a, s);
    default: return launch_batch<256>(a, s);
  }
}

__global__ void batch_to_float(long long n, const double* __restrict__ a, float* __restrict__ b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

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
  cudaError_t e = cudaMalloc(&B->d_sys_row, sizeof(int) * (nsys + 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_order, sizeof(int) * std::max(nsys, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_ptr, sizeof(int) * (m + 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_ind, sizeof(int) * std::max<long long>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_val, sizeof(double) * std::max<long long>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_val32, sizeof(float) * std::max<long long>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_r64, sizeof(double) * std::max(m, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_w32, sizeof(float) * 4 * (size_t)std::max(m, 1));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_queue, sizeof(unsigned) * 4);
  if (e == cudaSuccess) e = cudaMemcpy(B->d_sys_row, sys_row, sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nsys) e = cudaMemcpy(B->d_order, order.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B->d_ptr, ptr, sizeof(int) * (m + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz) e = cudaMemcpy(B->d_ind, local.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice);
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
  SB2_TRY(batch_run(B, x, b, prm, d_iters, d_relres, B->threads, s));
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

}  // extern "C"

extern "C" int sb2_batch_autotune(sb2_batch* B, double* x, const double* b,
                                  const sb2_batch_params* prm, void* stream) try {
  if (!B || !prm) return SB2_ERR_INVALID_VALUE;
  if (B->nsys == 0) return SB2_OK;
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  SB2_CUDA_TRY(cudaEventCreate(&e0));
  SB2_CUDA_TRY(cudaEventCreate(&e1));
  const int cand[3] = {128, 256, 512};
  float best = 1e30f;
  int best_t = B->threads;
  int st = SB2_OK;
  for (int c = 0; c < 3 && st == SB2_OK; c++) {
    // one untimed run, one timed run of the same solve
    st = sb2::batch_run(B, x, b, prm, nullptr, nullptr, cand[c], s);
    if (st != SB2_OK) break;
    cudaEventRecord(e0, s);
    st = sb2::batch_run(B, x, b, prm, nullptr, nullptr, cand[c], s);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) st = SB2_ERR_CUDA;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (st == SB2_OK && ms < best) {
      best = ms;
      best_t = cand[c];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st == SB2_OK) B->threads = best_t;
  return st;
} SB2_CATCH
