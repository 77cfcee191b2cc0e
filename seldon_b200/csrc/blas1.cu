// BLAS-1 on device vectors with deterministic reductions.
#include <cmath>

#include "sb2_internal.cuh"

namespace sb2 {

constexpr int kRedThreads = 256;

enum RedOp { kRedDot = 0, kRedNrm2 = 1 };

// Grid size is a function of n only, so the summation tree (and the result)
// is the same on every call.
static int red_blocks(long long n) {
  long long g = (n + 2047) / 2048;
  if (g < 1) g = 1;
  if (g > kRedMaxBlocks) g = kRedMaxBlocks;
  return (int)g;
}

// One pass: each thread sums a grid-strided subsequence in 4 independent
// chains, the CTA reduces in a fixed tree, and the last CTA to finish sums
// the per-CTA partials in index order and publishes the scalar.
template <int NT, int OP>
__global__ void __launch_bounds__(NT) reduce_kernel(
    int n, const double* __restrict__ x, const double* __restrict__ y,
    double* partials, unsigned* counter, double* out) {
  __shared__ double s_red[NT / 32];
  __shared__ bool s_last;
  const long long stride = (long long)gridDim.x * NT;
  long long i = (long long)blockIdx.x * NT + threadIdx.x;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  const double* y_ = (OP == kRedDot) ? y : x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    a0 = add_rn(a0, mul_rn(x[i], y_[i]));
    a1 = add_rn(a1, mul_rn(x[i + stride], y_[i + stride]));
    a2 = add_rn(a2, mul_rn(x[i + 2 * stride], y_[i + 2 * stride]));
    a3 = add_rn(a3, mul_rn(x[i + 3 * stride], y_[i + 3 * stride]));
  }
  for (; i < n; i += stride) a0 = add_rn(a0, mul_rn(x[i], y_[i]));
  double v = add_rn(add_rn(a0, a1), add_rn(a2, a3));
  v = block_sum<NT>(v, s_red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v;
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    double w = 0.0;
    const volatile double* vp = partials;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += NT) w = add_rn(w, vp[k]);
    w = block_sum<NT>(w, s_red);
    if (threadIdx.x == 0) {
      *out = (OP == kRedNrm2) ? sqrt(w) : w;
      *counter = 0u;
    }
  }
}

static int launch_reduce(int op, int n, const double* x, const double* y,
                         double* d_out, cudaStream_t s) {
  RedScratch* rs = nullptr;
  SB2_TRY(get_red_scratch(s, &rs));
  const int g = red_blocks(n);
  if (op == kRedDot)
    reduce_kernel<kRedThreads, kRedDot><<<g, kRedThreads, 0, s>>>(n, x, y, rs->partials, rs->counter, d_out);
  else
    reduce_kernel<kRedThreads, kRedNrm2><<<g, kRedThreads, 0, s>>>(n, x, y, rs->partials, rs->counter, d_out);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

static int reduce_to_host(int op, int n, const double* x, const double* y,
                          double* result, cudaStream_t s) {
  RedScratch* rs = nullptr;
  SB2_TRY(get_red_scratch(s, &rs));
  SB2_TRY(launch_reduce(op, n, x, y, rs->result, s));
  SB2_CUDA_TRY(cudaMemcpyAsync(result, rs->result, sizeof(double), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  return SB2_OK;
}

__global__ void axpy_kernel(int n, double alpha, const double* __restrict__ x,
                            double* __restrict__ y) {
  // Add: Y(i) += alpha * X(i) (Functions_Vector.cxx:103-104)
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = add_rn(y[i], mul_rn(alpha, x[i]));
}

__global__ void scal_kernel(int n, double alpha, double* __restrict__ x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = mul_rn(x[i], alpha);
}

__global__ void fill_kernel(int n, double v, double* __restrict__ x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = v;
}

static int elem_blocks(int n) {
  int g = (n + 255) / 256;
  const int cap = num_sms(current_device()) * 8;
  return g < 1 ? 1 : (g > cap ? cap : g);
}

}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_dot(int n, const double* x, const double* y, double* result, void* stream) try {
  if (n < 0 || !result || (n > 0 && (!x || !y))) return SB2_ERR_INVALID_VALUE;
  if (n == 0) { *result = 0.0; return SB2_OK; }
  return reduce_to_host(kRedDot, n, x, y, result, (cudaStream_t)stream);
} SB2_CATCH

int sb2_nrm2(int n, const double* x, double* result, void* stream) try {
  if (n < 0 || !result || (n > 0 && !x)) return SB2_ERR_INVALID_VALUE;
  if (n == 0) { *result = 0.0; return SB2_OK; }
  return reduce_to_host(kRedNrm2, n, x, nullptr, result, (cudaStream_t)stream);
} SB2_CATCH

int sb2_dot_device(int n, const double* x, const double* y, double* d_result, void* stream) try {
  if (n < 0 || !d_result || (n > 0 && (!x || !y))) return SB2_ERR_INVALID_VALUE;
  if (n == 0) {
    SB2_CUDA_TRY(cudaMemsetAsync(d_result, 0, sizeof(double), (cudaStream_t)stream));
    return SB2_OK;
  }
  return launch_reduce(kRedDot, n, x, y, d_result, (cudaStream_t)stream);
} SB2_CATCH

int sb2_nrm2_device(int n, const double* x, double* d_result, void* stream) try {
  if (n < 0 || !d_result || (n > 0 && !x)) return SB2_ERR_INVALID_VALUE;
  if (n == 0) {
    SB2_CUDA_TRY(cudaMemsetAsync(d_result, 0, sizeof(double), (cudaStream_t)stream));
    return SB2_OK;
  }
  return launch_reduce(kRedNrm2, n, x, nullptr, d_result, (cudaStream_t)stream);
} SB2_CATCH

int sb2_axpy(int n, double alpha, const double* x, double* y, void* stream) try {
  if (n < 0 || (n > 0 && (!x || !y))) return SB2_ERR_INVALID_VALUE;
  if (n == 0 || alpha == 0.0) return SB2_OK;  // Functions_Vector.cxx:94
  axpy_kernel<<<elem_blocks(n), 256, 0, (cudaStream_t)stream>>>(n, alpha, x, y);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
} SB2_CATCH

int sb2_scal(int n, double alpha, double* x, void* stream) try {
  if (n < 0 || (n > 0 && !x)) return SB2_ERR_INVALID_VALUE;
  if (n == 0) return SB2_OK;
  scal_kernel<<<elem_blocks(n), 256, 0, (cudaStream_t)stream>>>(n, alpha, x);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
} SB2_CATCH

int sb2_copy(int n, const double* x, double* y, void* stream) try {
  if (n < 0 || (n > 0 && (!x || !y))) return SB2_ERR_INVALID_VALUE;
  if (n == 0 || x == y) return SB2_OK;
  SB2_CUDA_TRY(cudaMemcpyAsync(y, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return SB2_OK;
} SB2_CATCH

int sb2_fill(int n, double value, double* x, void* stream) try {
  if (n < 0 || (n > 0 && !x)) return SB2_ERR_INVALID_VALUE;
  if (n == 0) return SB2_OK;
  fill_kernel<<<elem_blocks(n), 256, 0, (cudaStream_t)stream>>>(n, value, x);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
} SB2_CATCH

}  // extern "C"
