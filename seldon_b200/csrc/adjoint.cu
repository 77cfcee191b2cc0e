// Pieces of the hand-written adjoint of x = A^{-1} b (no counterpart in the
// reference): new values on a fixed pattern, and the gradients
//   dL/dA_ij = -lambda_i x_j  on the stored pattern        (A^T lambda = dL/dx)
//   dL/dtheta_e = -(lambda_i - lambda_j)(x_i - x_j)       (graph Laplacian edge e = (i, j))
// The adjoint solve itself is the library's own CG / BiCGSTAB on A (or A^T).
#include "sb2_internal.cuh"

namespace sb2 {

__global__ void set_values_kernel(long long nnz, const double* __restrict__ val,
                                  double* __restrict__ csr_val, const long long* __restrict__ pos,
                                  double* __restrict__ sval) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
       k += (long long)gridDim.x * blockDim.x) {
    const double v = val[k];
    csr_val[k] = v;
    if (pos) {
      const long long e = pos[k];
      if (e >= 0) sval[e] = v;
    }
  }
}

__global__ void grad_pattern_kernel(int m, const int* __restrict__ ptr, const int* __restrict__ ind,
                                    double alpha, const double* __restrict__ lambda,
                                    const double* __restrict__ x, double* __restrict__ g) {
  // one warp per row, entries in order
  const int lane = threadIdx.x & 31;
  for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m;
       i += ((long long)gridDim.x * blockDim.x) >> 5) {
    const double li = mul_rn(alpha, __ldg(lambda + i));
    for (int k = __ldg(ptr + i) + lane; k < __ldg(ptr + i + 1); k += 32)
      g[k] = mul_rn(li, __ldg(x + __ldg(ind + k)));
  }
}

__global__ void grad_edges_kernel(int ne, const int* __restrict__ ei, const int* __restrict__ ej,
                                  const double* __restrict__ lambda, const double* __restrict__ x,
                                  double* __restrict__ g) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = __ldg(ei + e), j = __ldg(ej + e);
    const double dl = __dsub_rn(__ldg(lambda + i), __ldg(lambda + j));
    const double dx = __dsub_rn(__ldg(x + i), __ldg(x + j));
    g[e] = -mul_rn(dl, dx);
  }
}

}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_csr_set_values(sb2_csr* A, const double* val, int on_device, void* stream) try {
  if (!A || (A->nnz_stored > 0 && !val)) return SB2_ERR_INVALID_VALUE;
  if (A->sym) return SB2_ERR_NOT_SUPPORTED;  // the expanded copy keeps no map to the stored half
  cudaStream_t s = (cudaStream_t)stream;
  const long long nnz = A->full.nnz;
  if (nnz == 0) return SB2_OK;
  std::lock_guard<std::mutex> g(A->mu);
  const double* src = val;
  double* tmp = nullptr;
  if (!on_device) {
    SB2_CUDA_TRY(pool_malloc((void**)&tmp, sizeof(double) * nnz, s));
    SB2_CUDA_TRY(cudaMemcpyAsync(tmp, val, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    src = tmp;
  }
  const SellArrays& S = A->full.sell;
  const int grid = num_sms(current_device()) * 8;
  set_values_kernel<<<grid, 256, 0, s>>>(nnz, src, A->full.d_val, S.nslice >= 0 ? S.d_pos : nullptr,
                                         S.d_sval);
  cudaError_t e = cudaGetLastError();
  if (tmp) cudaFreeAsync(tmp, s);
  if (e != cudaSuccess) return map_cuda_error(e);
  // derived copies are rebuilt on their next use
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  cudaFree(A->d_diag);
  A->d_diag = nullptr;
  cudaFree(A->d_diag32);
  A->d_diag32 = nullptr;
  cudaFree(A->d_val32);
  A->d_val32 = nullptr;
  cudaFree(A->full.sell.d_sval32);
  A->full.sell.d_sval32 = nullptr;
  free_csr(&A->trans);
  return SB2_OK;
} SB2_CATCH

int sb2_grad_pattern(const sb2_csr* A, double alpha, const double* lambda, const double* x,
                     double* grad_val, void* stream) try {
  SB2_TRACE("sb2_grad_pattern");
  if (!A || (A->nnz > 0 && (!lambda || !x || !grad_val))) return SB2_ERR_INVALID_VALUE;
  if (A->sym) return SB2_ERR_NOT_SUPPORTED;
  if (A->m == 0) return SB2_OK;
  const int grid = num_sms(current_device()) * 8;
  grad_pattern_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(A->m, A->full.d_ptr, A->full.d_ind,
                                                              alpha, lambda, x, grad_val);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
} SB2_CATCH

int sb2_grad_edges(int nedges, const int* ei, const int* ej, const double* lambda,
                   const double* x, double* grad, void* stream) try {
  SB2_TRACE("sb2_grad_edges");
  if (nedges < 0 || (nedges > 0 && (!ei || !ej || !lambda || !x || !grad)))
    return SB2_ERR_INVALID_VALUE;
  if (nedges == 0) return SB2_OK;
  const int grid = num_sms(current_device()) * 8;
  grad_edges_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(nedges, ei, ej, lambda, x, grad);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
} SB2_CATCH

}  // extern "C"
