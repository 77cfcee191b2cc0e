// Mixed-precision iterative refinement: FP32 inner Krylov solves inside an
// FP64 outer loop.  This file holds the CG inner solve; the GMRES one
// (restarted GMRES whose restarts are the FP64 refinement steps) is in
// gmres_cgs2.cu.
//
//   x = x0 (or 0);  r = b - A x                       FP64 (SELL SpMV)
//   while ||r|| / ||b|| >= tol:
//     solve A32 d = float(r) to inner_tol             FP32 values, vectors
//                                                     and accumulation (CG)
//     x += double(d);  r = b - A x                    FP64
//
// The FP32 operator is a copy of the SELL values in single precision sharing
// the FP64 operator's column indices, so an inner product streams 8 bytes per
// nonzero instead of 12.  The residual kernel fuses the FP64 product, the
// residual norm and the down-conversion of r.  The inner solve is the chained
// CG of chain.cu instantiated for float.
#include <algorithm>
#include <cmath>
#include <vector>

#include "chain.cuh"
#include "spmv_core.cuh"

namespace sb2 {

template <typename VT>
long long chain_part_slots(const SellOp<VT>& S, int n);
template <typename VT>
int reducing_slice_grid(const SellOp<VT>& S);
template <typename T, typename VT>
int chain_cg(const SellOp<VT>& S, int n, const T* diag, T* x, const T* b, T* work,
             ChainState<T>* st, T* part, double* hist, int* hist_it, int hist_cap, double tol,
             int max_iter, int init_guess_null, cudaStream_t s, ChainState<T>* out);
SellOp<double> sell_op(const CsrArrays& a);
template <typename T, typename VT>
int chain_ru_start(const SellOp<VT>& S, int n, const T* diag, T* x, T* r, T* work,
                   ChainState<T>* st, T* part, double facteur, double tol, double delta,
                   int max_iter, cudaStream_t s);
template <typename T, typename VT>
int chain_ru_resume(const SellOp<VT>& S, int n, const T* diag, T* x, T* r, T* work,
                    ChainState<T>* st, T* part, cudaStream_t s);
template <typename T, typename VT>
int chain_ru_enqueue(const SellOp<VT>& S, int n, const T* diag, T* x, T* r, T* work,
                     ChainState<T>* st, T* part, int chunk, cudaStream_t s);

int ir_gmres_solve(const sb2_csr* A, bool jacobi, double* x, const double* b,
                   const sb2_ir_params* prm, sb2_ir_result* res, double* hist, int hist_cap,
                   cudaStream_t s);

constexpr int IT = 256;

__global__ void to_float_kernel(long long n, const double* __restrict__ a, float* __restrict__ b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// FP32 copies of the operator's values (SELL values and CSR values of the
// long-row bins) and of the diagonal, built once per matrix.
int ensure_fp32(const sb2_csr* cA, bool need_diag) {
  sb2_csr* A = const_cast<sb2_csr*>(cA);
  if (need_diag) SB2_TRY(ensure_diag(A));
  std::lock_guard<std::mutex> g(A->mu);
  SellArrays& S = A->full.sell;
  const int grid = num_sms(current_device()) * 8;
  if (!S.d_sval32 && S.padded > 0) {
    SB2_CUDA_TRY(cudaMalloc(&S.d_sval32, sizeof(float) * S.padded));
    to_float_kernel<<<grid, IT>>>(S.padded, S.d_sval, S.d_sval32);
  }
  if (!A->d_val32) {
    const long long cap = padded_nnz(A->full.nnz);
    SB2_CUDA_TRY(cudaMalloc(&A->d_val32, sizeof(float) * cap));
    to_float_kernel<<<grid, IT>>>(cap, A->full.d_val, A->d_val32);
  }
  if (need_diag && !A->d_diag32) {
    SB2_CUDA_TRY(cudaMalloc(&A->d_diag32, sizeof(float) * std::max(A->m, 1)));
    to_float_kernel<<<grid, IT>>>(A->m, A->d_diag, A->d_diag32);
  }
  SB2_CUDA_TRY(cudaDeviceSynchronize());
  return SB2_OK;
}

SellOp<float> sell_op32(const sb2_csr* A) {
  const SellArrays& s = A->full.sell;
  return SellOp<float>{s.nslice, s.d_sptr, s.d_qinfo, s.d_qrows, s.d_scol, s.d_sval32, s.nwarp, s.d_wrows,
                       s.ncta, s.d_crows, A->full.d_ptr, A->full.d_ind, A->d_val32};
}

// r = b - A x in FP64, r32 = float(r), deposits of ||r||^2.
struct EpiIrResidual {
  const double* b;
  double* r;
  float* r32;
  double acc;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double v = add_rn(__ldg(b + i), -t);
    r[i] = v;
    r32[i] = (float)v;
    acc = add_rn(acc, mul_rn(v, v));
  }
};

template <int PART>
__global__ void __launch_bounds__(IT, PART == 0 ? 4 : 1)
    k_ir_residual(SellOp<double> S, const double* __restrict__ x, const double* __restrict__ b,
                  double* __restrict__ r, float* __restrict__ r32, double* part, unsigned* cnt,
                  double* out, int slot0, int tot) {
  __shared__ double s_red[IT / 32];
  __shared__ double s_out[1];
  EpiIrResidual epi{b, r, r32, 0.0};
  XLoadLdg<double> xl{x};
  if (PART == 0)
    sell_spmv_slices<IT, double, double>(S, xl, epi, blockIdx.x, gridDim.x);
  else
    sell_spmv_long<IT, double, double>(S, xl, epi, s_red, blockIdx.x, gridDim.x);
  double v[1] = {block_sum<IT>(epi.acc, s_red)};
  if (deposit_and_finish<IT, 1>(v, part, cnt, slot0 + blockIdx.x, tot, s_red, s_out) &&
      threadIdx.x == 0)
    *out = s_out[0];
}

// null initial guess: x = 0, r = b, r32 = float(b), deposits of ||b||^2
__global__ void __launch_bounds__(IT, 8) k_ir_init_null(int n, const double* __restrict__ b,
                                                        double* __restrict__ x,
                                                        double* __restrict__ r,
                                                        float* __restrict__ r32, double* part,
                                                        unsigned* cnt, double* out) {
  __shared__ double s_red[IT / 32];
  __shared__ double s_out[1];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * IT + threadIdx.x; i < n; i += (long long)gridDim.x * IT) {
    const double bi = __ldg(b + i);
    x[i] = 0.0;
    r[i] = bi;
    r32[i] = (float)bi;
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  double v[1] = {block_sum<IT>(acc, s_red)};
  if (deposit_and_finish<IT, 1>(v, part, cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0)
    *out = s_out[0];
}

// x += double(d); with `zero`, d = 0 afterwards (next correction starts empty)
__global__ void __launch_bounds__(IT, 8) k_ir_update(int n, double* __restrict__ x,
                                                     float* __restrict__ d, bool zero) {
  for (long long i = (long long)blockIdx.x * IT + threadIdx.x; i < n; i += (long long)gridDim.x * IT) {
    x[i] = add_rn(x[i], (double)d[i]);
    if (zero) d[i] = 0.0f;
  }
}

// ||b||^2
__global__ void __launch_bounds__(IT, 8) k_ir_normb(int n, const double* __restrict__ b,
                                                    double* part, unsigned* cnt, double* out) {
  __shared__ double s_red[IT / 32];
  __shared__ double s_out[1];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * IT + threadIdx.x; i < n; i += (long long)gridDim.x * IT) {
    const double bi = __ldg(b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  double v[1] = {block_sum<IT>(acc, s_red)};
  if (deposit_and_finish<IT, 1>(v, part, cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0)
    *out = s_out[0];
}

// The deposit array holds `slots` values (chain_part_slots); this product
// uses the same grid as the chained products, so its deposits fit.
static int ir_residual(const SellOp<double>& S, int n, const double* x, const double* b,
                       double* r, float* r32, double* part, unsigned* cnt, double* out,
                       long long slots, cudaStream_t s) {
  const int g1 = reducing_slice_grid(S);
  const int g2 = (S.nwarp_rows + S.ncta_rows) > 0 ? std::max((S.nwarp_rows + 7) / 8, S.ncta_rows) : 0;
  const int tot = g1 + g2;
  if (tot > slots) return SB2_ERR_INVALID_VALUE;
  if (g1) k_ir_residual<0><<<g1, IT, 0, s>>>(S, x, b, r, r32, part, cnt, out, 0, tot);
  if (g2) k_ir_residual<1><<<g2, IT, 0, s>>>(S, x, b, r, r32, part, cnt, out, g1, tot);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

static int ir_solve(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
                    const sb2_ir_params* prm, sb2_ir_result* res, double* hist, int hist_cap,
                    cudaStream_t s) {
  if (!A || !prm || !res || A->m != A->n) return SB2_ERR_INVALID_VALUE;
  if (A->m > 0 && (!x || !b || x == b)) return SB2_ERR_INVALID_VALUE;
  if (prm->solver != 0 && prm->solver != 1) return SB2_ERR_NOT_SUPPORTED;
  *res = sb2_ir_result{};
  const int n = A->m;
  if (n == 0) return SB2_OK;
  if (A->full.sell.nslice < 0) return SB2_ERR_NOT_SUPPORTED;
  int kind = M ? precond_kind(M) : SB2_PRECOND_IDENTITY;
  if (kind == SB2_PRECOND_SOR || kind == SB2_PRECOND_ILUT) return SB2_ERR_NOT_SUPPORTED;
  if (M && precond_matrix(M) != A) return SB2_ERR_INVALID_VALUE;
  const bool jac = (kind == SB2_PRECOND_JACOBI);
  if (prm->solver == 1) return ir_gmres_solve(A, jac, x, b, prm, res, hist, hist_cap, s);
  SB2_TRY(ensure_fp32(A, jac));
  const SellOp<double> S64 = sell_op(A->full);
  const SellOp<float> S32 = sell_op32(A);

  // workspace: r (FP64), r32, d, inner work (3 FP32 vectors), states, deposits
  // elementwise reductions of this solver: one deposit per CTA of `ge`
  const int ge = std::max(1, std::min((n + IT * 4 - 1) / (IT * 4), num_sms(current_device()) * 8));
  const long long slots =
      std::max<long long>(std::max(chain_part_slots(S32, n), chain_part_slots(S64, n)), ge + 16);
  const int hcap = std::max(prm->max_inner, 0) + 2;
  const size_t nn = (size_t)n;
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
  const size_t o_r = take(8 * nn), o_r32 = take(4 * nn), o_d = take(4 * nn), o_w = take(12 * nn);
  const size_t o_st = take(sizeof(ChainState<float>)), o_part = take(8 * (size_t)slots);
  const size_t o_cnt = take(16), o_out = take(16), o_h = take(8 * (size_t)hcap), o_hi = take(4 * (size_t)hcap);
  struct Buf {
    void* p = nullptr;
    cudaStream_t s;
    ~Buf() { if (p) cudaFreeAsync(p, s); }
  } buf;
  buf.s = s;
  SB2_CUDA_TRY(pool_malloc((void**)&buf.p, off, s));
  char* base = (char*)buf.p;
  double* r = (double*)(base + o_r);
  float* r32 = (float*)(base + o_r32);
  float* d = (float*)(base + o_d);
  float* w = (float*)(base + o_w);
  ChainState<float>* st = (ChainState<float>*)(base + o_st);
  void* part = base + o_part;
  unsigned* cnt = (unsigned*)(base + o_cnt);
  double* dout = (double*)(base + o_out);
  double* dh = (double*)(base + o_h);
  int* dhi = (int*)(base + o_hi);
  SB2_CUDA_TRY(cudaMemsetAsync(cnt, 0, 16, s));

  double h_out = 0.0;
  k_ir_normb<<<ge, IT, 0, s>>>(n, b, (double*)part, cnt, dout);
  SB2_CUDA_TRY(cudaMemcpyAsync(&h_out, dout, sizeof(double), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  const double nb = std::sqrt(h_out);
  if (nb == 0.0) {
    res->init_failed = 1;
    return SB2_OK;
  }
  if (prm->init_guess_null)
    k_ir_init_null<<<ge, IT, 0, s>>>(n, b, x, r, r32, (double*)part, cnt, dout);
  else
    SB2_TRY(ir_residual(S64, n, x, b, r, r32, (double*)part, cnt, dout, slots, s));
  SB2_CUDA_TRY(cudaGetLastError());
  int nh = 0, inner_total = 0, outer = 0;
  double rel = 0.0;
  if (prm->mode == 0) {
    // Reliable updates: one FP32 CG run whose residual is replaced by the FP64
    // true residual after every correction; the search direction carries on.
    SB2_CUDA_TRY(cudaMemcpyAsync(&h_out, dout, sizeof(double), cudaMemcpyDeviceToHost, s));
    SB2_CUDA_TRY(cudaStreamSynchronize(s));
    rel = std::sqrt(h_out) / nb;
    if (hist && nh < hist_cap) hist[nh] = rel;
    nh++;
    const float* dg = jac ? A->d_diag32 : nullptr;
    if (!(rel < prm->tol)) {
      SB2_TRY((chain_ru_start<float, float>(S32, n, dg, d, r32, w, st, (float*)part, 1.0 / nb,
                                            prm->tol, prm->inner_tol, prm->max_inner, s)));
      // chunks of 8, 16, then 32 iterations, one queued behind the one whose
      // state the host waits for; a pending correction turns the queued
      // chunk into no-ops
      ChainPipe<float> pipe;
      SB2_TRY(pipe.init());
      ChunkPlanner plan;
      int chunk = 8, launched = 0;
      auto enqueue = [&]() -> int {
        SB2_TRY((chain_ru_enqueue<float, float>(S32, n, dg, d, r32, w, st, (float*)part, chunk, s)));
        launched += chunk;
        return pipe.mark(st, launched, s);
      };
      auto prime = [&]() -> int {
        plan.reset();
        chunk = 8;
        SB2_TRY(enqueue());
        chunk = 16;
        return enqueue();
      };
      SB2_TRY(prime());
      for (;;) {
        ChainState<float> o;
        int at = 0;
        SB2_TRY(pipe.wait(&o, &at));
        inner_total = o.nb_iter;
        // every stop of the FP32 iteration sets `pending`, except breakdown
        // #2 inside the product, which sets `done` (and `fail`)
        if (!o.pending && !o.done && launched <= prm->max_inner + 64) {
          // the next correction comes when ||r|| has dropped by delta
          const double target = std::max(prm->tol, o.delta * o.rmax * o.facteur);
          chunk = plan.next(o.nb_iter, o.reste, target, launched - at, std::min(chunk * 2, 32), 4);
          SB2_TRY(enqueue());
          continue;
        }
        if (o.done) o.fail = o.fail ? o.fail : 2;
        // FP64 correction: x += d, d = 0, r = b - A x, r32 = float(r)
        k_ir_update<<<ge, IT, 0, s>>>(n, x, d, true);
        SB2_TRY(ir_residual(S64, n, x, b, r, r32, (double*)part, cnt, dout, slots, s));
        SB2_CUDA_TRY(cudaMemcpyAsync(&h_out, dout, sizeof(double), cudaMemcpyDeviceToHost, s));
        SB2_CUDA_TRY(cudaStreamSynchronize(s));
        pipe.reset();  // the stream has drained: no chunk is outstanding
        rel = std::sqrt(h_out) / nb;
        if (hist && nh < hist_cap) hist[nh] = rel;
        nh++;
        outer++;
        if (rel < prm->tol || o.fail || o.nb_iter >= prm->max_inner || outer >= prm->max_outer ||
            !(rel == rel))
          break;
        SB2_TRY((chain_ru_resume<float, float>(S32, n, dg, d, r32, w, st, (float*)part, s)));
        SB2_TRY(prime());
      }
      SB2_CUDA_TRY(cudaStreamSynchronize(s));
    }
    res->outer_iter = outer;
    res->inner_iter = inner_total;
    res->rel_residual = rel;
    res->hist_len = std::min(nh, std::max(hist_cap, 0));
    res->error_code = (rel < prm->tol) ? 0 : -2;
    return SB2_OK;
  }
  for (;;) {
    SB2_CUDA_TRY(cudaMemcpyAsync(&h_out, dout, sizeof(double), cudaMemcpyDeviceToHost, s));
    SB2_CUDA_TRY(cudaStreamSynchronize(s));
    rel = std::sqrt(h_out) / nb;
    if (hist && nh < hist_cap) hist[nh] = rel;
    nh++;
    if (rel < prm->tol || outer >= prm->max_outer || !(rel == rel)) break;
    // inner FP32 solve of A d = r32, d starting at zero
    ChainState<float> o;
    SB2_TRY((chain_cg<float, float>(S32, n, jac ? A->d_diag32 : nullptr, d, r32, w, st,
                                    (float*)part, dh, dhi, hcap, prm->inner_tol, prm->max_inner,
                                    1, s, &o)));
    inner_total += o.init_failed ? 0 : o.nb_iter;
    outer++;
    if (o.init_failed) break;
    k_ir_update<<<ge, IT, 0, s>>>(n, x, d, false);
    SB2_TRY(ir_residual(S64, n, x, b, r, r32, (double*)part, cnt, dout, slots, s));
  }
  res->outer_iter = outer;
  res->inner_iter = inner_total;
  res->rel_residual = rel;
  res->hist_len = std::min(nh, std::max(hist_cap, 0));
  res->error_code = (rel < prm->tol) ? 0 : -2;
  return SB2_OK;
}

}  // namespace sb2

extern "C" int sb2_ir_solve(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
                            const sb2_ir_params* params, sb2_ir_result* result, double* hist,
                            int hist_cap, void* stream) try {
  SB2_TRACE("sb2_ir_solve");
  return sb2::ir_solve(A, M, x, b, params, result, hist, hist_cap, (cudaStream_t)stream);
} SB2_CATCH
