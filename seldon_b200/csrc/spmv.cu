// Standalone SpMV: MltAdd / Mlt on device and host vectors.
#include <algorithm>

#include "sell.cuh"
#include "spmv_core.cuh"
#include "spmv_tma.cuh"

namespace sb2 {

// y = beta*y + alpha*t (MltAdd: Mlt(beta, Y) then Y(i) += alpha*temp,
// Functions_MatVect.cxx:414, :428) or y = alpha*t (Mlt: Y.Fill(0) first,
// Functions_MatVect.cxx:72-81).
struct EpiAxpby {
  double alpha, beta;
  double* __restrict__ y;
  bool overwrite;
  __device__ __forceinline__ void operator()(int r, double t) const {
    double v = mul_rn(alpha, t);
    if (!overwrite) v = add_rn(mul_rn(beta, y[r]), v);
    y[r] = v;
  }
};

template <int NT>
__global__ void __launch_bounds__(NT) spmv_kernel(
    const int* __restrict__ ptr, const int* __restrict__ ind,
    const double* __restrict__ val, const int* __restrict__ blk,
    const unsigned char* __restrict__ kind, double alpha,
    const double* __restrict__ x, double beta, double* __restrict__ y,
    bool overwrite) {
  __shared__ double s_prod[kNnzCap];
  __shared__ double s_red[NT / 32];
  const int b = blockIdx.x;
  EpiAxpby epi{alpha, beta, y, overwrite};
  XLoadLdg<double> xl{x};
  spmv_row_block<NT, double, double>(ptr, ind, val, blk[b], blk[b + 1], kind[b],
                                     xl, epi, s_prod, s_red);
}

// One product through the TMA-pipelined engine: each CTA streams its
// contiguous share of row blocks once.
template <int NT, int S>
__global__ void __launch_bounds__(NT, 2) spmv_tma_kernel(
    TmaOp<double> op, double alpha, const double* __restrict__ x, double beta,
    double* __restrict__ y, bool overwrite, int* status, unsigned long long limit_ns) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double s_red[NT / 32];
  TmaRing<S, double, double> R;
  R.carve(smem);
  R.init(op);
  EpiAxpby epi{alpha, beta, y, overwrite};
  XLoadLdg<double> xl{x};
  if (!tma_spmv_pass<NT, S>(R, op, xl, epi, s_red, (unsigned)R.nb, limit_ns, status))
    R.drain(limit_ns);
}

// Product algorithm (set by the autotuner): binned SELL-32 by default, the
// row-block stream kernel or the TMA-pipelined kernel; and the TMA launch
// configuration (threads per CTA, ring stages).
static std::atomic<int> g_spmv_algo{SB2_SPMV_SELL}, g_spmv_threads{256}, g_spmv_stages{4};

// y = beta*y + alpha*t, or y = alpha*t when OVERWRITE (Mlt)
template <bool OVERWRITE>
struct EpiAxpbyT {
  double alpha, beta;
  double* __restrict__ y;
  __device__ __forceinline__ void operator()(int r, double t) const {
    double v = mul_rn(alpha, t);
    if (!OVERWRITE) v = add_rn(mul_rn(beta, y[r]), v);
    y[r] = v;
  }
  // rows r..r+3 (r % 4 == 0): the same arithmetic with 16-byte accesses
  __device__ __forceinline__ void quad(int r, const double* t) const {
    if (!is_aligned16(y + r)) {
      for (int j = 0; j < 4; j++) (*this)(r + j, t[j]);
      return;
    }
    double v[4], yo[4];
    if (!OVERWRITE) vld4_cg(y + r, yo);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      v[j] = mul_rn(alpha, t[j]);
      if (!OVERWRITE) v[j] = add_rn(mul_rn(beta, yo[j]), v[j]);
    }
    vst4(y + r, v);
  }
};

// Thread bin: one warp per slice of 128 rows, 4 CTAs of 256 threads per SM
// (64 registers: a lane keeps four rows' loads in flight).
template <int NT, bool OVERWRITE>
__global__ void __launch_bounds__(NT, 4) sell_slices_kernel(SellOp<double> S, double alpha,
                                                            const double* __restrict__ x,
                                                            double beta, double* __restrict__ y) {
  EpiAxpbyT<OVERWRITE> epi{alpha, beta, y};
  XLoadLdg<double> xl{x};
  sell_spmv_slices<NT, double, double>(S, xl, epi, blockIdx.x, gridDim.x);
}

// Warp and CTA bins (rows longer than 32), launched only when present.
template <int NT, bool OVERWRITE>
__global__ void __launch_bounds__(NT) sell_long_kernel(SellOp<double> S, double alpha,
                                                       const double* __restrict__ x, double beta,
                                                       double* __restrict__ y) {
  __shared__ double s_red[NT / 32];
  EpiAxpbyT<OVERWRITE> epi{alpha, beta, y};
  XLoadLdg<double> xl{x};
  sell_spmv_long<NT, double, double>(S, xl, epi, s_red, blockIdx.x, gridDim.x);
}

// Measurement kernel: sum_k val[k] * x[ind[k]] over one array of entries,
// with no rows (val == nullptr: sum_k x[ind[k]]).  It streams the index and
// value arrays and gathers x exactly as a CSR product over the same arrays
// does, without the per-row sums: its time bounds from below what any row
// binning of that product can reach.  Each CTA writes one partial sum.
__global__ void __launch_bounds__(256) probe_gather_kernel(long long nnz, const int* __restrict__ ind,
                                                          const double* __restrict__ val,
                                                          const double* __restrict__ x,
                                                          double* __restrict__ partials) {
  __shared__ double s_red[8];
  double acc0 = 0.0, acc1 = 0.0;
  const long long q4 = nnz / 4;  // groups of 4 entries (16-byte index loads)
  for (long long g = (long long)blockIdx.x * 256 + threadIdx.x; g < q4; g += (long long)gridDim.x * 256) {
    const int4 c = __ldcs(reinterpret_cast<const int4*>(ind) + g);
    const double x0 = __ldg(x + c.x), x1 = __ldg(x + c.y), x2 = __ldg(x + c.z), x3 = __ldg(x + c.w);
    if (val) {
      double v[4];
      ld_stream_val4(val + 4 * g, v);
      acc0 = add_rn(acc0, add_rn(mul_rn(v[0], x0), mul_rn(v[1], x1)));
      acc1 = add_rn(acc1, add_rn(mul_rn(v[2], x2), mul_rn(v[3], x3)));
    } else {
      acc0 = add_rn(acc0, add_rn(x0, x1));
      acc1 = add_rn(acc1, add_rn(x2, x3));
    }
  }
  for (long long k = 4 * q4 + (long long)blockIdx.x * 256 + threadIdx.x; k < nnz;
       k += (long long)gridDim.x * 256)
    acc0 = add_rn(acc0, val ? mul_rn(__ldg(val + k), __ldg(x + __ldg(ind + k))) : __ldg(x + __ldg(ind + k)));
  const double t = block_sum<256>(add_rn(acc0, acc1), s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

SellOp<double> sell_op(const CsrArrays& a) {
  const SellArrays& s = a.sell;
  return SellOp<double>{s.nslice, s.d_sptr, s.d_qinfo, s.d_qrows, s.d_scol, s.d_sval, s.nwarp,
                        s.d_wrows, s.ncta, s.d_crows, a.d_ptr, a.d_ind, a.d_val};
}

template <int NT, int S>
static int launch_tma(const CsrArrays& a, double alpha, const double* x, double beta, double* y,
                      bool overwrite, cudaStream_t s, int* status) {
  // the shared-memory opt-in is a per-device setting: taken, with the
  // occupancy it gives, on each device's first launch
  static std::mutex mu;
  static std::map<int, int> per_sm_of;
  const size_t smem = TmaRing<S, double, double>::smem_bytes();
  const int dev = current_device();
  int per_sm;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = per_sm_of.find(dev);
    if (it == per_sm_of.end()) {
      SB2_CUDA_TRY(cudaFuncSetAttribute(spmv_tma_kernel<NT, S>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int v = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, spmv_tma_kernel<NT, S>, NT, smem) !=
          cudaSuccess)
        v = 1;
      it = per_sm_of.emplace(dev, v < 1 ? 1 : v).first;
    }
    per_sm = it->second;
  }
  const int g = std::min(a.tma.nblk, per_sm * num_sms(dev));
  TmaOp<double> op{a.d_ptr, a.d_ind, a.d_val, a.tma.d_desc, a.tma.nblk, a.rows};
  spmv_tma_kernel<NT, S><<<g, NT, smem, s>>>(op, alpha, x, beta, y, overwrite, status,
                                             ring_wait_ns());
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

int launch_spmv(const CsrArrays& a, double alpha, const double* x, double beta,
                double* y, bool overwrite, cudaStream_t s) {
  if (a.rows == 0) return SB2_OK;
  if (g_spmv_algo == SB2_SPMV_SELL && a.sell.nslice >= 0) {
    const SellOp<double> op = sell_op(a);
    if (a.sell.nslice > 0) {
      const unsigned g = (unsigned)std::min<long long>(((long long)a.sell.nslice + 7) / 8, 1 << 30);
      if (overwrite)
        sell_slices_kernel<256, true><<<g, 256, 0, s>>>(op, alpha, x, beta, y);
      else
        sell_slices_kernel<256, false><<<g, 256, 0, s>>>(op, alpha, x, beta, y);
    }
    if (a.sell.nwarp + a.sell.ncta > 0) {
      const unsigned g = (unsigned)std::max<long long>(((long long)a.sell.nwarp + 7) / 8, a.sell.ncta);
      if (overwrite)
        sell_long_kernel<256, true><<<g, 256, 0, s>>>(op, alpha, x, beta, y);
      else
        sell_long_kernel<256, false><<<g, 256, 0, s>>>(op, alpha, x, beta, y);
    }
    SB2_CUDA_TRY(cudaGetLastError());
    return SB2_OK;
  }
  if (g_spmv_algo == SB2_SPMV_TMA && a.tma.nblk > 0) {
    RedScratch* rs = nullptr;
    SB2_TRY(get_red_scratch(s, &rs));
    if (g_spmv_threads == 512)
      return g_spmv_stages == 3 ? launch_tma<512, 3>(a, alpha, x, beta, y, overwrite, s, rs->status)
                                : launch_tma<512, 4>(a, alpha, x, beta, y, overwrite, s, rs->status);
    return g_spmv_stages == 3 ? launch_tma<256, 3>(a, alpha, x, beta, y, overwrite, s, rs->status)
                              : launch_tma<256, 4>(a, alpha, x, beta, y, overwrite, s, rs->status);
  }
  spmv_kernel<kSpmvThreads><<<a.part.nblk, kSpmvThreads, 0, s>>>(
      a.d_ptr, a.d_ind, a.d_val, a.part.d_blk, a.part.d_kind, alpha, x, beta,
      y, overwrite);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

static bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const char* pa = static_cast<const char*>(a);
  const char* pb = static_cast<const char*>(b);
  return pa < pb + nb && pb < pa + na;
}

static int spmv_common(const sb2_csr* A, int trans, double alpha,
                       const double* x, double beta, double* y, bool overwrite,
                       cudaStream_t s) {
  if (!A || (!x && (trans ? A->m : A->n) > 0) || (!y && (trans ? A->n : A->m) > 0))
    return SB2_ERR_INVALID_VALUE;
  const int nx = trans ? A->m : A->n, ny = trans ? A->n : A->m;
  if (nx > 0 && ny > 0 && overlaps(x, sizeof(double) * nx, y, sizeof(double) * ny))
    return SB2_ERR_INVALID_VALUE;
  // A symmetric operator is its own transpose (Functions_MatVect.cxx:915-927).
  if (trans && !A->sym) {
    SB2_TRY(ensure_transpose(A));
    return launch_spmv(A->trans, alpha, x, beta, y, overwrite, s);
  }
  return launch_spmv(A->full, alpha, x, beta, y, overwrite, s);
}

}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_spmv(const sb2_csr* A, int trans, double alpha, const double* x,
             double beta, double* y, void* stream) try {
  SB2_TRACE("sb2_spmv");
  return spmv_common(A, trans, alpha, x, beta, y, false, (cudaStream_t)stream);
} SB2_CATCH

int sb2_mlt(const sb2_csr* A, int trans, double alpha, const double* x,
            double* y, void* stream) try {
  SB2_TRACE("sb2_mlt");
  return spmv_common(A, trans, alpha, x, 0.0, y, true, (cudaStream_t)stream);
} SB2_CATCH

static int spmv_host_common(const sb2_csr* cA, int trans, double alpha,
                            const double* x_host, double beta, double* y_host,
                            bool overwrite, cudaStream_t s) {
  if (!cA) return SB2_ERR_INVALID_VALUE;
  sb2_csr* A = const_cast<sb2_csr*>(cA);
  const int nx = trans ? A->m : A->n, ny = trans ? A->n : A->m;
  if ((nx > 0 && !x_host) || (ny > 0 && !y_host)) return SB2_ERR_INVALID_VALUE;
  std::lock_guard<std::mutex> g(A->host_mu);
  // staging vectors sized for both orientations, allocated on first use
  if (!A->d_hx) {
    const size_t len = (size_t)std::max(std::max(A->m, A->n), 1);
    SB2_CUDA_TRY(cudaMalloc(&A->d_hx, sizeof(double) * len));
    SB2_CUDA_TRY(cudaMalloc(&A->d_hy, sizeof(double) * len));
  }
  double *dx = A->d_hx, *dy = A->d_hy;
  if (nx > 0)
    SB2_CUDA_TRY(cudaMemcpyAsync(dx, x_host, sizeof(double) * nx, cudaMemcpyHostToDevice, s));
  if (ny > 0 && !overwrite)
    SB2_CUDA_TRY(cudaMemcpyAsync(dy, y_host, sizeof(double) * ny, cudaMemcpyHostToDevice, s));
  SB2_TRY(spmv_common(A, trans, alpha, dx, beta, dy, overwrite, s));
  if (ny > 0)
    SB2_CUDA_TRY(cudaMemcpyAsync(y_host, dy, sizeof(double) * ny, cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  return SB2_OK;
}

int sb2_spmv_host(const sb2_csr* A, int trans, double alpha,
                  const double* x_host, double beta, double* y_host,
                  void* stream) try {
  SB2_TRACE("sb2_spmv_host");
  // y is copied in too: MltAdd scales it by beta even when beta == 0.
  return spmv_host_common(A, trans, alpha, x_host, beta, y_host, false,
                          (cudaStream_t)stream);
} SB2_CATCH

int sb2_spmv_set_config(int algo, int threads, int stages) try {
  if (algo < SB2_SPMV_SELL || algo > SB2_SPMV_TMA) return SB2_ERR_INVALID_VALUE;
  if ((threads != 256 && threads != 512) || (stages != 3 && stages != 4))
    return SB2_ERR_INVALID_VALUE;
  g_spmv_algo = algo;
  g_spmv_threads = threads;
  g_spmv_stages = stages;
  return SB2_OK;
} SB2_CATCH

int sb2_mlt_host(const sb2_csr* A, int trans, double alpha,
                 const double* x_host, double* y_host, void* stream) try {
  SB2_TRACE("sb2_mlt_host");
  return spmv_host_common(A, trans, alpha, x_host, 0.0, y_host, true,
                          (cudaStream_t)stream);
} SB2_CATCH

// y_i = alpha*op(A)*x_i for a batch of host vectors.  Two device buffers per
// side and two copy streams: the copy of x_{i+1} in, the product i and the
// copy of y_{i-1} out run at the same time (host-to-device and
// device-to-host transfers use separate copy engines).  Events order the
// reuse of each buffer: x into buffer b waits for the product that last read
// it, the product into y buffer b waits for the copy out that last read it.
int sb2_mlt_host_batch(const sb2_csr* cA, int trans, double alpha, int count,
                       const double* x_host, double* y_host, void* stream) try {
  SB2_TRACE("sb2_mlt_host_batch");
  if (!cA || count < 0) return SB2_ERR_INVALID_VALUE;
  sb2_csr* A = const_cast<sb2_csr*>(cA);
  const int nx = trans ? A->m : A->n, ny = trans ? A->n : A->m;
  if (count == 0) return SB2_OK;
  if ((nx > 0 && !x_host) || (ny > 0 && !y_host)) return SB2_ERR_INVALID_VALUE;
  cudaStream_t s = (cudaStream_t)stream;
  std::lock_guard<std::mutex> g(A->host_mu);
  const size_t len = (size_t)std::max(std::max(A->m, A->n), 1);
  if (!A->s_in) {
    // Everything is created into locals and published only when all of it
    // exists; a failure part-way releases what was made, so a later call
    // starts the set-up afresh without leaking.
    struct Pipe {
      double *bx[2] = {nullptr, nullptr}, *by[2] = {nullptr, nullptr};
      cudaEvent_t ein[2] = {nullptr, nullptr}, ekern[2] = {nullptr, nullptr},
                  eout[2] = {nullptr, nullptr};
      cudaStream_t sin = nullptr, sout = nullptr;
      bool keep = false;
      ~Pipe() {
        if (keep) return;
        for (int i = 0; i < 2; i++) {
          if (bx[i]) cudaFree(bx[i]);
          if (by[i]) cudaFree(by[i]);
          if (ein[i]) cudaEventDestroy(ein[i]);
          if (ekern[i]) cudaEventDestroy(ekern[i]);
          if (eout[i]) cudaEventDestroy(eout[i]);
        }
        if (sin) cudaStreamDestroy(sin);
        if (sout) cudaStreamDestroy(sout);
      }
    } p;
    for (int i = 0; i < 2; i++) {
      SB2_CUDA_TRY(cudaMalloc(&p.bx[i], sizeof(double) * len));
      SB2_CUDA_TRY(cudaMalloc(&p.by[i], sizeof(double) * len));
      SB2_CUDA_TRY(cudaEventCreateWithFlags(&p.ein[i], cudaEventDisableTiming));
      SB2_CUDA_TRY(cudaEventCreateWithFlags(&p.ekern[i], cudaEventDisableTiming));
      SB2_CUDA_TRY(cudaEventCreateWithFlags(&p.eout[i], cudaEventDisableTiming));
    }
    SB2_CUDA_TRY(cudaStreamCreateWithFlags(&p.sout, cudaStreamNonBlocking));
    SB2_CUDA_TRY(cudaStreamCreateWithFlags(&p.sin, cudaStreamNonBlocking));
    for (int i = 0; i < 2; i++) {
      A->d_bx[i] = p.bx[i];
      A->d_by[i] = p.by[i];
      A->e_in[i] = p.ein[i];
      A->e_kern[i] = p.ekern[i];
      A->e_out[i] = p.eout[i];
    }
    A->s_out = p.sout;
    A->s_in = p.sin;
    p.keep = true;
  }
  // the copy streams start after the work already queued on the caller's stream
  SB2_CUDA_TRY(cudaEventRecord(A->e_kern[0], s));
  SB2_CUDA_TRY(cudaStreamWaitEvent(A->s_in, A->e_kern[0], 0));
  SB2_CUDA_TRY(cudaStreamWaitEvent(A->s_out, A->e_kern[0], 0));
  for (int i = 0; i < count; i++) {
    const int b = i & 1;
    if (i >= 2) SB2_CUDA_TRY(cudaStreamWaitEvent(A->s_in, A->e_kern[b], 0));
    if (nx > 0)
      SB2_CUDA_TRY(cudaMemcpyAsync(A->d_bx[b], x_host + (size_t)i * nx, sizeof(double) * nx,
                                   cudaMemcpyHostToDevice, A->s_in));
    SB2_CUDA_TRY(cudaEventRecord(A->e_in[b], A->s_in));
    SB2_CUDA_TRY(cudaStreamWaitEvent(s, A->e_in[b], 0));
    if (i >= 2) SB2_CUDA_TRY(cudaStreamWaitEvent(s, A->e_out[b], 0));
    SB2_TRY(spmv_common(A, trans, alpha, A->d_bx[b], 0.0, A->d_by[b], true, s));
    SB2_CUDA_TRY(cudaEventRecord(A->e_kern[b], s));
    SB2_CUDA_TRY(cudaStreamWaitEvent(A->s_out, A->e_kern[b], 0));
    if (ny > 0)
      SB2_CUDA_TRY(cudaMemcpyAsync(y_host + (size_t)i * ny, A->d_by[b], sizeof(double) * ny,
                                   cudaMemcpyDeviceToHost, A->s_out));
    SB2_CUDA_TRY(cudaEventRecord(A->e_out[b], A->s_out));
  }
  // every product and every copy out has completed when s_out has
  SB2_CUDA_TRY(cudaStreamSynchronize(A->s_out));
  return SB2_OK;
} SB2_CATCH

int sb2_probe_gather(long long nnz, const int* ind, const double* val, const double* x,
                     double* partials, int max_blocks, int* blocks, void* stream) try {
  if (nnz < 0 || max_blocks < 1 || !blocks || (nnz > 0 && (!ind || !x || !partials)))
    return SB2_ERR_INVALID_VALUE;
  if ((reinterpret_cast<uintptr_t>(ind) & 15u) || (val && (reinterpret_cast<uintptr_t>(val) & 15u)))
    return SB2_ERR_INVALID_VALUE;  // 16-byte loads of the streams
  const int g = std::max(1, std::min(max_blocks, num_sms(current_device()) * 8));
  *blocks = g;
  probe_gather_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(nnz, ind, val, x, partials);
  return map_cuda_error(cudaGetLastError());
} SB2_CATCH

}  // extern "C"
