// Krylov loops as chains of full-occupancy kernels (large systems).
//
// For large n the cost of an iteration is the HBM traffic of its passes, and
// each pass runs best at the occupancy its own kernel allows (the SpMV at 8
// CTAs per SM).  The chain keeps every scalar of the iteration (rho, alpha,
// beta, the residual, the counters and the stop flag) in device memory:
// kernels read them, the last CTA of each reducing kernel updates them, and a
// kernel launched after the solve has stopped returns at once.  The host
// enqueues iterations in chunks and reads the stop flag once per chunk, so
// the device never waits for the host.
//
// Reductions are deterministic: every CTA deposits its partial sum, and the
// CTA that completes the deposits sums them in CTA order.  A reduction may
// span two kernels (SELL slices + long rows): both deposit into one array
// and the last depositor of the pair finishes it.
#pragma once

#include <algorithm>
#include <cmath>

#include "sell.cuh"

namespace sb2 {

// Device-resident state of one chained solve, in the vector precision T.
template <typename T>
struct ChainState {
  T rho, rho_1, alpha, beta;
  double facteur;  // 1 / ||b||
  double reste;    // relative residual of the last Finished() test
  int nb_iter, max_iter, done, fail, init_failed, hist_len, hist_cap;
  double tol;
  unsigned cnt;  // deposits of the reduction in progress
  // reliable updates (mixed precision): when the low-precision residual has
  // dropped by `delta` since the last correction, or predicts convergence,
  // the iteration halts with `pending` set and the host applies the
  // high-precision correction before resuming
  int pending;
  double delta;
  double rmax;   // ||r|| at the last correction
  T zc;          // coefficient of z in the next p update (1 except right
                 // after a correction, where it also removes from p its
                 // component along the replaced residual)
  // BiCgStab (chain_pbicgstab): omega, and `fin` once Finished(||s||) has
  // stopped the solve in mid-loop (x still takes alpha * phat)
  T omega;
  int fin;
};

template <typename T>
struct ChainArgs {
  int n;
  const T* b;
  T* x;
  T* r;
  T* p;
  T* q;
  const T* diag;  // Jacobi: z = r / diag; nullptr: identity
  ChainState<T>* st;
  T* part;        // deposits (2 per CTA at most)
  double* hist;   // relative residual of each Finished() test
  int* hist_it;
};

// Device-resident scalars of chain_pgmres beyond ChainState's (whose
// `pending` flags the end of a cycle there).
struct GmresChainExtra {
  int m, ld;
  int ncol;       // steps done in the current cycle
  int inner_max;  // iteration count at which the cycle ends
  double beta;    // ||r|| at the start of the cycle
  double h;       // the coefficient of the next MGS pass
  double hi;      // ||w|| of the last step
};

// A preconditioner apply z = M^{-1} r enqueued on a stream (chain_pcg).
struct PrecondLaunch {
  const sb2_precond* M;
  bool trans;
  int operator()(const double* r, double* z, cudaStream_t s) const;
};

// Size of the next chunk of a chained loop: from the residual's decrease over
// the last chunk, the iterations still needed to reach `target` (a relative
// residual: the stop, or the next correction), less those already queued,
// within [lo, hi]; `dflt` until two states have been seen.  Fewer iterations
// queued past the stop means fewer kernels that only return.
struct ChunkPlanner {
  int prev_it = -1;
  double prev_res = 0.0;
  void reset() { prev_it = -1; }
  int next(int it, double res, double target, int in_flight, int dflt, int lo = 8, int hi = 32) {
    int c = dflt;
    if (prev_it >= 0 && it > prev_it && res > 0.0 && res < prev_res && target > 0.0) {
      const double q = std::pow(res / prev_res, 1.0 / (double)(it - prev_it));
      const double need = target < res ? std::log(target / res) / std::log(q) : 0.0;
      c = (int)std::ceil(need) - in_flight + 1;
    }
    prev_it = it;
    prev_res = res;
    return std::max(lo, std::min(hi, c));
  }
};

// Host side of a chained loop.  After each chunk of iterations the state is
// copied to pinned host memory and an event marks its arrival; the caller
// keeps one chunk queued behind the one it waits on, so the device does not
// idle while the host wakes up (kernels queued after the stop return at
// once).  The two pinned snapshot slots are allocated once per host thread
// and kept until exit.
template <typename T>
class ChainPipe {
 public:
  ChainPipe() = default;
  ChainPipe(const ChainPipe&) = delete;
  ChainPipe& operator=(const ChainPipe&) = delete;
  ~ChainPipe() {
    for (int i = 0; i < 2; i++)
      if (ev_[i]) cudaEventDestroy(ev_[i]);
  }
  int init() {
    static thread_local void* pinned = nullptr;
    if (!pinned) {
      cudaError_t e = cudaHostAlloc(&pinned, 2 * sizeof(ChainState<double>), cudaHostAllocPortable);
      if (e != cudaSuccess) {
        pinned = nullptr;
        return map_cuda_error(e);
      }
    }
    snap_ = static_cast<ChainState<T>*>(pinned);
    for (int i = 0; i < 2; i++) {
      cudaError_t e = cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return map_cuda_error(e);
    }
    return SB2_OK;
  }
  // a chunk has been enqueued: snapshot the state behind it
  int mark(const ChainState<T>* st, int launched, cudaStream_t s) {
    const int k = w_;
    w_ ^= 1;
    at_[k] = launched;
    out_++;
    cudaError_t e = cudaMemcpyAsync(&snap_[k], st, sizeof(ChainState<T>), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(ev_[k], s);
    return map_cuda_error(e);
  }
  // the oldest snapshot not yet read (waits for its chunk)
  int wait(ChainState<T>* h, int* launched) {
    const int k = r_;
    r_ ^= 1;
    out_--;
    cudaError_t e = cudaEventSynchronize(ev_[k]);
    if (e != cudaSuccess) return map_cuda_error(e);
    *h = snap_[k];
    if (launched) *launched = at_[k];
    return SB2_OK;
  }
  int outstanding() const { return out_; }
  // every marked chunk has completed (the stream was synchronized)
  void reset() {
    w_ = r_ = out_ = 0;
  }

 private:
  ChainState<T>* snap_ = nullptr;
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  int at_[2] = {0, 0};
  int w_ = 0, r_ = 0, out_ = 0;
};

#ifdef __CUDACC__

template <typename T>
__device__ __forceinline__ T zval(const T* diag, long long i, T r) {
  return diag ? r / __ldg(diag + i) : r;  // IEEE division, as the reference's Jacobi
}

// Deposit K block sums (valid in thread 0) at slots [off, off+K*tot) with
// stride tot; the CTA completing `tot` deposits sums them in order and
// returns true (all its threads), with the totals in out[0..K).
template <int NT, int K, typename T>
__device__ __forceinline__ bool deposit_and_finish(const T (&v)[K], T* part, unsigned* cnt,
                                                   int slot, int tot, T* s_red, T* out) {
  __shared__ int s_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) part[(size_t)k * tot + slot] = v[k];
    __threadfence();
    s_last = (atomicAdd(cnt, 1u) == (unsigned)tot - 1u) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; k++) {
    // four independent chains keep several loads in flight; the order of
    // every addition is fixed by (slot, thread), so the total is too
    const T* pv = part + (size_t)k * tot;
    T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
    int i = threadIdx.x;
    for (; i + 3 * NT < tot; i += 4 * NT) {
      a0 = add_rn(a0, __ldcg(pv + i));
      a1 = add_rn(a1, __ldcg(pv + i + NT));
      a2 = add_rn(a2, __ldcg(pv + i + 2 * NT));
      a3 = add_rn(a3, __ldcg(pv + i + 3 * NT));
    }
    for (; i < tot; i += NT) a0 = add_rn(a0, __ldcg(pv + i));
    T a = block_sum<NT>(add_rn(add_rn(a0, a1), add_rn(a2, a3)), s_red);
    if (threadIdx.x == 0) out[k] = a;
  }
  if (threadIdx.x == 0) *cnt = 0u;
  __syncthreads();
  return true;
}

#endif  // __CUDACC__

}  // namespace sb2
