// Persistent-kernel plumbing: a bounded grid barrier that also performs the
// deterministic cross-CTA reduction, and the per-solve device state.
//
// The kernels using it are launched cooperatively (all CTAs co-resident).
// Every wait is bounded by a wall-clock limit read from %globaltimer: a CTA
// that waits too long sets `status` and the whole grid unwinds, so a solve can
// never hang the GPU.
#pragma once

#include "spmv_core.cuh"

namespace sb2 {

constexpr int kMaxRed = 8;  // scalars reduced by one barrier at most

struct GridSync {
  unsigned count;  // arrivals at the current barrier
  unsigned gen;    // barrier generation
  int status;      // 0 ok, 1 a wait ran out
  int pad;
  double res[kMaxRed];
};

struct SolveOut {
  int nb_iter;
  int error_code;
  int init_failed;
  int hist_len;
  double facteur_reste;
  double last_residual;
};

struct Persist {
  GridSync* sync;
  double* partials;  // [kMaxRed * gridDim.x]
  unsigned long long wait_ns;
};

// Record of the relative residual of one Finished() test.
struct History {
  double* res;
  int* it;
  int cap;
};

#ifdef __CUDACC__

// Grid barrier.  Thread 0 of each CTA deposits K block sums (s_vals[0..K)),
// the last CTA to arrive sums the deposits in CTA order (the same tree on
// every run), publishes them and releases the grid; on return s_vals holds
// the K grid sums in every CTA.  Returns false when a wait ran out or another
// CTA reported so.
template <int NT>
__device__ __forceinline__ bool grid_sync(const Persist& P, unsigned& epoch, int K,
                                          double* s_vals, double* s_red) {
  __shared__ int s_last, s_ok;  // separate: a lagging warp may still read s_last
  const int tid = threadIdx.x;
  const unsigned G = gridDim.x;
  if (tid == 0)
    for (int k = 0; k < K; k++) P.partials[k * G + blockIdx.x] = s_vals[k];
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&P.sync->count, 1u);
    s_last = (prev == G - 1) ? 1 : 0;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    for (int k = 0; k < K; k++) {
      const double* pv = P.partials + k * G;
      double v0 = 0.0, v1 = 0.0;
      unsigned i = tid;
      for (; i + NT < G; i += 2 * NT) {
        v0 = add_rn(v0, __ldcg(pv + i));
        v1 = add_rn(v1, __ldcg(pv + i + NT));
      }
      if (i < G) v0 = add_rn(v0, __ldcg(pv + i));
      const double v = block_sum<NT>(add_rn(v0, v1), s_red);
      if (tid == 0) P.sync->res[k] = v;
    }
    if (tid == 0) {
      P.sync->count = 0u;
      __threadfence();
      st_release_u32(&P.sync->gen, epoch + 1u);
    }
  } else if (tid == 0) {
    const unsigned long long t0 = global_timer_ns();
    while (ld_acquire_u32(&P.sync->gen) == epoch) {
      if (global_timer_ns() - t0 > P.wait_ns) {
        atomicExch(&P.sync->status, 1);
        break;
      }
      __nanosleep(32);
    }
    // a gpu-scope fence after the wait, as cooperative groups' grid.sync
    // takes: with the CTA barrier below, the L1-cached gathers of the next
    // phase (XLoadCa) see every write made before the barrier
    __threadfence();
  }
  if (tid == 0) {
    for (int k = 0; k < K; k++) s_vals[k] = __ldcg(P.sync->res + k);
    s_ok = (*((volatile int*)&P.sync->status) == 0) ? 1 : 0;
  }
  __syncthreads();
  epoch++;
  return s_ok != 0;
}

// Gathers of the product's operand inside a persistent kernel: cached in L1
// (ld.ca), where a stencil's neighbouring columns hit.  The operand must have
// been written in an EARLIER phase, never in the phase that gathers it: every
// phase ends at grid_sync / grid_sync_wide, whose gpu-scope fences (the
// waiting thread's acquire and fence, the last CTA's fence) and CTA barrier
// order these loads after every write released before the barrier -- the
// guarantee ordinary loads have after cooperative groups' grid.sync.  The
// read-only matrix uses the streaming path.
template <typename T>
struct XLoadCa {
  const T* x;
  __device__ __forceinline__ T operator()(int j) const { return __ldca(x + j); }
  template <typename O>
  __device__ __forceinline__ void gather4(const int4& c, O (&o)[4]) const {
    T v[4];
    if (quad_contiguous(x, c)) {
      vld4_ca(x + c.x, v);
    } else {
      v[0] = __ldca(x + c.x); v[1] = __ldca(x + c.y); v[2] = __ldca(x + c.z); v[3] = __ldca(x + c.w);
    }
    o[0] = O(v[0]); o[1] = O(v[1]); o[2] = O(v[2]); o[3] = O(v[3]);
  }
};

#endif  // __CUDACC__

}  // namespace sb2
