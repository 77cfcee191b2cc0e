// Conjugate gradients as a chain of full-occupancy kernels (see chain.cuh).
//
// Same iteration as the reference's Cg (Cg.cxx:45-116) and as the persistent
// kernel of krylov.cu:
//   while (!Finished(r)) { z = M^{-1} r; rho = (r, z); [rho == 0: fail 1]
//     p = z | p = beta*p + z;  q = A p;  delta = (p, q); [delta == 0: fail 2]
//     alpha = rho/delta;  x += alpha p;  r -= alpha q;  ++iter }
// with one kernel per pass:  K_p (p update), K_q (q = A p fused with (p, q)),
// K_x (x and r updates fused with ||r||^2 and (r, z) and the stopping test).
// Templated on the vector/scalar type T and the matrix value type VT, so the
// same chain runs the FP64 drop-in and the FP32 inner solves of iterative
// refinement.
#include <algorithm>
#include <cmath>
#include <vector>

#include "chain.cuh"
#include "givens.cuh"
#include "spmv_core.cuh"

namespace sb2 {

constexpr int CT = 256;

template <typename T>
__device__ __forceinline__ bool chain_done(const ChainState<T>* st) {
  return (*((volatile const int*)&st->done) | *((volatile const int*)&st->pending)) != 0;
}

// Finished() at the current nb_iter (Iterative.cxx:299-319), run by one thread.
template <typename T>
__device__ __forceinline__ bool chain_finished_at(ChainState<T>* st, double* hist, int* hist_it,
                                                  T rr) {
  const T res = (T)sqrt(rr);
  const double reste = (double)((T)st->facteur * res);
  st->reste = reste;
  if (st->hist_len < st->hist_cap) {
    hist[st->hist_len] = reste;
    hist_it[st->hist_len] = st->nb_iter;
  }
  st->hist_len++;
  return (reste < st->tol) || (st->nb_iter >= st->max_iter);
}

template <typename T>
__device__ __forceinline__ bool chain_finished(ChainArgs<T>& a, T rr) {
  return chain_finished_at(a.st, a.hist, a.hist_it, rr);
}

// ||b||: Init(b) (Iterative.cxx:235-249).
template <typename T>
__global__ void __launch_bounds__(CT, 8) k_norm_b(ChainArgs<T> a) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[1];
  T acc = T(0);
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    const T bi = __ldg(a.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  T v[1] = {block_sum<CT>(acc, s_red)};
  if (deposit_and_finish<CT, 1>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    const T nb = (T)sqrt(s_out[0]);
    if (nb == T(0)) {
      a.st->init_failed = 1;
      a.st->done = 1;
    } else {
      a.st->facteur = (double)(T(1) / nb);
    }
  }
}

// Start of the loop once r is known: Finished(r) at iteration 0, then rho.
template <typename T>
__device__ __forceinline__ void chain_start(ChainArgs<T>& a, T rr, T rz) {
  if (chain_finished(a, rr)) {
    a.st->done = 1;
    return;
  }
  a.st->rho = rz;
  if (rz == T(0)) {
    a.st->fail = 1;
    a.st->done = 1;
  }
}

// Null initial guess: x = 0, r = b, with ||r||^2 and (r, z).
template <typename T>
__global__ void __launch_bounds__(CT, 8) k_init_null(ChainArgs<T> a) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[2];
  if (chain_done(a.st)) return;
  T rr = T(0), rz = T(0);
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    const T bi = __ldg(a.b + i);
    a.x[i] = T(0);
    a.r[i] = bi;
    rr = add_rn(rr, mul_rn(bi, bi));
    rz = add_rn(rz, mul_rn(bi, zval(a.diag, i, bi)));
  }
  T v[2] = {block_sum<CT>(rr, s_red), block_sum<CT>(rz, s_red)};
  if (deposit_and_finish<CT, 2>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0)
    chain_start(a, s_out[0], s_out[1]);
}

// r = b - A x (Copy(b, r); MltAdd(-1, A, x, 1, r)) with ||r||^2 and (r, z).
template <typename T>
struct EpiChainResidual {
  ChainArgs<T> a;
  T rr, rz;
  __device__ __forceinline__ void operator()(int i, T t) {
    const T v = add_rn(__ldg(a.b + i), -t);
    a.r[i] = v;
    rr = add_rn(rr, mul_rn(v, v));
    rz = add_rn(rz, mul_rn(v, zval(a.diag, i, v)));
  }
};

// q = A p with (p, q).
template <typename T>
struct EpiChainDot {
  T* q;
  const T* p;
  T acc;
  __device__ __forceinline__ void operator()(int i, T t) {
    q[i] = t;
    acc = add_rn(acc, mul_rn(__ldg(p + i), t));
  }
  __device__ __forceinline__ void quad(int i, const T* t) {
    if (!is_aligned16(q + i) || !is_aligned16(p + i)) {
      for (int j = 0; j < 4; j++) (*this)(i + j, t[j]);
      return;
    }
    T pv[4];
    const T tv[4] = {t[0], t[1], t[2], t[3]};
    vld4_ldg(p + i, pv);
    vst4(q + i, tv);
#pragma unroll
    for (int j = 0; j < 4; j++) acc = add_rn(acc, mul_rn(pv[j], t[j]));
  }
};

// After the (p, q) reduction: alpha = rho / delta, or breakdown #2.
template <typename T>
__device__ __forceinline__ void chain_after_delta(ChainArgs<T>& a, T delta) {
  if (delta == T(0)) {
    a.st->fail = 2;
    a.st->done = 1;
    return;
  }
  a.st->alpha = a.st->rho / delta;
}

// One SELL product fused with a reduction; MODE 0: q = A p and (p, q);
// MODE 1: r = b - A x with ||r||^2, (r, z).  PART 0: slices, PART 1: long
// rows (deposit slots after the slices').
// Slice-kernel shape per value type: resident CTAs per SM (the launch
// bound and the reducing grid) and groups in flight per lane.
template <typename VT>
constexpr int chain_spmv_occ() { return sizeof(VT) == 8 ? 4 : 4; }
template <typename VT>
constexpr int chain_spmv_unroll() { return sizeof(VT) == 8 ? 1 : 3; }

template <typename T, typename VT, int MODE, int PART>
__global__ void __launch_bounds__(CT, PART == 1 ? 1 : chain_spmv_occ<VT>())
    k_spmv(ChainArgs<T> a, SellOp<VT> S, int slot0, int tot) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[2];
  pdl_wait();
  pdl_release();
  if (chain_done(a.st)) return;
  if (MODE == 0) {
    EpiChainDot<T> epi{a.q, a.p, T(0)};
    XLoadLdg<T> xl{a.p};
    if (PART == 0)
      sell_spmv_slices<CT, VT, T, XLoadLdg<T>, EpiChainDot<T>, chain_spmv_unroll<VT>()>(
          S, xl, epi, blockIdx.x, gridDim.x);
    else
      sell_spmv_long<CT, VT, T>(S, xl, epi, s_red, blockIdx.x, gridDim.x);
    T v[1] = {block_sum<CT>(epi.acc, s_red)};
    if (deposit_and_finish<CT, 1>(v, a.part, &a.st->cnt, slot0 + blockIdx.x, tot, s_red, s_out) &&
        threadIdx.x == 0)
      chain_after_delta(a, s_out[0]);
  } else {
    EpiChainResidual<T> epi{a, T(0), T(0)};
    XLoadLdg<T> xl{a.x};
    if (PART == 0)
      sell_spmv_slices<CT, VT, T, XLoadLdg<T>, EpiChainResidual<T>, chain_spmv_unroll<VT>()>(
          S, xl, epi, blockIdx.x, gridDim.x);
    else
      sell_spmv_long<CT, VT, T>(S, xl, epi, s_red, blockIdx.x, gridDim.x);
    T v[2] = {block_sum<CT>(epi.rr, s_red), block_sum<CT>(epi.rz, s_red)};
    if (deposit_and_finish<CT, 2>(v, a.part, &a.st->cnt, slot0 + blockIdx.x, tot, s_red, s_out) &&
        threadIdx.x == 0)
      chain_start(a, s_out[0], s_out[1]);
  }
}

// Elementwise passes work on groups of 4 consecutive entries loaded with
// 16-byte accesses (the work vectors come from one 256-byte-aligned block;
// a caller's x or b that is not 16-byte aligned takes the scalar path).
template <typename T>
struct Quad {
  T v[4];
};
template <typename T>
__device__ __forceinline__ Quad<T> ld4(const T* p) {
  Quad<T> q;
  if (sizeof(T) == 8) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *(reinterpret_cast<const double2*>(p) + 1);
    q.v[0] = (T)a.x; q.v[1] = (T)a.y; q.v[2] = (T)b.x; q.v[3] = (T)b.y;
  } else {
    const float4 a = *reinterpret_cast<const float4*>(p);
    q.v[0] = (T)a.x; q.v[1] = (T)a.y; q.v[2] = (T)a.z; q.v[3] = (T)a.w;
  }
  return q;
}
template <typename T>
__device__ __forceinline__ void st4(T* p, const Quad<T>& q) {
  if (sizeof(T) == 8) {
    *reinterpret_cast<double2*>(p) = make_double2((double)q.v[0], (double)q.v[1]);
    *(reinterpret_cast<double2*>(p) + 1) = make_double2((double)q.v[2], (double)q.v[3]);
  } else {
    *reinterpret_cast<float4*>(p) = make_float4((float)q.v[0], (float)q.v[1], (float)q.v[2], (float)q.v[3]);
  }
}

__device__ __forceinline__ bool aligned16(const void* p) {
  return (reinterpret_cast<unsigned long long>(p) & 15ull) == 0;
}

// p = z (first iteration) | p = beta*p + z: Mlt(beta, p); Add(1, z, p).
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_p(ChainArgs<T> a) {
  pdl_wait();
  pdl_release();
  if (chain_done(a.st)) return;
  const bool first = (a.st->nb_iter == 0);
  const T beta = a.st->beta;
  const T zc = a.st->zc;  // 1 in the reference's recurrence: 1*z == z exactly
  T* __restrict__ p = a.p;
  const T* __restrict__ r = a.r;
  constexpr int H = sizeof(T) == 8 ? 1 : 2;  // quads per stream: 32 bytes in flight each
  const long long n8 = (aligned16(p) && aligned16(r) && (!a.diag || aligned16(a.diag))) ? a.n / (4 * H) : 0;
  const long long t0 = (long long)blockIdx.x * CT + threadIdx.x, ts = (long long)gridDim.x * CT;
  for (long long g = t0; g < n8; g += ts) {
    const long long i = 4 * H * g;
    Quad<T> rq[H], dq[H], pq[H];
#pragma unroll
    for (int h = 0; h < H; h++) {
      rq[h] = ld4(r + i + 4 * h);
      if (a.diag) dq[h] = ld4(a.diag + i + 4 * h);
      if (!first) pq[h] = ld4(p + i + 4 * h);
    }
#pragma unroll
    for (int h = 0; h < H; h++) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const T z = a.diag ? rq[h].v[k] / dq[h].v[k] : rq[h].v[k];
        pq[h].v[k] = first ? z : add_rn(mul_rn(pq[h].v[k], beta), mul_rn(zc, z));
      }
      st4(p + i + 4 * h, pq[h]);
    }
  }
  for (long long i = 4 * H * n8 + t0; i < a.n; i += ts) {
    const T z = zval(a.diag, i, r[i]);
    p[i] = first ? z : add_rn(mul_rn(p[i], beta), mul_rn(zc, z));
  }
}

// Add(alpha, p, x); Add(-alpha, q, r); ||r||^2, (r, z); ++iter; the test.
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_x(ChainArgs<T> a) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[2];
  pdl_wait();
  pdl_release();
  if (chain_done(a.st)) return;
  const T alpha = a.st->alpha;
  T* __restrict__ x = a.x;
  T* __restrict__ r = a.r;
  const T* __restrict__ p = a.p;
  const T* __restrict__ q = a.q;
  T rr = T(0), rz = T(0);
  const bool vec = aligned16(x) && aligned16(r) && aligned16(p) && aligned16(q) &&
                   (!a.diag || aligned16(a.diag));
  constexpr int H = sizeof(T) == 8 ? 1 : 2;  // quads per stream: 32 bytes in flight each
  const long long n8 = vec ? a.n / (4 * H) : 0;
  const long long t0 = (long long)blockIdx.x * CT + threadIdx.x, ts = (long long)gridDim.x * CT;
  for (long long g = t0; g < n8; g += ts) {
    const long long i = 4 * H * g;
    Quad<T> xq[H], rq[H], pq[H], qq[H], dq[H];
#pragma unroll
    for (int h = 0; h < H; h++) {
      xq[h] = ld4(x + i + 4 * h);
      rq[h] = ld4(r + i + 4 * h);
      pq[h] = ld4(p + i + 4 * h);
      qq[h] = ld4(q + i + 4 * h);
      if (a.diag) dq[h] = ld4(a.diag + i + 4 * h);
    }
#pragma unroll
    for (int h = 0; h < H; h++) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (alpha != T(0)) xq[h].v[k] = add_rn(xq[h].v[k], mul_rn(alpha, pq[h].v[k]));
        if (-alpha != T(0)) rq[h].v[k] = add_rn(rq[h].v[k], mul_rn(-alpha, qq[h].v[k]));
        const T ri = rq[h].v[k];
        rr = add_rn(rr, mul_rn(ri, ri));
        rz = add_rn(rz, mul_rn(ri, a.diag ? ri / dq[h].v[k] : ri));
      }
      if (alpha != T(0)) st4(x + i + 4 * h, xq[h]);
      if (-alpha != T(0)) st4(r + i + 4 * h, rq[h]);
    }
  }
  for (long long i = 4 * H * n8 + t0; i < a.n; i += ts) {
    if (alpha != T(0)) x[i] = add_rn(x[i], mul_rn(alpha, __ldg(p + i)));
    T ri = r[i];
    if (-alpha != T(0)) {
      ri = add_rn(ri, mul_rn(-alpha, __ldg(q + i)));
      r[i] = ri;
    }
    rr = add_rn(rr, mul_rn(ri, ri));
    rz = add_rn(rz, mul_rn(ri, zval(a.diag, i, ri)));
  }
  T v[2] = {block_sum<CT>(rr, s_red), block_sum<CT>(rz, s_red)};
  if (deposit_and_finish<CT, 2>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    ChainState<T>* st = a.st;
    st->nb_iter++;
    if (chain_finished(a, s_out[0])) {
      st->done = 1;
      return;
    }
    st->rho_1 = st->rho;
    st->rho = s_out[1];
    if (st->rho == T(0)) {
      st->fail = 1;
      st->done = 1;
      return;
    }
    st->beta = st->rho / st->rho_1;
  }
}

// Reliable-update form of k_x (mixed precision): x here is the low-precision
// correction accumulated since the last high-precision update.  The test uses
// ||r|| / ||b|| as the estimate of the true residual; a drop by `delta` since
// the last correction, or a predicted convergence, halts with `pending`.
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_x_ru(ChainArgs<T> a) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[2];
  pdl_wait();
  pdl_release();
  if (chain_done(a.st)) return;
  const T alpha = a.st->alpha;
  T* __restrict__ x = a.x;
  T* __restrict__ r = a.r;
  const T* __restrict__ p = a.p;
  const T* __restrict__ q = a.q;
  T rr = T(0), rz = T(0);
  const bool vec = aligned16(x) && aligned16(r) && aligned16(p) && aligned16(q) &&
                   (!a.diag || aligned16(a.diag));
  constexpr int H = sizeof(T) == 8 ? 1 : 2;  // quads per stream: 32 bytes in flight each
  const long long n8 = vec ? a.n / (4 * H) : 0;
  const long long t0 = (long long)blockIdx.x * CT + threadIdx.x, ts = (long long)gridDim.x * CT;
  for (long long g = t0; g < n8; g += ts) {
    const long long i = 4 * H * g;
    Quad<T> xq[H], rq[H], pq[H], qq[H], dq[H];
#pragma unroll
    for (int h = 0; h < H; h++) {
      xq[h] = ld4(x + i + 4 * h);
      rq[h] = ld4(r + i + 4 * h);
      pq[h] = ld4(p + i + 4 * h);
      qq[h] = ld4(q + i + 4 * h);
      if (a.diag) dq[h] = ld4(a.diag + i + 4 * h);
    }
#pragma unroll
    for (int h = 0; h < H; h++) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        xq[h].v[k] = add_rn(xq[h].v[k], mul_rn(alpha, pq[h].v[k]));
        rq[h].v[k] = add_rn(rq[h].v[k], mul_rn(-alpha, qq[h].v[k]));
        const T ri = rq[h].v[k];
        rr = add_rn(rr, mul_rn(ri, ri));
        rz = add_rn(rz, mul_rn(ri, a.diag ? ri / dq[h].v[k] : ri));
      }
      st4(x + i + 4 * h, xq[h]);
      st4(r + i + 4 * h, rq[h]);
    }
  }
  for (long long i = 4 * H * n8 + t0; i < a.n; i += ts) {
    x[i] = add_rn(x[i], mul_rn(alpha, __ldg(p + i)));
    const T ri = add_rn(r[i], mul_rn(-alpha, __ldg(q + i)));
    r[i] = ri;
    rr = add_rn(rr, mul_rn(ri, ri));
    rz = add_rn(rz, mul_rn(ri, zval(a.diag, i, ri)));
  }
  T v[2] = {block_sum<CT>(rr, s_red), block_sum<CT>(rz, s_red)};
  if (deposit_and_finish<CT, 2>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    ChainState<T>* st = a.st;
    st->nb_iter++;
    st->zc = T(1);
    const double res = sqrt((double)s_out[0]);
    st->reste = st->facteur * res;
    st->rho_1 = st->rho;
    st->rho = s_out[1];
    if (st->nb_iter >= st->max_iter) {
      st->pending = 1;  // correct once more, then stop
      return;
    }
    if (st->reste < st->tol || res < st->delta * st->rmax) {
      st->pending = 1;
      return;
    }
    if (st->rho == T(0)) {
      st->fail = 1;
      st->pending = 1;
      return;
    }
    st->beta = st->rho / st->rho_1;
  }
}

// After a high-precision correction replaced r: rho = (r, z) of the new
// residual, beta against the previous iteration's rho, new ||r|| reference.
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_rho_ru(ChainArgs<T> a) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[3];
  T rr = T(0), rz = T(0), rp = T(0);
  const bool have_p = (a.st->nb_iter > 0);
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    const T ri = a.r[i];
    rr = add_rn(rr, mul_rn(ri, ri));
    rz = add_rn(rz, mul_rn(ri, zval(a.diag, i, ri)));
    if (have_p) rp = add_rn(rp, mul_rn(ri, a.p[i]));
  }
  T v[3] = {block_sum<CT>(rr, s_red), block_sum<CT>(rz, s_red), block_sum<CT>(rp, s_red)};
  if (deposit_and_finish<CT, 3>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    ChainState<T>* st = a.st;
    st->rmax = sqrt((double)s_out[0]);
    st->rho = s_out[1];
    st->zc = T(1);
    if (!have_p) {
      st->pending = 0;  // first direction: p = z
      return;
    }
    if (st->rho == T(0)) {
      st->fail = 1;
      st->done = 1;
      return;
    }
    st->beta = st->rho / st->rho_1;
    // p <- z + beta (p - ((r, p) / (r, z)) z): the previous direction loses
    // its component along the replaced residual, restoring r orthogonal to p
    st->zc = T(1) - st->beta * (s_out[2] / st->rho);
    st->pending = 0;
  }
}

// ----------------------------------------------------------------- any preconditioner
//
// Cg with a preconditioner applied by its own launches (SOR sweeps, ILUT
// sweeps): z = M^{-1} r is materialized between the passes, and the loop is
//   [M apply] -> K_rz (rho = (r, z), beta) -> K_pz (p) -> K_q (q = A p, delta,
//   alpha) -> K_xr (x, r, ||r||^2, the test)
// with every scalar in device memory, as in the chain above.  The apply's
// launches do not read the stop flag: after the stop they recompute z from
// the final r, and the passes after them return at once.

// rho = (r, z) (Cg.cxx: DotProdConj(r, z)); breakdown #1; beta = rho / rho_1.
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_pc_rz(ChainArgs<T> a, const T* __restrict__ z) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[1];
  pdl_wait();
  pdl_release();
  if (chain_done(a.st)) return;
  T rz = T(0);
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT)
    rz = add_rn(rz, mul_rn(__ldg(a.r + i), __ldg(z + i)));
  T v[1] = {block_sum<CT>(rz, s_red)};
  if (deposit_and_finish<CT, 1>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    ChainState<T>* st = a.st;
    st->rho = s_out[0];
    if (st->rho == T(0)) {
      st->fail = 1;
      st->done = 1;
      return;
    }
    if (st->nb_iter > 0) st->beta = st->rho / st->rho_1;
  }
}

// p = z (first) | p = beta*p + z: Mlt(beta, p); Add(1, z, p).
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_pc_p(ChainArgs<T> a, const T* __restrict__ z) {
  pdl_wait();
  pdl_release();
  if (chain_done(a.st)) return;
  const bool first = (a.st->nb_iter == 0);
  const T beta = a.st->beta;
  T* __restrict__ p = a.p;
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    const T zi = __ldg(z + i);
    p[i] = first ? zi : add_rn(mul_rn(p[i], beta), zi);
  }
}

// Add(alpha, p, x); Add(-alpha, q, r); rho_1 = rho; ++iter; Finished(r).
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_pc_x(ChainArgs<T> a) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[1];
  pdl_wait();
  pdl_release();
  if (chain_done(a.st)) return;
  const T alpha = a.st->alpha;
  T rr = T(0);
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    if (alpha != T(0)) a.x[i] = add_rn(a.x[i], mul_rn(alpha, __ldg(a.p + i)));
    T ri = a.r[i];
    if (-alpha != T(0)) {
      ri = add_rn(ri, mul_rn(-alpha, __ldg(a.q + i)));
      a.r[i] = ri;
    }
    rr = add_rn(rr, mul_rn(ri, ri));
  }
  T v[1] = {block_sum<CT>(rr, s_red)};
  if (deposit_and_finish<CT, 1>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    ChainState<T>* st = a.st;
    st->rho_1 = st->rho;
    st->nb_iter++;
    if (chain_finished(a, s_out[0])) st->done = 1;
  }
}

// ----------------------------------------------------------------- BiCgStab, any preconditioner
//
// BiCgStab (BiCgStab.cxx:43-145) with a preconditioner applied by its own
// launches, every scalar in device memory.  One loop (two iterations of the
// reference's counter):
//   K_bp (p) -> [M apply: phat] -> K_bv (v = A phat, sigma = (rt, v), alpha)
//   -> K_bs (s = r - alpha v, ++iter, Finished(||s||)) -> [M apply: shat]
//   -> K_bt (t = A shat, (t, s), (t, t), omega)
//   -> K_bxr (x += alpha phat + omega shat, r = s - omega t, ++iter,
//             Finished(||r||), rho = (rt, r), the breakdowns, beta)
// A stop on ||s|| sets `fin`: the products after it return, K_bxr only adds
// alpha phat to x and ends the solve.

template <typename T>
struct BicgChain {
  int n;
  T* x;
  T* r;
  T* rt;
  T* p;
  T* phat;
  T* v;
  T* s;
  T* shat;
  T* t;
  ChainState<T>* st;
  T* part;
  double* hist;
  int* hist_it;
};

template <typename T>
__device__ __forceinline__ bool bicg_stopped(const ChainState<T>* st) {
  return (*((volatile const int*)&st->done) | *((volatile const int*)&st->fin)) != 0;
}

// rt = r: the shadow residual (Copy(r, rtilde)), after the start kernels
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_b_copy(BicgChain<T> a) {
  if (*((volatile const int*)&a.st->done)) return;
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT)
    a.rt[i] = a.r[i];
}

// p = r (first loop) | Add(-omega, v, p); Mlt(beta, p); Add(1, r, p)
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_b_p(BicgChain<T> a) {
  pdl_wait();
  pdl_release();
  if (bicg_stopped(a.st)) return;
  const bool first = (a.st->nb_iter == 0);
  const T beta = a.st->beta, mo = -a.st->omega;
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    if (first) {
      a.p[i] = a.r[i];
      continue;
    }
    T pi = a.p[i];
    if (mo != T(0)) pi = add_rn(pi, mul_rn(mo, a.v[i]));
    pi = mul_rn(beta, pi);
    a.p[i] = add_rn(pi, a.r[i]);
  }
}

// v = A phat with sigma = (rt, v) (MODE 0); t = A shat with (t, s), (t, t)
// (MODE 1).
template <typename T, int MODE>
struct EpiBicg {
  T* out;
  const T* w;
  T acc0, acc1;
  __device__ __forceinline__ void operator()(int i, T t) {
    out[i] = t;
    if (MODE == 0) {
      acc0 = add_rn(acc0, mul_rn(__ldg(w + i), t));
    } else {
      acc0 = add_rn(acc0, mul_rn(t, __ldg(w + i)));
      acc1 = add_rn(acc1, mul_rn(t, t));
    }
  }
};

template <typename T, typename VT, int MODE, int PART>
__global__ void __launch_bounds__(CT, PART == 1 ? 1 : chain_spmv_occ<VT>())
    k_b_spmv(BicgChain<T> a, SellOp<VT> S, int slot0, int tot) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[2];
  pdl_wait();
  pdl_release();
  if (bicg_stopped(a.st)) return;
  EpiBicg<T, MODE> epi{MODE == 0 ? a.v : a.t, MODE == 0 ? a.rt : a.s, T(0), T(0)};
  XLoadLdg<T> xl{MODE == 0 ? a.phat : a.shat};
  if (PART == 0)
    sell_spmv_slices<CT, VT, T, XLoadLdg<T>, EpiBicg<T, MODE>, chain_spmv_unroll<VT>()>(
        S, xl, epi, blockIdx.x, gridDim.x);
  else
    sell_spmv_long<CT, VT, T>(S, xl, epi, s_red, blockIdx.x, gridDim.x);
  T v[2] = {block_sum<CT>(epi.acc0, s_red), block_sum<CT>(epi.acc1, s_red)};
  if (deposit_and_finish<CT, 2>(v, a.part, &a.st->cnt, slot0 + blockIdx.x, tot, s_red, s_out) &&
      threadIdx.x == 0) {
    ChainState<T>* st = a.st;
    if (MODE == 0) {
      if (s_out[0] == T(0)) {  // breakdown #3
        st->fail = 3;
        st->done = 1;
        return;
      }
      st->alpha = st->rho / s_out[0];
    } else {
      st->omega = s_out[0] / s_out[1];
    }
  }
}

// Copy(r, s); Add(-alpha, v, s); ++iter; Finished(||s||)
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_b_s(BicgChain<T> a) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[1];
  pdl_wait();
  pdl_release();
  if (bicg_stopped(a.st)) return;
  const T ma = -a.st->alpha;
  T ss = T(0);
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    T si = a.r[i];
    if (ma != T(0)) si = add_rn(si, mul_rn(ma, a.v[i]));
    a.s[i] = si;
    ss = add_rn(ss, mul_rn(si, si));
  }
  T v[1] = {block_sum<CT>(ss, s_red)};
  if (deposit_and_finish<CT, 1>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    ChainState<T>* st = a.st;
    st->nb_iter++;
    if (chain_finished_at(st, a.hist, a.hist_it, s_out[0])) st->fin = 1;
  }
}

// Add(alpha, phat, x); Add(omega, shat, x); Copy(s, r); Add(-omega, t, r);
// rho_2 = rho_1; ++iter; then the top of the next loop: Finished(||r||),
// rho_1 = (rt, r), breakdowns #1 and #2, beta = (rho_1/rho_2)(alpha/omega).
// After a stop on ||s||: Add(alpha, phat, x) only, and the solve ends.
template <typename T>
__global__ void __launch_bounds__(CT, 4) k_b_xr(BicgChain<T> a) {
  __shared__ T s_red[CT / 32];
  __shared__ T s_out[2];
  pdl_wait();
  pdl_release();
  ChainState<T>* st = a.st;
  if (*((volatile const int*)&st->done)) return;
  const bool fin = *((volatile const int*)&st->fin) != 0;
  const T alpha = st->alpha, omega = st->omega;
  T rr = T(0), rtr = T(0);
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    T xi = a.x[i];
    if (alpha != T(0)) xi = add_rn(xi, mul_rn(alpha, a.phat[i]));
    if (!fin) {
      if (omega != T(0)) xi = add_rn(xi, mul_rn(omega, a.shat[i]));
      T ri = a.s[i];
      if (-omega != T(0)) ri = add_rn(ri, mul_rn(-omega, a.t[i]));
      a.r[i] = ri;
      rr = add_rn(rr, mul_rn(ri, ri));
      rtr = add_rn(rtr, mul_rn(a.rt[i], ri));
    }
    a.x[i] = xi;
  }
  T v[2] = {block_sum<CT>(rr, s_red), block_sum<CT>(rtr, s_red)};
  if (deposit_and_finish<CT, 2>(v, a.part, &st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    if (fin) {
      st->done = 1;
      return;
    }
    st->rho_1 = st->rho;
    st->nb_iter++;
    if (chain_finished_at(st, a.hist, a.hist_it, s_out[0])) {
      st->done = 1;
      return;
    }
    st->rho = s_out[1];
    if (st->rho == T(0)) {
      st->fail = 1;
      st->done = 1;
      return;
    }
    if (st->omega == T(0)) {
      st->fail = 2;
      st->done = 1;
      return;
    }
    st->beta = mul_rn(st->rho / st->rho_1, st->alpha / st->omega);
  }
}

// ----------------------------------------------------------------- Gmres, any preconditioner
//
// Restarted Gmres(m) (Gmres.cxx:44-183, left preconditioned, Seldon's
// modified Gram-Schmidt) with a preconditioner applied by its own launches,
// every scalar, the Hessenberg matrix, the rotations and s in device memory.
// Step i of a cycle:
//   K_gprod (u = A V_i) -> [M apply: w] -> K_gdot0 (H(0,i) = (V_0, w))
//   -> K_gmgs(k), k = 0..i: Add(-H(k,i), V_k, w), then H(k+1,i) = (V_{k+1}, w)
//      or, for k = i, ||w|| and the step's tail (rotations, ++iter, the inner
//      test) -> K_gvnext (V_{i+1} = w / ||w||)
// A step's kernels run only if the steps before it completed in this cycle
// and no inner test has stopped it (the host enqueues steps ahead; the
// applies cannot check, and compute from stale input).  At the end of a
// cycle: K_gsolve (back-solve, one thread) -> K_gxupd (x += V y) -> the
// residual product -> [M apply: r] -> K_gbeta (||r||, the outer test, the
// next cycle's s).  The cycle-end flag is ChainState::pending, which the host
// reads from its snapshots.

struct GmresChain {
  int n;
  const double* b;
  double* x;
  double* w;
  double* r;
  double* u;
  double* V;     // m+1 vectors, ldv apart
  long long ldv;
  ChainState<double>* st;
  GmresChainExtra* ex;
  double* Hm;    // (m+1) x (m+1), column-major, rotated in place
  double* sv;    // s(0..m)
  double* cs;
  double* sn;
  double* part;
  double* hist;
  int* hist_it;
};

__device__ __forceinline__ bool g_done(const GmresChain& a) {
  return *((volatile const int*)&a.st->done) != 0;
}
// step i's kernels run after steps 0..i-1 of this cycle, until an inner stop
__device__ __forceinline__ bool g_step_live(const GmresChain& a, int i) {
  return !g_done(a) && !*((volatile const int*)&a.st->pending) &&
         *((volatile const int*)&a.ex->ncol) == i;
}

// w = b - A x: Copy(b, w); MltAdd(-1, A, x, 1, w)
struct EpiGResidual {
  const double* b;
  double* w;
  __device__ __forceinline__ void operator()(int i, double t) {
    w[i] = add_rn(__ldg(b + i), mul_rn(-1.0, t));
  }
};
// u = A v
struct EpiGStore {
  double* u;
  __device__ __forceinline__ void operator()(int i, double t) { u[i] = t; }
};

template <typename VT, int PART>
__global__ void __launch_bounds__(CT, PART == 1 ? 1 : chain_spmv_occ<VT>())
    k_gresid(GmresChain a, SellOp<VT> S) {
  __shared__ double s_red[CT / 32];
  pdl_wait();
  pdl_release();
  if (g_done(a)) return;
  EpiGResidual epi{a.b, a.w};
  XLoadLdg<double> xl{a.x};
  if (PART == 0)
    sell_spmv_slices<CT, VT, double, XLoadLdg<double>, EpiGResidual, chain_spmv_unroll<VT>()>(
        S, xl, epi, blockIdx.x, gridDim.x);
  else
    sell_spmv_long<CT, VT, double>(S, xl, epi, s_red, blockIdx.x, gridDim.x);
}

template <typename VT, int PART>
__global__ void __launch_bounds__(CT, PART == 1 ? 1 : chain_spmv_occ<VT>())
    k_gprod(GmresChain a, SellOp<VT> S, int i) {
  __shared__ double s_red[CT / 32];
  pdl_wait();
  pdl_release();
  if (!g_step_live(a, i)) return;
  EpiGStore epi{a.u};
  XLoadLdg<double> xl{a.V + (long long)i * a.ldv};
  if (PART == 0)
    sell_spmv_slices<CT, VT, double, XLoadLdg<double>, EpiGStore, chain_spmv_unroll<VT>()>(
        S, xl, epi, blockIdx.x, gridDim.x);
  else
    sell_spmv_long<CT, VT, double>(S, xl, epi, s_red, blockIdx.x, gridDim.x);
}

// Null initial guess: x = 0, w = b
__global__ void __launch_bounds__(CT, 4) k_gnull(GmresChain a) {
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    a.x[i] = 0.0;
    a.w[i] = __ldg(a.b + i);
  }
}

// beta = ||r||; the first time the Init test (a zero r ends the solve,
// x untouched); then the outer test Finished(beta), and the next cycle's s
__global__ void __launch_bounds__(CT, 4) k_gbeta(GmresChain a, int init) {
  __shared__ double s_red[CT / 32];
  __shared__ double s_out[1];
  pdl_wait();
  pdl_release();
  if (g_done(a)) return;
  double rr = 0.0;
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT) {
    const double ri = a.r[i];
    rr = add_rn(rr, mul_rn(ri, ri));
  }
  double v[1] = {block_sum<CT>(rr, s_red)};
  if (deposit_and_finish<CT, 1>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    ChainState<double>* st = a.st;
    GmresChainExtra* ex = a.ex;
    const double beta = sqrt(s_out[0]);
    if (init) {
      if (beta == 0.0) {
        st->init_failed = 1;
        st->done = 1;
        return;
      }
      st->facteur = 1.0 / beta;
    }
    if (chain_finished_at(st, a.hist, a.hist_it, s_out[0])) {
      st->done = 1;
      return;
    }
    ex->beta = beta;
    for (int k = 0; k < ex->ld; k++) a.sv[k] = 0.0;
    a.sv[0] = beta;
    ex->ncol = 0;
    ex->inner_max = st->nb_iter + ex->m;
    st->pending = 0;
  }
}

// V_0 = r / beta: Copy(r, V_0); Mlt(1/beta, V_0)
__global__ void __launch_bounds__(CT, 4) k_gv0(GmresChain a) {
  pdl_wait();
  pdl_release();
  if (g_done(a)) return;
  const double inv = 1.0 / a.ex->beta;
  for (long long i = (long long)blockIdx.x * CT + threadIdx.x; i < a.n; i += (long long)gridDim.x * CT)
    a.V[i] = mul_rn(a.r[i], inv);
}

// H(0,i) = (V_0, w)
__global__ void __launch_bounds__(CT, 4) k_gdot0(GmresChain a, int i) {
  __shared__ double s_red[CT / 32];
  __shared__ double s_out[1];
  pdl_wait();
  pdl_release();
  if (!g_step_live(a, i)) return;
  double acc = 0.0;
  for (long long e = (long long)blockIdx.x * CT + threadIdx.x; e < a.n; e += (long long)gridDim.x * CT)
    acc = add_rn(acc, mul_rn(a.V[e], a.w[e]));
  double v[1] = {block_sum<CT>(acc, s_red)};
  if (deposit_and_finish<CT, 1>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    a.ex->h = s_out[0];
    a.Hm[0 + (size_t)i * a.ex->ld] = s_out[0];
  }
}

// Add(-H(k,i), V_k, w); then H(k+1,i) = (V_{k+1}, w) (k < i) or, for k = i,
// ||w|| and the step's tail: the rotations of column i (ApplyRot with the
// earlier ones, GenRot, ApplyRot on s), ++iter and the inner test on |s(i+1)|
__global__ void __launch_bounds__(CT, 4) k_gmgs(GmresChain a, int i, int k) {
  __shared__ double s_red[CT / 32];
  __shared__ double s_out[1];
  pdl_wait();
  pdl_release();
  if (!g_step_live(a, i)) return;
  const double mh = -a.ex->h;
  const double* vk = a.V + (long long)k * a.ldv;
  const double* vn = k < i ? a.V + (long long)(k + 1) * a.ldv : nullptr;
  double acc = 0.0;
  for (long long e = (long long)blockIdx.x * CT + threadIdx.x; e < a.n; e += (long long)gridDim.x * CT) {
    double we = a.w[e];
    if (mh != 0.0) {
      we = add_rn(we, mul_rn(mh, vk[e]));
      a.w[e] = we;
    }
    acc = add_rn(acc, vn ? mul_rn(vn[e], we) : mul_rn(we, we));
  }
  double v[1] = {block_sum<CT>(acc, s_red)};
  if (deposit_and_finish<CT, 1>(v, a.part, &a.st->cnt, blockIdx.x, gridDim.x, s_red, s_out) &&
      threadIdx.x == 0) {
    GmresChainExtra* ex = a.ex;
    const int ld = ex->ld;
    if (k < i) {
      ex->h = s_out[0];
      a.Hm[k + 1 + (size_t)i * ld] = s_out[0];
      return;
    }
    ChainState<double>* st = a.st;
    double hi = sqrt(s_out[0]);
    ex->hi = hi;
    double* Hc = a.Hm + (size_t)i * ld;
    for (int q = 0; q < i; q++) apply_rot(Hc[q], Hc[q + 1], a.cs[q], a.sn[q]);
    if (hi != 0.0) {
      gen_rot(Hc[i], hi, a.cs[i], a.sn[i]);
      apply_rot(a.sv[i], a.sv[i + 1], a.cs[i], a.sn[i]);
    }
    st->nb_iter++;
    ex->ncol = i + 1;
    // inner.Finished(|s(i+1)|): its limit is the end of the cycle
    const double reste = st->facteur * fabs(a.sv[i + 1]);
    st->reste = reste;
    if (st->hist_len < st->hist_cap) {
      a.hist[st->hist_len] = reste;
      a.hist_it[st->hist_len] = st->nb_iter;
    }
    st->hist_len++;
    if (reste < st->tol || st->nb_iter >= ex->inner_max) st->pending = 1;
  }
}

// V_{i+1} = w, scaled by 1/||w|| unless ||w|| = 0
__global__ void __launch_bounds__(CT, 4) k_gvnext(GmresChain a, int i) {
  pdl_wait();
  pdl_release();
  if (g_done(a) || *((volatile const int*)&a.ex->ncol) != i + 1) return;
  const double hi = a.ex->hi;
  const double inv = hi != 0.0 ? 1.0 / hi : 1.0;
  double* vn = a.V + (long long)(i + 1) * a.ldv;
  for (long long e = (long long)blockIdx.x * CT + threadIdx.x; e < a.n; e += (long long)gridDim.x * CT)
    vn[e] = hi != 0.0 ? mul_rn(a.w[e], inv) : a.w[e];
}

// Solve(H, s) on the leading ncol x ncol block (the netlib DTRSV column
// sweep the reference's cblas path takes), one thread
__global__ void k_gsolve(GmresChain a) {
  pdl_wait();
  pdl_release();
  if (g_done(a) || threadIdx.x != 0 || blockIdx.x != 0) return;
  const int nc = a.ex->ncol, ld = a.ex->ld;
  double* sv = a.sv;
  for (int j = nc - 1; j >= 0; j--)
    if (sv[j] != 0.0) {
      sv[j] = sv[j] / a.Hm[j + (size_t)j * ld];
      const double t = sv[j];
      for (int q = j - 1; q >= 0; q--) sv[q] = __dsub_rn(sv[q], mul_rn(t, a.Hm[q + (size_t)j * ld]));
    }
}

// x += sum_k s(k) V_k, k in order (Add skipped for s(k) = 0)
__global__ void __launch_bounds__(CT, 4) k_gxupd(GmresChain a) {
  pdl_wait();
  pdl_release();
  if (g_done(a)) return;
  const int nc = a.ex->ncol;
  for (long long e = (long long)blockIdx.x * CT + threadIdx.x; e < a.n; e += (long long)gridDim.x * CT) {
    double xe = a.x[e];
    for (int k = 0; k < nc; k++) {
      const double y = a.sv[k];
      if (y != 0.0) xe = add_rn(xe, mul_rn(y, a.V[(long long)k * a.ldv + e]));
    }
    a.x[e] = xe;
  }
}

// ----------------------------------------------------------------- host driver

// Elementwise passes: at most one resident wave (4 CTAs per SM), threads
// looping over the vector; a partial second wave would leave SMs idle.
static int chain_elem_grid(int n) {
  const int cap = num_sms(current_device()) * 4;
  return std::max(1, std::min((n + CT * 32 - 1) / (CT * 32), cap));
}

// CTAs of a reducing product: one slice per warp up to one resident wave,
// beyond that warps loop over slices: the fewer deposits, the shorter the
// finishing sum.
template <typename VT>
int reducing_slice_grid(const SellOp<VT>& S) {
  if (S.nslice <= 0) return 0;
  const int cap = num_sms(current_device()) * chain_spmv_occ<VT>();
  return std::min((S.nslice + 7) / 8, cap);
}

// Launch of an iteration kernel with programmatic stream serialization: it
// is scheduled while the previous kernel drains and waits (pdl_wait) for its
// results, which hides the launch latency between the passes.
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*k)(KArgs...), int grid, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(CT);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

template <typename T, typename VT>
static int launch_spmv_pair(int mode, const ChainArgs<T>& a, const SellOp<VT>& S,
                            cudaStream_t s) {
  const int g1 = reducing_slice_grid(S);
  const int g2 = (S.nwarp_rows + S.ncta_rows) > 0 ? std::max((S.nwarp_rows + 7) / 8, S.ncta_rows) : 0;
  const int tot = g1 + g2;
  if (tot == 0) return SB2_ERR_NOT_SUPPORTED;
  if (mode == 0) {
    if (g1) SB2_CUDA_TRY(launch_pdl(k_spmv<T, VT, 0, 0>, g1, s, a, S, 0, tot));
    if (g2) SB2_CUDA_TRY(launch_pdl(k_spmv<T, VT, 0, 1>, g2, s, a, S, g1, tot));
  } else {
    if (g1) k_spmv<T, VT, 1, 0><<<g1, CT, 0, s>>>(a, S, 0, tot);
    if (g2) k_spmv<T, VT, 1, 1><<<g2, CT, 0, s>>>(a, S, g1, tot);
  }
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

// Deposit slots one solve needs (two values per CTA of the widest kernel).
template <typename VT>
long long chain_part_slots(const SellOp<VT>& S, int n) {
  const long long g1 = reducing_slice_grid(S);
  const long long g2 = std::max<long long>((S.nwarp_rows + 7) / 8, S.ncta_rows);
  return 2 * std::max<long long>(g1 + g2, chain_elem_grid(n)) + 16;
}

template <typename T, typename VT>
int chain_cg(const SellOp<VT>& S, int n, const T* diag, T* x, const T* b, T* work,
             ChainState<T>* st, T* part, double* hist, int* hist_it, int hist_cap, double tol,
             int max_iter, int init_guess_null, cudaStream_t s, ChainState<T>* out) {
  ChainState<T> init{};
  init.max_iter = max_iter;
  init.tol = tol;
  init.hist_cap = hist_cap;
  init.zc = T(1);
  SB2_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  ChainArgs<T> a{n, b, x, work, work + n, work + 2 * (size_t)n, diag, st, part, hist, hist_it};
  const int ge = chain_elem_grid(n);
  k_norm_b<T><<<ge, CT, 0, s>>>(a);
  if (init_guess_null)
    k_init_null<T><<<ge, CT, 0, s>>>(a);
  else
    SB2_TRY((launch_spmv_pair<T, VT>(1, a, S, s)));
  SB2_CUDA_TRY(cudaGetLastError());
  // iterations in chunks (8, 16, then 32), one chunk always queued behind
  // the one whose state the host waits for
  ChainPipe<T> pipe;
  SB2_TRY(pipe.init());
  ChunkPlanner plan;
  int launched = 0, chunk = 8;
  auto enqueue = [&]() -> int {
    for (int c = 0; c < chunk; c++) {
      SB2_CUDA_TRY(launch_pdl(k_p<T>, ge, s, a));
      SB2_TRY((launch_spmv_pair<T, VT>(0, a, S, s)));
      SB2_CUDA_TRY(launch_pdl(k_x<T>, ge, s, a));
    }
    SB2_CUDA_TRY(cudaGetLastError());
    launched += chunk;
    return pipe.mark(st, launched, s);
  };
  SB2_TRY(enqueue());
  chunk = 16;
  SB2_TRY(enqueue());
  for (;;) {
    ChainState<T> h;
    int at = 0;
    SB2_TRY(pipe.wait(&h, &at));
    if (h.done || at > max_iter + 1) break;
    chunk = plan.next(h.nb_iter, h.reste, tol, launched - at, std::min(chunk * 2, 32));
    SB2_TRY(enqueue());
  }
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  SB2_CUDA_TRY(cudaMemcpy(out, st, sizeof(*out), cudaMemcpyDeviceToHost));
  return SB2_OK;
}

// Cg with a preconditioner applied by `apply(r, z, stream)` (any launches on
// the stream); the same chunked pipeline as chain_cg.  work holds p, q, r and
// z (4 n).
int chain_pcg(const SellOp<double>& S, int n, const PrecondLaunch& apply, double* x,
              const double* b, double* work, ChainState<double>* st, double* part, double* hist,
              int* hist_it, int hist_cap, double tol, int max_iter, int init_guess_null,
              cudaStream_t s, ChainState<double>* out) {
  ChainState<double> init{};
  init.max_iter = max_iter;
  init.tol = tol;
  init.hist_cap = hist_cap;
  init.zc = 1.0;
  SB2_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  double* z = work + 3 * (size_t)n;
  // ChainArgs: r = work, p = work + n, q = work + 2n; no diagonal (the
  // initial (r, z) of k_init_null / the residual product is discarded)
  ChainArgs<double> a{n, b, x, work, work + n, work + 2 * (size_t)n, nullptr, st, part, hist,
                      hist_it};
  const int ge = chain_elem_grid(n);
  k_norm_b<double><<<ge, CT, 0, s>>>(a);
  if (init_guess_null)
    k_init_null<double><<<ge, CT, 0, s>>>(a);
  else
    SB2_TRY((launch_spmv_pair<double, double>(1, a, S, s)));
  SB2_CUDA_TRY(cudaGetLastError());
  // An iteration here costs a preconditioner apply, whose launches cannot
  // see the stop flag: no chunk is queued ahead of the one the host waits
  // for (an apply after the stop would be wasted), and the chunk is sized
  // from the residual's decay so that it ends near the stop.
  ChainPipe<double> pipe;
  SB2_TRY(pipe.init());
  ChunkPlanner plan;
  int launched = 0, chunk = 4;
  for (;;) {
    for (int c = 0; c < chunk; c++) {
      SB2_TRY(apply(a.r, z, s));
      SB2_CUDA_TRY(launch_pdl(k_pc_rz<double>, ge, s, a, (const double*)z));
      SB2_CUDA_TRY(launch_pdl(k_pc_p<double>, ge, s, a, (const double*)z));
      SB2_TRY((launch_spmv_pair<double, double>(0, a, S, s)));
      SB2_CUDA_TRY(launch_pdl(k_pc_x<double>, ge, s, a));
    }
    SB2_CUDA_TRY(cudaGetLastError());
    launched += chunk;
    SB2_TRY(pipe.mark(st, launched, s));
    ChainState<double> h;
    int at = 0;
    SB2_TRY(pipe.wait(&h, &at));
    if (h.done || at > max_iter + 1) break;
    chunk = plan.next(h.nb_iter, h.reste, tol, 0, std::min(chunk * 2, 16), 1, 16);
  }
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  SB2_CUDA_TRY(cudaMemcpy(out, st, sizeof(*out), cudaMemcpyDeviceToHost));
  return SB2_OK;
}

// The two kernels of a BiCgStab product (slices, long rows), one deposit array.
template <typename VT>
static int launch_b_spmv(int mode, const BicgChain<double>& a, const SellOp<VT>& S,
                         cudaStream_t s) {
  const int g1 = reducing_slice_grid(S);
  const int g2 = (S.nwarp_rows + S.ncta_rows) > 0 ? std::max((S.nwarp_rows + 7) / 8, S.ncta_rows) : 0;
  const int tot = g1 + g2;
  if (tot == 0) return SB2_ERR_NOT_SUPPORTED;
  if (mode == 0) {
    if (g1) SB2_CUDA_TRY(launch_pdl(k_b_spmv<double, VT, 0, 0>, g1, s, a, S, 0, tot));
    if (g2) SB2_CUDA_TRY(launch_pdl(k_b_spmv<double, VT, 0, 1>, g2, s, a, S, g1, tot));
  } else {
    if (g1) SB2_CUDA_TRY(launch_pdl(k_b_spmv<double, VT, 1, 0>, g1, s, a, S, 0, tot));
    if (g2) SB2_CUDA_TRY(launch_pdl(k_b_spmv<double, VT, 1, 1>, g2, s, a, S, g1, tot));
  }
  return SB2_OK;
}

// BiCgStab with a preconditioner's own launches (SOR, ILUT, Jacobi) or none
// (apply.M == NULL: identity), as a device-resident chain.  work: 8n doubles
// (r, rt, p, phat, v, s, shat, t).
// As in chain_pcg, no chunk is queued ahead of the one the host waits for.
int chain_pbicgstab(const SellOp<double>& S, int n, const PrecondLaunch& apply, double* x,
                    const double* b, double* work, ChainState<double>* st, double* part,
                    double* hist, int* hist_it, int hist_cap, double tol, int max_iter,
                    int init_guess_null, cudaStream_t s, ChainState<double>* out) {
  ChainState<double> init{};
  init.max_iter = max_iter;
  init.tol = tol;
  init.hist_cap = hist_cap;
  init.zc = 1.0;
  SB2_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  const size_t nn = (size_t)n;
  BicgChain<double> bc{n, x, work, work + nn, work + 2 * nn, work + 3 * nn, work + 4 * nn,
                       work + 5 * nn, work + 6 * nn, work + 7 * nn, st, part, hist, hist_it};
  // identity (no preconditioner object): phat is p and shat is s, no applies
  const bool ident = apply.M == nullptr;
  if (ident) {
    bc.phat = bc.p;
    bc.shat = bc.s;
  }
  // the start: ||b||, r = b (- A x) with Finished(||r||) and rho = (r, r) = (rt, r)
  ChainArgs<double> a{n, b, x, bc.r, bc.p, bc.v, nullptr, st, part, hist, hist_it};
  const int ge = chain_elem_grid(n);
  k_norm_b<double><<<ge, CT, 0, s>>>(a);
  if (init_guess_null)
    k_init_null<double><<<ge, CT, 0, s>>>(a);
  else
    SB2_TRY((launch_spmv_pair<double, double>(1, a, S, s)));
  k_b_copy<double><<<ge, CT, 0, s>>>(bc);
  SB2_CUDA_TRY(cudaGetLastError());
  ChainPipe<double> pipe;
  SB2_TRY(pipe.init());
  ChunkPlanner plan;
  int launched = 0, chunk = 2;
  for (;;) {
    for (int c = 0; c < chunk; c++) {
      SB2_CUDA_TRY(launch_pdl(k_b_p<double>, ge, s, bc));
      if (!ident) SB2_TRY(apply(bc.p, bc.phat, s));
      SB2_TRY(launch_b_spmv<double>(0, bc, S, s));
      SB2_CUDA_TRY(launch_pdl(k_b_s<double>, ge, s, bc));
      if (!ident) SB2_TRY(apply(bc.s, bc.shat, s));
      SB2_TRY(launch_b_spmv<double>(1, bc, S, s));
      SB2_CUDA_TRY(launch_pdl(k_b_xr<double>, ge, s, bc));
    }
    SB2_CUDA_TRY(cudaGetLastError());
    launched += chunk;
    SB2_TRY(pipe.mark(st, launched, s));
    ChainState<double> h;
    int at = 0;
    SB2_TRY(pipe.wait(&h, &at));
    if (h.done || 2 * at > max_iter + 2) break;
    // two iterations of the counter a loop
    chunk = (plan.next(h.nb_iter, h.reste, tol, 0, std::min(chunk * 4, 16), 2, 16) + 1) / 2;
  }
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  SB2_CUDA_TRY(cudaMemcpy(out, st, sizeof(*out), cudaMemcpyDeviceToHost));
  return SB2_OK;
}

// The residual product w = b - A x, or step i's product u = A V_i.
template <typename VT>
static int launch_gspmv(bool resid, const GmresChain& a, const SellOp<VT>& S, int i,
                        cudaStream_t s) {
  const int g1 = reducing_slice_grid(S);
  const int g2 = (S.nwarp_rows + S.ncta_rows) > 0 ? std::max((S.nwarp_rows + 7) / 8, S.ncta_rows) : 0;
  if (g1 + g2 == 0) return SB2_ERR_NOT_SUPPORTED;
  if (resid) {
    if (g1) SB2_CUDA_TRY(launch_pdl(k_gresid<VT, 0>, g1, s, a, S));
    if (g2) SB2_CUDA_TRY(launch_pdl(k_gresid<VT, 1>, g2, s, a, S));
  } else {
    if (g1) SB2_CUDA_TRY(launch_pdl(k_gprod<VT, 0>, g1, s, a, S, i));
    if (g2) SB2_CUDA_TRY(launch_pdl(k_gprod<VT, 1>, g2, s, a, S, i));
  }
  return SB2_OK;
}

// Gmres(m) with a preconditioner's own launches (SOR, ILUT), as a
// device-resident chain.  work: (m+4) vectors `ldv` apart (w, r, u, V_0..V_m);
// hbuf: (m+1)^2 + 3(m+1) doubles (H, s, cos, sin).  The host enqueues the
// steps of a cycle in chunks sized from the residual's decay and reads the
// state behind each chunk; once an inner test has stopped the cycle
// (ChainState::pending), it enqueues the cycle's end: the back-solve, the
// update of x, the new residual and the outer test.
int chain_pgmres(const SellOp<double>& S, int n, int m, const PrecondLaunch& apply, double* x,
                 const double* b, double* work, long long ldv, ChainState<double>* st,
                 GmresChainExtra* ex, double* hbuf, double* part, double* hist, int* hist_it,
                 int hist_cap, double tol, int max_iter, int init_guess_null, cudaStream_t s,
                 ChainState<double>* out) {
  const int ld = m + 1;
  ChainState<double> init{};
  init.max_iter = max_iter;
  init.tol = tol;
  init.hist_cap = hist_cap;
  GmresChainExtra ei{};
  ei.m = m;
  ei.ld = ld;
  SB2_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  SB2_CUDA_TRY(cudaMemcpyAsync(ex, &ei, sizeof(ei), cudaMemcpyHostToDevice, s));
  SB2_CUDA_TRY(cudaMemsetAsync(hbuf, 0, sizeof(double) * ((size_t)ld * ld + 3 * (size_t)ld), s));
  GmresChain a{n, b, x, work, work + ldv, work + 2 * ldv, work + 3 * ldv, ldv, st, ex, hbuf,
               hbuf + (size_t)ld * ld, hbuf + (size_t)ld * ld + ld, hbuf + (size_t)ld * ld + 2 * ld,
               part, hist, hist_it};
  const int ge = chain_elem_grid(n);
  if (init_guess_null) {
    k_gnull<<<ge, CT, 0, s>>>(a);
    SB2_CUDA_TRY(cudaGetLastError());
  } else {
    SB2_TRY(launch_gspmv<double>(true, a, S, 0, s));
  }
  SB2_TRY(apply(a.w, a.r, s));
  SB2_CUDA_TRY(launch_pdl(k_gbeta, ge, s, a, 1));
  ChainPipe<double> pipe;
  SB2_TRY(pipe.init());
  int launched = 0, at = 0;
  ChainState<double> h;
  SB2_TRY(pipe.mark(st, ++launched, s));
  SB2_TRY(pipe.wait(&h, &at));
  ChunkPlanner plan;
  int chunk = std::min(4, m);
  for (int cycles = 0; !h.done && cycles <= max_iter; cycles++) {
    SB2_CUDA_TRY(launch_pdl(k_gv0, ge, s, a));
    int step = 0;
    for (;;) {
      for (int c = 0; c < chunk && step < m; c++, step++) {
        SB2_TRY(launch_gspmv<double>(false, a, S, step, s));
        SB2_TRY(apply(a.u, a.w, s));
        SB2_CUDA_TRY(launch_pdl(k_gdot0, ge, s, a, step));
        for (int k = 0; k <= step; k++) SB2_CUDA_TRY(launch_pdl(k_gmgs, ge, s, a, step, k));
        SB2_CUDA_TRY(launch_pdl(k_gvnext, ge, s, a, step));
      }
      SB2_TRY(pipe.mark(st, ++launched, s));
      SB2_TRY(pipe.wait(&h, &at));
      if (h.done || h.pending || step >= m) break;
      chunk = plan.next(h.nb_iter, h.reste, tol, 0, std::min(chunk * 2, m), 1, m - step);
    }
    if (h.done) break;
    // the cycle's end: Solve(H, s), x += V s, r = M^{-1}(b - A x), Finished(||r||)
    SB2_CUDA_TRY(launch_pdl(k_gsolve, 1, s, a));
    SB2_CUDA_TRY(launch_pdl(k_gxupd, ge, s, a));
    SB2_TRY(launch_gspmv<double>(true, a, S, 0, s));
    SB2_TRY(apply(a.w, a.r, s));
    SB2_CUDA_TRY(launch_pdl(k_gbeta, ge, s, a, 0));
    SB2_TRY(pipe.mark(st, ++launched, s));
    SB2_TRY(pipe.wait(&h, &at));
  }
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  SB2_CUDA_TRY(cudaMemcpy(out, st, sizeof(*out), cudaMemcpyDeviceToHost));
  return SB2_OK;
}

template <typename T, typename VT>
int chain_ru_resume(const SellOp<VT>& S, int n, const T* diag, T* x, T* r, T* work,
                    ChainState<T>* st, T* part, cudaStream_t s);

// Reliable-update CG iterations: the caller's loop applies the corrections.
// ru_start: state for an initial residual r already in place (x = 0);
template <typename T, typename VT>
int chain_ru_start(const SellOp<VT>& S, int n, const T* diag, T* x, T* r, T* work,
                   ChainState<T>* st, T* part, double facteur, double tol, double delta,
                   int max_iter, cudaStream_t s) {
  ChainState<T> init{};
  init.max_iter = max_iter;
  init.tol = tol;
  init.delta = delta;
  init.facteur = facteur;
  init.pending = 1;
  init.zc = T(1);
  SB2_CUDA_TRY(cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  SB2_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(T) * (size_t)n, s));
  return chain_ru_resume<T, VT>(S, n, diag, x, r, work, st, part, s);
}

template <typename T, typename VT>
int chain_ru_resume(const SellOp<VT>& S, int n, const T* diag, T* x, T* r, T* work,
                    ChainState<T>* st, T* part, cudaStream_t s) {
  ChainArgs<T> a{n, nullptr, x, r, work, work + n, diag, st, part, nullptr, nullptr};
  k_rho_ru<T><<<chain_elem_grid(n), CT, 0, s>>>(a);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

// ru_enqueue: `chunk` iterations queued on s (no wait; the caller's
// ChainPipe reads the state behind them).
template <typename T, typename VT>
int chain_ru_enqueue(const SellOp<VT>& S, int n, const T* diag, T* x, T* r, T* work,
                     ChainState<T>* st, T* part, int chunk, cudaStream_t s) {
  ChainArgs<T> a{n, nullptr, x, r, work, work + n, diag, st, part, nullptr, nullptr};
  const int ge = chain_elem_grid(n);
  for (int c = 0; c < chunk; c++) {
    SB2_CUDA_TRY(launch_pdl(k_p<T>, ge, s, a));
    SB2_TRY((launch_spmv_pair<T, VT>(0, a, S, s)));
    SB2_CUDA_TRY(launch_pdl(k_x_ru<T>, ge, s, a));
  }
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

template int chain_ru_start<float, float>(const SellOp<float>&, int, const float*, float*, float*,
                                          float*, ChainState<float>*, float*, double, double,
                                          double, int, cudaStream_t);
template int chain_ru_resume<float, float>(const SellOp<float>&, int, const float*, float*,
                                           float*, float*, ChainState<float>*, float*,
                                           cudaStream_t);
template int chain_ru_enqueue<float, float>(const SellOp<float>&, int, const float*, float*,
                                            float*, float*, ChainState<float>*, float*, int,
                                            cudaStream_t);

template int reducing_slice_grid<double>(const SellOp<double>&);
template int reducing_slice_grid<float>(const SellOp<float>&);
template long long chain_part_slots<double>(const SellOp<double>&, int);
template long long chain_part_slots<float>(const SellOp<float>&, int);
template int chain_cg<double, double>(const SellOp<double>&, int, const double*, double*,
                                      const double*, double*, ChainState<double>*, double*,
                                      double*, int*, int, double, int, int, cudaStream_t,
                                      ChainState<double>*);
template int chain_cg<float, float>(const SellOp<float>&, int, const float*, float*,
                                    const float*, float*, ChainState<float>*, float*, double*,
                                    int*, int, double, int, int, cudaStream_t,
                                    ChainState<float>*);

}  // namespace sb2
