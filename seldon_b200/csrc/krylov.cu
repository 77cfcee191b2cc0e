// Seldon's Krylov drivers on the device.
//
// Identity and Jacobi preconditioning run as ONE cooperative persistent
// kernel per solve: the whole iteration loop, the Iteration<double> stopping
// rule, the breakdown tests and (GMRES) the Givens rotations and Hessenberg
// back-solve stay on the GPU; the only host round trip is the final result.
// Each iteration fuses the SpMV with the dot product that follows it and the
// vector updates with the next residual norm; grid-wide reductions are
// deterministic (fixed CTA order).
//
// SOR and ILUT preconditioning (level-scheduled sweeps, many dependent
// launches) of Cg, BiCgStab and Gmres run as device-resident chains around the
// sweeps (chain.cu); the other drivers with them, and every driver when those
// chains are switched off, go through a host-driven driver over the same
// device kernels, one operation at a time, in the reference's order.
//
// References: Cg.cxx:45-116, BiCgStab.cxx:43-145, Gmres.cxx:44-183,
// Cgs.cxx:45-132, TfQmr.cxx:44-243, MinRes.cxx:46-153, Gcr.cxx:45-141,
// BiCgStabl.cxx:43-180, QCgs.cxx:46-165, BiCg.cxx:46-134, CoCg.cxx:45-116,
// Cgne.cxx:40-127, BiCgcr.cxx:44-118, Lsqr.cxx:40-135, QmrSym.cxx:41-165,
// Symmlq.cxx:45-161, Iterative.cxx:235-354.
#include <cooperative_groups.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <vector>

#include "chain.cuh"
#include "givens.cuh"
#include "persist.cuh"
#include "sell.cuh"

namespace sb2 {

int precond_apply(const sb2_precond* M, bool trans, const double* r, double* z,
                  cudaStream_t s);

constexpr int NT = kSpmvThreads;

// ----------------------------------------------------------------- common

struct OpArgs {
  const int* ptr;
  const int* ind;
  const double* val;
  const int* blk;
  const unsigned char* kind;
  int nblk;
  int n;
  const double* diag;  // nullptr: identity preconditioner, else Jacobi
  SellOp<double> sell; // binned SELL-32 (nslice < 0: use the row blocks)
};

struct IterArgs {
  double tol;
  int max_iter;
  int restart;
  int init_guess_null;
};

#define SB2_SHARED_DECL                     \
  __shared__ double s_prod[kNnzCap];        \
  __shared__ double s_red[NT / 32];         \
  __shared__ double s_vals[kMaxRed]

__device__ __forceinline__ double precond_val(const double* diag, int i, double r) {
  return diag ? __ddiv_rn(r, diag[i]) : r;  // Jacobi z_i = r_i / A(i,i)
}

// W consecutive entries of a vector (W = 1, or 2 read and written as one
// 16-byte access)
template <int W>
struct Ents {
  double v[W];
};

template <int W>
__device__ __forceinline__ Ents<W> ldw(const double* p, long long i) {
  Ents<W> o;
  if constexpr (W == 2) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p + i));
    o.v[0] = a.x;
    o.v[1] = a.y;
  } else {
    o.v[0] = __ldcg(p + i);
  }
  return o;
}

template <int W>
__device__ __forceinline__ void stw(double* p, long long i, const Ents<W>& a) {
  if constexpr (W == 2) *reinterpret_cast<double2*>(p + i) = make_double2(a.v[0], a.v[1]);
  else p[i] = a.v[0];
}

// Jacobi (or identity) on W entries
template <int W>
__device__ __forceinline__ Ents<W> precond_w(const double* diag, long long i, Ents<W> r) {
  if (diag) {
    Ents<W> d;
    if constexpr (W == 2) {
      const double2 a = __ldg(reinterpret_cast<const double2*>(diag + i));
      d.v[0] = a.x;
      d.v[1] = a.y;
    } else {
      d.v[0] = __ldg(diag + i);
    }
#pragma unroll
    for (int j = 0; j < W; j++) r.v[j] = __ddiv_rn(r.v[j], d.v[j]);
  }
  return r;
}

// A grid-stride vector pass over entries [0, n).  With `paired` (every vector
// the pass touches 16-byte aligned) each step takes two consecutive entries
// with 16-byte loads and stores, which keeps twice the bytes in flight per
// register, and the odd last entry follows alone; otherwise one entry a step.
// f(std::integral_constant<int, W>, i) handles entries i .. i + W - 1.
template <class F>
__device__ __forceinline__ void vec_pass(long long n, long long gt, long long gs, bool paired,
                                         F&& f) {
  if (paired) {
    const long long n2 = n >> 1;
#pragma unroll 2
    for (long long k = gt; k < n2; k += gs) f(std::integral_constant<int, 2>(), 2 * k);
    if ((n & 1) && gt == 0) f(std::integral_constant<int, 1>(), n - 1);
  } else {
#pragma unroll 4
    for (long long i = gt; i < n; i += gs) f(std::integral_constant<int, 1>(), i);
  }
}

__device__ __forceinline__ bool al16(const void* p) {
  return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

__device__ __forceinline__ void hist_push(const History& h, int* len, int it, double res) {
  if (*len < h.cap) {
    h.res[*len] = res;
    h.it[*len] = it;
  }
  (*len)++;
}

__device__ __forceinline__ void write_out(SolveOut* out, int nb_iter, int max_iter, int fail,
                                          double facteur, double last, int hist_len) {
  out->nb_iter = nb_iter;
  // Iteration::ErrorCode (Iterative.cxx:344-354)
  out->error_code = (nb_iter >= max_iter) ? -2 : fail;
  out->init_failed = 0;
  out->facteur_reste = facteur;
  out->last_residual = last;
  out->hist_len = hist_len;
}

// epilogue: y_r = t; acc += w_r * t   (SpMV fused with the dot that follows)
struct EpiStoreDot {
  double* y;
  const double* w;
  double acc;
  __device__ __forceinline__ void operator()(int r, double t) {
    y[r] = t;
    acc = add_rn(acc, mul_rn(__ldcg(w + r), t));
  }
  // rows r..r+3 of one lane (r % 4 == 0) with 32-byte accesses
  __device__ __forceinline__ void quad(int r, const double* t) {
    if (!al16(y + r) || !al16(w + r)) {
      for (int j = 0; j < 4; j++) (*this)(r + j, t[j]);
      return;
    }
    double wv[4];
    const double tv[4] = {t[0], t[1], t[2], t[3]};
    vld4_cg(w + r, wv);
    vst4(y + r, tv);
#pragma unroll
    for (int j = 0; j < 4; j++) acc = add_rn(acc, mul_rn(wv[j], t[j]));
  }
};

// epilogue: r_r = b_r - t (MltAdd(-1, A, x, 1, r) after Copy(b, r)), then the
// preconditioned z_r; accumulate r.r and r.z.
struct EpiResidual {
  const double* b;
  double* r;
  const double* diag;
  double rr, rz;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double v = add_rn(__ldg(b + i), -t);
    r[i] = v;
    const double z = precond_val(diag, i, v);
    rr = add_rn(rr, mul_rn(v, v));
    rz = add_rn(rz, mul_rn(v, z));
  }
};

template <class Epi>
__device__ __forceinline__ void spmv_phase(const OpArgs& A, const double* x, Epi& epi,
                                           double* s_prod, double* s_red) {
  XLoadCa<double> xl{x};
  if (A.sell.nslice >= 0) {
    sell_spmv<NT, double, double>(A.sell, xl, epi, s_red, blockIdx.x, gridDim.x);
    return;
  }
  for (int b = blockIdx.x; b < A.nblk; b += gridDim.x)
    spmv_row_block<NT, double, double>(A.ptr, A.ind, A.val, A.blk[b], A.blk[b + 1], A.kind[b],
                                       xl, epi, s_prod, s_red);
}

// ----------------------------------------------------------------- CG

struct CgVecs {
  const double* b;
  double *x, *r, *p, *q;
};

__global__ void __launch_bounds__(NT, 4) cg_fused_kernel(OpArgs A, CgVecs v, IterArgs it,
                                                      Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  // iter.Init(b): facteur_reste = 1/||b|| (Iterative.cxx:235-249)
  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // r = b - A x (or x = 0, r = b), with ||r||^2 and r.z
  double rr = 0.0, rz = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      const double bi = __ldg(v.b + i);
      v.x[i] = 0.0;
      v.r[i] = bi;
      const double z = precond_val(A.diag, (int)i, bi);
      rr = add_rn(rr, mul_rn(bi, bi));
      rz = add_rn(rz, mul_rn(bi, z));
    }
  } else {
    EpiResidual epi{v.b, v.r, A.diag, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    rr = epi.rr;
    rz = epi.rz;
  }
  rr = block_sum<NT>(rr, s_red);
  rz = block_sum<NT>(rz, s_red);
  if (tid == 0) { s_vals[0] = rr; s_vals[1] = rz; }
  if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
  rr = s_vals[0];
  double rho = s_vals[1], rho_1 = 1.0;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    // while (!iter.Finished(r))
    reste = facteur * sqrt(rr);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    // z = M^{-1} r; rho = (r, z): already reduced with the norm
    if (rho == 0.0) { fail = 1; break; }
    // p = z (first) | p = beta*p + z: Mlt(beta, p); Add(1, z, p)
    {
      const bool first = nb_iter == 0;
      const double beta = first ? 0.0 : rho / rho_1;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> z = precond_w<W>(A.diag, i, ldw<W>(v.r, i));
        if (first) {
          stw<W>(v.p, i, z);
        } else {
          Ents<W> pi = ldw<W>(v.p, i);
#pragma unroll
          for (int j = 0; j < W; j++) pi.v[j] = add_rn(mul_rn(pi.v[j], beta), z.v[j]);
          stw<W>(v.p, i, pi);
        }
      });
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // q = A p fused with delta = (p, q)
    EpiStoreDot epi{v.q, v.p, 0.0};
    spmv_phase(A, v.p, epi, s_prod, s_red);
    double d = block_sum<NT>(epi.acc, s_red);
    if (tid == 0) s_vals[0] = d;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    const double delta = s_vals[0];
    if (delta == 0.0) { fail = 2; break; }
    const double alpha = rho / delta;
    // Add(alpha, p, x); Add(-alpha, q, r); then ||r||^2 and (r, z) for the next test
    rr = 0.0;
    rz = 0.0;
    vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      if (alpha != 0.0) {
        Ents<W> xi = ldw<W>(v.x, i);
        const Ents<W> pi = ldw<W>(v.p, i);
#pragma unroll
        for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(alpha, pi.v[j]));
        stw<W>(v.x, i, xi);
      }
      Ents<W> ri = ldw<W>(v.r, i);
      if (-alpha != 0.0) {
        const Ents<W> qi = ldw<W>(v.q, i);
#pragma unroll
        for (int j = 0; j < W; j++) ri.v[j] = add_rn(ri.v[j], mul_rn(-alpha, qi.v[j]));
        stw<W>(v.r, i, ri);
      }
      const Ents<W> z = precond_w<W>(A.diag, i, ri);
#pragma unroll
      for (int j = 0; j < W; j++) {
        rr = add_rn(rr, mul_rn(ri.v[j], ri.v[j]));
        rz = add_rn(rz, mul_rn(ri.v[j], z.v[j]));
      }
    });
    rr = block_sum<NT>(rr, s_red);
    rz = block_sum<NT>(rz, s_red);
    if (tid == 0) { s_vals[0] = rr; s_vals[1] = rz; }
    if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
    rr = s_vals[0];
    rho_1 = rho;
    rho = s_vals[1];
    nb_iter++;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- BiCGSTAB

struct BicgVecs {
  const double* b;
  double *x, *r, *rt, *p, *ph, *v, *s, *sh, *t;
};

// epilogue: y_r = t; acc0 += w0_r t; with `self`, acc1 += t t
struct EpiStoreDot2 {
  double* y;
  const double* w0;
  bool self;
  double acc0, acc1;
  __device__ __forceinline__ void operator()(int r, double t) {
    y[r] = t;
    acc0 = add_rn(acc0, mul_rn(__ldcg(w0 + r), t));
    if (self) acc1 = add_rn(acc1, mul_rn(t, t));
  }
  __device__ __forceinline__ void quad(int r, const double* t) {
    if (!al16(y + r) || !al16(w0 + r)) {
      for (int j = 0; j < 4; j++) (*this)(r + j, t[j]);
      return;
    }
    double wv[4];
    const double tv[4] = {t[0], t[1], t[2], t[3]};
    vld4_cg(w0 + r, wv);
    vst4(y + r, tv);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      acc0 = add_rn(acc0, mul_rn(wv[j], t[j]));
      if (self) acc1 = add_rn(acc1, mul_rn(t[j], t[j]));
    }
  }
};

__global__ void __launch_bounds__(NT, 4) bicgstab_fused_kernel(OpArgs A, BicgVecs v, IterArgs it,
                                                            Persist P, History H,
                                                            SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // r = b - A x (or x = 0); rtilde = r; ||r||^2 and (rtilde, r)
  double rr = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      const double bi = __ldg(v.b + i);
      v.x[i] = 0.0;
      v.r[i] = bi;
      v.rt[i] = bi;
      rr = add_rn(rr, mul_rn(bi, bi));
    }
  } else {
    EpiResidual epi{v.b, v.r, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    rr = epi.rr;
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    for (long long i = gt; i < n; i += gs) v.rt[i] = __ldcg(v.r + i);
  }
  rr = block_sum<NT>(rr, s_red);
  if (tid == 0) { s_vals[0] = rr; s_vals[1] = rr; }
  if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
  rr = s_vals[0];
  double rho_1 = s_vals[1];  // (rtilde, r) with rtilde = r
  double rho_2 = 0.0, alpha = 0.0, omega = 0.0;
  const bool jac = (A.diag != nullptr);
  double* ph = jac ? v.ph : v.p;  // identity: phat aliases p, shat aliases s
  double* sh = jac ? v.sh : v.s;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * sqrt(rr);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    if (rho_1 == 0.0) { fail = 1; break; }
    if (nb_iter == 0) {
      // Copy(r, p); phat = M^{-1} p
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> pi = ldw<W>(v.r, i);
        stw<W>(v.p, i, pi);
        if (jac) stw<W>(ph, i, precond_w<W>(A.diag, i, pi));
      });
    } else {
      if (omega == 0.0) { fail = 2; break; }
      const double beta = (rho_1 / rho_2) * (alpha / omega);
      // Add(-omega, v, p); Mlt(beta, p); Add(1, r, p); phat = M^{-1} p
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        Ents<W> pi = ldw<W>(v.p, i);
        const Ents<W> vi = ldw<W>(v.v, i), ri = ldw<W>(v.r, i);
#pragma unroll
        for (int j = 0; j < W; j++) {
          pi.v[j] = add_rn(pi.v[j], mul_rn(-omega, vi.v[j]));
          pi.v[j] = add_rn(mul_rn(pi.v[j], beta), ri.v[j]);
        }
        stw<W>(v.p, i, pi);
        if (jac) stw<W>(ph, i, precond_w<W>(A.diag, i, pi));
      });
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // v = A phat, sigma = (rtilde, v)
    EpiStoreDot2 e1{v.v, v.rt, false, 0.0, 0.0};
    spmv_phase(A, ph, e1, s_prod, s_red);
    double d = block_sum<NT>(e1.acc0, s_red);
    if (tid == 0) s_vals[0] = d;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    const double sigma = s_vals[0];
    if (sigma == 0.0) { fail = 3; break; }
    alpha = rho_1 / sigma;
    // Copy(r, s); Add(-alpha, v, s); shat = M^{-1} s; ||s||^2
    double ss = 0.0;
    vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      Ents<W> si = ldw<W>(v.r, i);
      if (-alpha != 0.0) {
        const Ents<W> vi = ldw<W>(v.v, i);
#pragma unroll
        for (int j = 0; j < W; j++) si.v[j] = add_rn(si.v[j], mul_rn(-alpha, vi.v[j]));
      }
      stw<W>(v.s, i, si);
      if (jac) stw<W>(sh, i, precond_w<W>(A.diag, i, si));
#pragma unroll
      for (int j = 0; j < W; j++) ss = add_rn(ss, mul_rn(si.v[j], si.v[j]));
    });
    ss = block_sum<NT>(ss, s_red);
    if (tid == 0) s_vals[0] = ss;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    nb_iter++;
    reste = facteur * sqrt(s_vals[0]);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) {
      // Add(alpha, phat, x)
      if (alpha != 0.0)
        for (long long i = gt; i < n; i += gs)
          v.x[i] = add_rn(__ldcg(v.x + i), mul_rn(alpha, __ldcg(ph + i)));
      break;
    }
    // t = A shat; omega = (t, s) / (t, t)
    EpiStoreDot2 e2{v.t, v.s, true, 0.0, 0.0};
    spmv_phase(A, sh, e2, s_prod, s_red);
    const double ts = block_sum<NT>(e2.acc0, s_red);
    const double tt = block_sum<NT>(e2.acc1, s_red);
    if (tid == 0) { s_vals[0] = ts; s_vals[1] = tt; }
    if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
    omega = s_vals[0] / s_vals[1];
    // Add(alpha, phat, x); Add(omega, shat, x); Copy(s, r); Add(-omega, t, r)
    rr = 0.0;
    double rtr = 0.0;
    vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      Ents<W> xi = ldw<W>(v.x, i);
      if (alpha != 0.0) {
        const Ents<W> pi = ldw<W>(ph, i);
#pragma unroll
        for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(alpha, pi.v[j]));
      }
      if (omega != 0.0) {
        const Ents<W> si = ldw<W>(sh, i);
#pragma unroll
        for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(omega, si.v[j]));
      }
      stw<W>(v.x, i, xi);
      Ents<W> ri = ldw<W>(v.s, i);
      if (-omega != 0.0) {
        const Ents<W> ti = ldw<W>(v.t, i);
#pragma unroll
        for (int j = 0; j < W; j++) ri.v[j] = add_rn(ri.v[j], mul_rn(-omega, ti.v[j]));
      }
      stw<W>(v.r, i, ri);
      const Ents<W> rti = ldw<W>(v.rt, i);
#pragma unroll
      for (int j = 0; j < W; j++) {
        rr = add_rn(rr, mul_rn(ri.v[j], ri.v[j]));
        rtr = add_rn(rtr, mul_rn(rti.v[j], ri.v[j]));
      }
    });
    rr = block_sum<NT>(rr, s_red);
    rtr = block_sum<NT>(rtr, s_red);
    if (tid == 0) { s_vals[0] = rr; s_vals[1] = rtr; }
    if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
    rr = s_vals[0];
    rho_2 = rho_1;
    rho_1 = s_vals[1];
    nb_iter++;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- CGS

struct CgsVecs {
  const double* b;
  double *x, *r, *rt, *u, *p, *ph, *q, *vh, *uh;
};

// epilogue of qhat = A uhat: Add(-alpha, qhat, r), then ||r||^2 and
// (rtilde, r) for the next test and rho (qhat itself is not kept)
struct EpiResidUpdate {
  double* r;
  const double* rt;
  double malpha;
  double rr, rtr;
  __device__ __forceinline__ void operator()(int i, double t) {
    double ri = __ldcg(r + i);
    if (malpha != 0.0) {
      ri = add_rn(ri, mul_rn(malpha, t));
      r[i] = ri;
    }
    rr = add_rn(rr, mul_rn(ri, ri));
    rtr = add_rn(rtr, mul_rn(__ldcg(rt + i), ri));
  }
  __device__ __forceinline__ void quad(int i, const double* t) {
    if (!al16(r + i) || !al16(rt + i)) {
      for (int j = 0; j < 4; j++) (*this)(i + j, t[j]);
      return;
    }
    double rv[4], tv[4];
    vld4_cg(r + i, rv);
    vld4_cg(rt + i, tv);
    if (malpha != 0.0) {
#pragma unroll
      for (int j = 0; j < 4; j++) rv[j] = add_rn(rv[j], mul_rn(malpha, t[j]));
      vst4(r + i, rv);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      rr = add_rn(rr, mul_rn(rv[j], rv[j]));
      rtr = add_rn(rtr, mul_rn(tv[j], rv[j]));
    }
  }
};

// Cgs (Cgs.cxx:45-132): four grid barriers per loop, two products; the
// second product is fused with the residual update and both reductions.
__global__ void __launch_bounds__(NT, 4) cgs_fused_kernel(OpArgs A, CgsVecs v, IterArgs it,
                                                       Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // r = b - A x (or x = 0, r = b); rtilde = r; ||r||^2 (= (rtilde, r))
  double rr = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      const double bi = __ldg(v.b + i);
      v.x[i] = 0.0;
      v.r[i] = bi;
      v.rt[i] = bi;
      rr = add_rn(rr, mul_rn(bi, bi));
    }
  } else {
    EpiResidual epi{v.b, v.r, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    rr = epi.rr;
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    for (long long i = gt; i < n; i += gs) v.rt[i] = __ldcg(v.r + i);
  }
  rr = block_sum<NT>(rr, s_red);
  if (tid == 0) s_vals[0] = rr;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  rr = s_vals[0];
  double rho_1 = rr, rho_2 = 0.0;
  const bool jac = (A.diag != nullptr);
  double* ph = jac ? v.ph : v.p;  // identity: phat aliases p, uhat aliases u
  double* uh = jac ? v.uh : v.u;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * sqrt(rr);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    if (rho_1 == 0.0) { fail = 1; break; }
    if (nb_iter == 0) {
      // Copy(r, u); Copy(u, p); phat = M^{-1} p
      vec_pass(n, gt, gs, true, [&](auto w, long long i) {
        constexpr int W = decltype(w)::value;
        const Ents<W> ri = ldw<W>(v.r, i);
        stw<W>(v.u, i, ri);
        stw<W>(v.p, i, ri);
        if (jac) stw<W>(ph, i, precond_w<W>(A.diag, i, ri));
      });
    } else {
      // Copy(r, u); Add(beta, q, u); Mlt(beta, p); Add(1, q, p); Mlt(beta, p);
      // Add(1, u, p); phat = M^{-1} p
      const double beta = rho_1 / rho_2;
      vec_pass(n, gt, gs, true, [&](auto w, long long i) {
        constexpr int W = decltype(w)::value;
        const Ents<W> qi = ldw<W>(v.q, i);
        Ents<W> ui = ldw<W>(v.r, i), pi = ldw<W>(v.p, i);
#pragma unroll
        for (int j = 0; j < W; j++) {
          if (beta != 0.0) ui.v[j] = add_rn(ui.v[j], mul_rn(beta, qi.v[j]));
          pi.v[j] = add_rn(mul_rn(add_rn(mul_rn(pi.v[j], beta), qi.v[j]), beta), ui.v[j]);
        }
        stw<W>(v.u, i, ui);
        stw<W>(v.p, i, pi);
        if (jac) stw<W>(ph, i, precond_w<W>(A.diag, i, pi));
      });
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // vhat = A phat fused with delta = (rtilde, vhat)
    EpiStoreDot e1{v.vh, v.rt, 0.0};
    spmv_phase(A, ph, e1, s_prod, s_red);
    const double d = block_sum<NT>(e1.acc, s_red);
    if (tid == 0) s_vals[0] = d;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    nb_iter++;
    const double delta = s_vals[0];
    if (delta == 0.0) { fail = 2; break; }
    const double alpha = rho_1 / delta;
    // Copy(u, q); Add(-alpha, vhat, q); Add(1, q, u); uhat = M^{-1} u;
    // Add(alpha, uhat, x)
    vec_pass(n, gt, gs, al16(v.x), [&](auto w, long long i) {
      constexpr int W = decltype(w)::value;
      Ents<W> ui = ldw<W>(v.u, i), qi = ui, xi = ldw<W>(v.x, i);
      const Ents<W> vhi = ldw<W>(v.vh, i);
#pragma unroll
      for (int j = 0; j < W; j++) {
        if (-alpha != 0.0) qi.v[j] = add_rn(qi.v[j], mul_rn(-alpha, vhi.v[j]));
        ui.v[j] = add_rn(ui.v[j], qi.v[j]);
      }
      stw<W>(v.q, i, qi);
      stw<W>(v.u, i, ui);
      const Ents<W> uhi = precond_w<W>(A.diag, i, ui);
      if (jac) stw<W>(uh, i, uhi);
      if (alpha != 0.0) {
#pragma unroll
        for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(alpha, uhi.v[j]));
        stw<W>(v.x, i, xi);
      }
    });
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // qhat = A uhat fused with Add(-alpha, qhat, r), ||r||^2 and (rtilde, r)
    EpiResidUpdate e2{v.r, v.rt, -alpha, 0.0, 0.0};
    spmv_phase(A, uh, e2, s_prod, s_red);
    rr = block_sum<NT>(e2.rr, s_red);
    const double rtr = block_sum<NT>(e2.rtr, s_red);
    if (tid == 0) { s_vals[0] = rr; s_vals[1] = rtr; }
    if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
    rr = s_vals[0];
    rho_2 = rho_1;
    rho_1 = s_vals[1];
    nb_iter++;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- TFQMR

struct TfqmrVecs {
  const double* b;
  double *x, *rt, *w, *y1, *y0, *v, *g, *h, *d;
};

// epilogue of the initial residual: r0 = M^{-1}(b - A x); w = y1 = rtilde =
// r0; d = 0; accumulate ||r0||^2
struct EpiTfqmrInit {
  const double* b;
  const double* diag;
  double *w, *y1, *rt, *d;
  double rr;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double r0 = precond_val(diag, i, add_rn(__ldg(b + i), -t));
    w[i] = r0;
    y1[i] = r0;
    rt[i] = r0;
    d[i] = 0.0;
    rr = add_rn(rr, mul_rn(r0, r0));
  }
};

// epilogue of v = M^{-1} A y1 at the start: g = v; accumulate (rtilde, v)
struct EpiTfqmrFirstV {
  const double* diag;
  const double* rt;
  double *v, *g;
  double sigma;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double vi = precond_val(diag, i, t);
    v[i] = vi;
    g[i] = vi;
    sigma = add_rn(sigma, mul_rn(__ldcg(rt + i), vi));
  }
};

// epilogue of h = M^{-1} A y0 (the end of the first half step and the start
// of the second): Add(eta, d, x); Copy(h, g) is implied (g is overwritten
// before its next read, so h is read in its place); Add(-alpha, h, w);
// Mlt(c1, d); Add(1, y0, d); accumulate ||w||^2 and (rtilde, w)
struct EpiTfqmrHalf {
  const double* diag;
  const double *rt, *y0;
  double *h, *x, *w, *d;
  double eta, malpha, c1;
  double ww, rtw;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double hi = precond_val(diag, i, t);
    h[i] = hi;
    double di = __ldcg(d + i);
    if (eta != 0.0) x[i] = add_rn(__ldcg(x + i), mul_rn(eta, di));
    double wi = __ldcg(w + i);
    if (malpha != 0.0) {
      wi = add_rn(wi, mul_rn(malpha, hi));
      w[i] = wi;
    }
    d[i] = add_rn(mul_rn(di, c1), __ldcg(y0 + i));
    ww = add_rn(ww, mul_rn(wi, wi));
    rtw = add_rn(rtw, mul_rn(__ldcg(rt + i), wi));
  }
  __device__ __forceinline__ void quad(int i, const double* t) {
    if (!al16(x + i) || (diag && !al16(diag + i))) {
      for (int j = 0; j < 4; j++) (*this)(i + j, t[j]);
      return;
    }
    double hv[4] = {t[0], t[1], t[2], t[3]}, dv[4], xv[4], wv[4], yv[4], rv[4];
    if (diag) {
      double gv[4];
      vld4_ldg(diag + i, gv);
#pragma unroll
      for (int j = 0; j < 4; j++) hv[j] = __ddiv_rn(t[j], gv[j]);
    }
    vld4_cg(d + i, dv);
    vld4_cg(w + i, wv);
    vld4_cg(y0 + i, yv);
    vld4_cg(rt + i, rv);
    vst4(h + i, hv);
    if (eta != 0.0) {
      vld4_cg(x + i, xv);
#pragma unroll
      for (int j = 0; j < 4; j++) xv[j] = add_rn(xv[j], mul_rn(eta, dv[j]));
      vst4(x + i, xv);
    }
    if (malpha != 0.0) {
#pragma unroll
      for (int j = 0; j < 4; j++) wv[j] = add_rn(wv[j], mul_rn(malpha, hv[j]));
      vst4(w + i, wv);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) dv[j] = add_rn(mul_rn(dv[j], c1), yv[j]);
    vst4(d + i, dv);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      ww = add_rn(ww, mul_rn(wv[j], wv[j]));
      rtw = add_rn(rtw, mul_rn(rv[j], wv[j]));
    }
  }
};

// epilogue of g = M^{-1} A y1: Mlt(beta^2, v); Add(beta, h, v); Add(1, g, v);
// accumulate (rtilde, v) for the next loop's sigma
struct EpiTfqmrNextV {
  const double* diag;
  const double *rt, *h;
  double *g, *v;
  double beta, bb;
  double sigma;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double gi = precond_val(diag, i, t);
    g[i] = gi;
    double vi = mul_rn(__ldcg(v + i), bb);
    if (beta != 0.0) vi = add_rn(vi, mul_rn(beta, __ldcg(h + i)));
    vi = add_rn(vi, gi);
    v[i] = vi;
    sigma = add_rn(sigma, mul_rn(__ldcg(rt + i), vi));
  }
  __device__ __forceinline__ void quad(int i, const double* t) {
    if (diag && !al16(diag + i)) {
      for (int j = 0; j < 4; j++) (*this)(i + j, t[j]);
      return;
    }
    double gv[4] = {t[0], t[1], t[2], t[3]}, vv[4], hv[4], rv[4];
    if (diag) {
      double dv[4];
      vld4_ldg(diag + i, dv);
#pragma unroll
      for (int j = 0; j < 4; j++) gv[j] = __ddiv_rn(t[j], dv[j]);
    }
    vld4_cg(v + i, vv);
    vld4_cg(h + i, hv);
    vld4_cg(rt + i, rv);
    vst4(g + i, gv);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      vv[j] = mul_rn(vv[j], bb);
      if (beta != 0.0) vv[j] = add_rn(vv[j], mul_rn(beta, hv[j]));
      vv[j] = add_rn(vv[j], gv[j]);
    }
    vst4(v + i, vv);
#pragma unroll
    for (int j = 0; j < 4; j++) sigma = add_rn(sigma, mul_rn(rv[j], vv[j]));
  }
};

// TfQmr (TfQmr.cxx:44-243), left preconditioned: four grid barriers and two
// products per loop of two half steps.  The vector work of each half step
// rides in the epilogue of the product that follows it.
__global__ void __launch_bounds__(NT, 4) tfqmr_fused_kernel(OpArgs A, TfqmrVecs v, IterArgs it,
                                                         Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  // 1.-2. r0 = M^{-1}(b - A x) (or x = 0); w = y1 = rtilde = r0; d = 0
  double rr = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      v.x[i] = 0.0;
      const double r0 = precond_val(A.diag, (int)i, __ldg(v.b + i));
      v.w[i] = r0;
      v.y1[i] = r0;
      v.rt[i] = r0;
      v.d[i] = 0.0;
      rr = add_rn(rr, mul_rn(r0, r0));
    }
  } else {
    EpiTfqmrInit epi{v.b, A.diag, v.w, v.y1, v.rt, v.d, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    rr = epi.rr;
  }
  rr = block_sum<NT>(rr, s_red);
  if (tid == 0) s_vals[0] = rr;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  // iter.Init(r0); tau = Norm2(r0); rho = (rtilde, r0) with rtilde = r0
  const double tau0 = sqrt(s_vals[0]);
  if (tau0 == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / tau0;
  double tau = tau0, rho = s_vals[0], theta = 0.0, eta = 0.0;
  // 3. g = v = M^{-1} A y1, with the first sigma = (rtilde, v)
  {
    EpiTfqmrFirstV epi{A.diag, v.rt, v.v, v.g, 0.0};
    spmv_phase(A, v.y1, epi, s_prod, s_red);
    const double sg = block_sum<NT>(epi.sigma, s_red);
    if (tid == 0) s_vals[0] = sg;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  }
  double sigma = s_vals[0];

  int nb_iter = 0, fail = 0;
  double reste = 0.0;
  bool done = false;
  for (;;) {
    // 9.-11. alpha = rho / sigma; y0 = y1 - alpha v; the breakdown tests of
    // the first half step come before any vector that outlives the loop
    if (sigma == 0.0) { fail = 1; break; }
    const double alpha = rho / sigma;
    if (alpha == 0.0) { fail = 2; break; }
    if (tau == 0.0) { fail = 3; break; }
    // first half: Add(-alpha, g, w); Mlt(theta^2 eta / alpha, d); Add(1, y1, d)
    {
      const double c1 = theta * theta * eta / alpha;
      double ww = 0.0;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> y1i = ldw<W>(v.y1, i), vi = ldw<W>(v.v, i), gi = ldw<W>(v.g, i);
        Ents<W> y0i, wi = ldw<W>(v.w, i), di = ldw<W>(v.d, i);
#pragma unroll
        for (int j = 0; j < W; j++) {
          y0i.v[j] = add_rn(y1i.v[j], mul_rn(-alpha, vi.v[j]));
          wi.v[j] = add_rn(wi.v[j], mul_rn(-alpha, gi.v[j]));
          di.v[j] = add_rn(mul_rn(di.v[j], c1), y1i.v[j]);
          ww = add_rn(ww, mul_rn(wi.v[j], wi.v[j]));
        }
        stw<W>(v.y0, i, y0i);
        stw<W>(v.w, i, wi);
        stw<W>(v.d, i, di);
      });
      ww = block_sum<NT>(ww, s_red);
      if (tid == 0) s_vals[0] = ww;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    // 14.-21. theta, c, tau, eta; x += eta d; Finished(kappa)
    theta = sqrt(s_vals[0]) / tau;
    double c = 1.0 / sqrt(add_rn(1.0, mul_rn(theta, theta)));
    tau = tau * c * theta;
    eta = c * c * alpha;
    double kappa = tau * sqrt(2. * (nb_iter + 1));
    reste = facteur * kappa;
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) {
      if (eta != 0.0)
        for (long long i = gt; i < n; i += gs)
          v.x[i] = add_rn(__ldcg(v.x + i), mul_rn(eta, __ldcg(v.d + i)));
      break;
    }
    nb_iter++;
    // h = M^{-1} A y0 with the first half's x update and the second half's
    // w and d updates
    {
      EpiTfqmrHalf epi{A.diag, v.rt, v.y0, v.h, v.x, v.w, v.d,
                        eta, -alpha, theta * theta * eta / alpha, 0.0, 0.0};
      spmv_phase(A, v.y0, epi, s_prod, s_red);
      const double ww = block_sum<NT>(epi.ww, s_red);
      const double rtw = block_sum<NT>(epi.rtw, s_red);
      if (tid == 0) { s_vals[0] = ww; s_vals[1] = rtw; }
      if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
    }
    if (tau == 0.0) { fail = 4; break; }
    theta = sqrt(s_vals[0]) / tau;
    c = 1.0 / sqrt(add_rn(1.0, mul_rn(theta, theta)));
    tau = tau * c * theta;
    eta = c * c * alpha;
    kappa = tau * sqrt(2. * (nb_iter + 1) + 1.);
    reste = facteur * kappa;
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    const double rho0 = rho;
    rho = s_vals[1];
    // Add(eta, d, x) comes before the test and the last breakdown
    done = (reste < it.tol || nb_iter >= it.max_iter);
    if (!done && rho0 == 0.0) fail = 5;
    const double beta = (done || fail) ? 0.0 : rho / rho0;
    // x += eta d; 24. y1 = w + beta y0
    const bool next = !done && !fail;
    vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      if (eta != 0.0) {
        Ents<W> xi = ldw<W>(v.x, i);
        const Ents<W> di = ldw<W>(v.d, i);
#pragma unroll
        for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(eta, di.v[j]));
        stw<W>(v.x, i, xi);
      }
      if (next) {
        Ents<W> yi = ldw<W>(v.w, i);
        if (beta != 0.0) {
          const Ents<W> y0i = ldw<W>(v.y0, i);
#pragma unroll
          for (int j = 0; j < W; j++) yi.v[j] = add_rn(yi.v[j], mul_rn(beta, y0i.v[j]));
        }
        stw<W>(v.y1, i, yi);
      }
    });
    if (done || fail) break;
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // 25.-26. g = M^{-1} A y1; v = beta^2 v + beta h + g; next sigma
    {
      EpiTfqmrNextV epi{A.diag, v.rt, v.h, v.g, v.v, beta, beta * beta, 0.0};
      spmv_phase(A, v.y1, epi, s_prod, s_red);
      const double sg = block_sum<NT>(epi.sigma, s_red);
      if (tid == 0) s_vals[0] = sg;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    sigma = s_vals[0];
    nb_iter++;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- MINRES

struct MinresVecs {
  const double* b;
  double *x, *r, *z;
  double *u, *u_old, *v, *v_old, *w, *w_old, *w_oold;  // initial roles
};

// MinRes (MinRes.cxx:46-153): per iteration the product fused with
// (r, u), one pass forming r and z with (r, z), and one pass forming w, x
// and the next v and u -- three grid barriers.  Seldon's copies between the
// old and new vectors (Copy(w_old, w_oold), Copy(v, v_old), ...) are role
// rotations of the buffers: every thread swaps the same register pointers.  The
// scalar recurrences are rounded step by step (mul_rn / add_rn), as the
// reference's separately rounded products and sums.
__global__ void __launch_bounds__(NT, 4) minres_fused_kernel(OpArgs A, MinresVecs v, IterArgs it,
                                                          Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  // iter.Init(b)
  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // r = b - A x (or x = 0, r = b); z = M^{-1} r; dp = (r, z)
  double dp = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      const double bi = __ldg(v.b + i);
      v.x[i] = 0.0;
      v.r[i] = bi;
      dp = add_rn(dp, mul_rn(bi, precond_val(A.diag, (int)i, bi)));
    }
  } else {
    EpiResidual epi{v.b, v.r, A.diag, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    dp = epi.rz;
  }
  dp = block_sum<NT>(dp, s_red);
  if (tid == 0) s_vals[0] = dp;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  double beta = sqrt(s_vals[0]);
  double eta = beta;
  {
    // v = r / beta, u = z / beta (Copy then Mlt(ibeta, .)); the old vectors
    // and the w's start at zero
    const double ibeta = 1.0 / beta;
    vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      const Ents<W> ri = ldw<W>(v.r, i);
      const Ents<W> zi = precond_w<W>(A.diag, i, ri);
      Ents<W> a, c, zero;
#pragma unroll
      for (int j = 0; j < W; j++) {
        a.v[j] = mul_rn(ri.v[j], ibeta);
        c.v[j] = mul_rn(zi.v[j], ibeta);
        zero.v[j] = 0.0;
      }
      stw<W>(v.v, i, a);
      stw<W>(v.u, i, c);
      stw<W>(v.u_old, i, zero);
      stw<W>(v.v_old, i, zero);
      stw<W>(v.w, i, zero);
      stw<W>(v.w_old, i, zero);
      stw<W>(v.w_oold, i, zero);
    });
  }
  if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  double c = 1.0, s = 0.0, cold = 1.0, sold = 0.0;
  double np = normb;  // Norm2(b)
  double *u = v.u, *u_old = v.u_old, *vv = v.v, *v_old = v.v_old;
  double *w = v.w, *w_old = v.w_old, *w_oold = v.w_oold;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * np;
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    // r = A u fused with alpha = (r, u)
    {
      EpiStoreDot epi{v.r, u, 0.0};
      spmv_phase(A, u, epi, s_prod, s_red);
      const double a = block_sum<NT>(epi.acc, s_red);
      if (tid == 0) s_vals[0] = a;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    const double alpha = s_vals[0];
    // z = M^{-1} r; Add(-alpha, v, r); Add(-alpha, u, z); Add(-beta, v_old, r);
    // Add(-beta, u_old, z); dp = (r, z)
    {
      double d = 0.0;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        Ents<W> ri = ldw<W>(v.r, i);
        Ents<W> zi = precond_w<W>(A.diag, i, ri);
        if (-alpha != 0.0) {
          const Ents<W> a = ldw<W>(vv, i), b = ldw<W>(u, i);
#pragma unroll
          for (int j = 0; j < W; j++) {
            ri.v[j] = add_rn(ri.v[j], mul_rn(-alpha, a.v[j]));
            zi.v[j] = add_rn(zi.v[j], mul_rn(-alpha, b.v[j]));
          }
        }
        if (-beta != 0.0) {
          const Ents<W> a = ldw<W>(v_old, i), b = ldw<W>(u_old, i);
#pragma unroll
          for (int j = 0; j < W; j++) {
            ri.v[j] = add_rn(ri.v[j], mul_rn(-beta, a.v[j]));
            zi.v[j] = add_rn(zi.v[j], mul_rn(-beta, b.v[j]));
          }
        }
        stw<W>(v.r, i, ri);
        stw<W>(v.z, i, zi);
#pragma unroll
        for (int j = 0; j < W; j++) d = add_rn(d, mul_rn(ri.v[j], zi.v[j]));
      });
      d = block_sum<NT>(d, s_red);
      if (tid == 0) s_vals[0] = d;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    const double beta_old = beta;
    beta = sqrt(s_vals[0]);
    // QR factorization
    const double coold = cold, soold = sold;
    cold = c;
    sold = s;
    const double rho0 = add_rn(mul_rn(cold, alpha), -mul_rn(mul_rn(coold, sold), beta_old));
    const double rho1 = sqrt(add_rn(mul_rn(rho0, rho0), mul_rn(beta, beta)));
    const double rho2 = add_rn(mul_rn(sold, alpha), mul_rn(mul_rn(coold, cold), beta_old));
    const double rho3 = mul_rn(soold, beta_old);
    if (rho1 == 0.0) { fail = 1; break; }
    c = rho0 / rho1;
    s = beta / rho1;
    // w_oold <- w_old, w_old <- w, w <- (u - rho2 w_old - rho3 w_oold) / rho1,
    // written over the old w_oold; x += c eta w; then v_old <- v, u_old <- u,
    // v <- r / beta, u <- z / beta, written over the old v_old and u_old
    const double inv_rho1 = 1. / rho1;
    const double ceta = mul_rn(c, eta);
    eta = mul_rn(-s, eta);
    const bool last = (beta == 0.0);
    const double ibeta = last ? 0.0 : 1.0 / beta;
    vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      Ents<W> wn = ldw<W>(u, i);
      if (-rho2 != 0.0) {
        const Ents<W> a = ldw<W>(w, i);
#pragma unroll
        for (int j = 0; j < W; j++) wn.v[j] = add_rn(wn.v[j], mul_rn(-rho2, a.v[j]));
      }
      if (-rho3 != 0.0) {
        const Ents<W> a = ldw<W>(w_old, i);
#pragma unroll
        for (int j = 0; j < W; j++) wn.v[j] = add_rn(wn.v[j], mul_rn(-rho3, a.v[j]));
      }
#pragma unroll
      for (int j = 0; j < W; j++) wn.v[j] = mul_rn(wn.v[j], inv_rho1);
      stw<W>(w_oold, i, wn);
      if (ceta != 0.0) {
        Ents<W> xi = ldw<W>(v.x, i);
#pragma unroll
        for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(ceta, wn.v[j]));
        stw<W>(v.x, i, xi);
      }
      if (!last) {
        Ents<W> ri = ldw<W>(v.r, i), zi = ldw<W>(v.z, i);
#pragma unroll
        for (int j = 0; j < W; j++) {
          ri.v[j] = mul_rn(ri.v[j], ibeta);
          zi.v[j] = mul_rn(zi.v[j], ibeta);
        }
        stw<W>(v_old, i, ri);
        stw<W>(u_old, i, zi);
      }
    });
    if (last) { fail = 2; break; }
    {
      double* t = w_oold;  // the new w sits where w_oold was
      w_oold = w_old;
      w_old = w;
      w = t;
    }
    {
      double* t = u;  // the new u and v sit where u_old and v_old were
      u = u_old;
      u_old = t;
      t = vv;
      vv = v_old;
      v_old = t;
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    np = mul_rn(np, fabs(s));
    nb_iter++;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- GCR

// Largest restart the persistent Gcr takes: a step reduces ceil(m / 2)
// projections in one barrier, at most kMaxRed.
constexpr int kGcrMaxRestart = 2 * kMaxRed;

struct GcrVecs {
  const double* b;
  double *x, *r;
  double* P;  // p_0 .. p_m, `ld` apart
  double* W;  // w_0 .. w_m
  long long ld;
};

// epilogue of the initial residual: r = M^{-1}(b - A x), with ||r||^2
struct EpiPrecResidual {
  const double* b;
  double* r;
  const double* diag;
  double rr;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double ri = precond_val(diag, i, add_rn(__ldg(b + i), -t));
    r[i] = ri;
    rr = add_rn(rr, mul_rn(ri, ri));
  }
};

// epilogue of w_j = M^{-1} A p_j: (w_j, w_j) and (w_j, r)
struct EpiGcrW {
  double* w;
  const double* r;
  const double* diag;
  double ww, wr;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double wi = precond_val(diag, i, t);
    w[i] = wi;
    ww = add_rn(ww, mul_rn(wi, wi));
    wr = add_rn(wr, mul_rn(wi, __ldcg(r + i)));
  }
};

// epilogue of q = M^{-1} A r: the projections (w_k, q), k < nd; q itself is
// never stored
struct EpiGcrQ {
  const double* W;
  long long ld;
  const double* diag;
  int nd;
  double acc[kMaxRed];
  __device__ __forceinline__ void operator()(int i, double t) {
    const double qi = precond_val(diag, i, t);
#pragma unroll
    for (int k = 0; k < kMaxRed; k++)
      if (k < nd) acc[k] = add_rn(acc[k], mul_rn(__ldcg(W + k * ld + i), qi));
  }
};

// Gcr(m) (Gcr.cxx:45-141), left preconditioned.  An inner step takes two
// products and four grid barriers: w_j = M^{-1} A p_j with (w_j, w_j) and
// (w_j, r); the x and r updates with ||r||^2; q = M^{-1} A r with the j + 1
// projections (w_i, q); then p_{j+1} = r + sum_i delta_i p_i.  The outer and
// the inner Iteration test the same residual, and both tests are logged, as
// the reference's two Finished() calls are.  Where the reference never
// returns -- a cycle whose inner loop takes no step, which every later cycle
// then repeats -- the solve stops after that cycle.
__global__ void __launch_bounds__(NT, 4) gcr_fused_kernel(OpArgs A, GcrVecs v, IterArgs it,
                                                       Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  __shared__ double s_beta[kGcrMaxRestart + 1];
  __shared__ double s_delta[kMaxRed];
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const int m = it.restart;
  const long long ld = v.ld;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  // outer.Init(b)
  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // u = b - A x (or x = 0, u = b); r = M^{-1} u; ||r||^2
  double rr = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      v.x[i] = 0.0;
      const double ri = precond_val(A.diag, (int)i, __ldg(v.b + i));
      v.r[i] = ri;
      rr = add_rn(rr, mul_rn(ri, ri));
    }
  } else {
    EpiPrecResidual epi{v.b, v.r, A.diag, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    rr = epi.rr;
  }
  rr = block_sum<NT>(rr, s_red);
  if (tid == 0) s_vals[0] = rr;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  rr = s_vals[0];
  double normr = sqrt(rr);

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    // outer.Finished(r)
    reste = facteur * sqrt(rr);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    const int inner_max = nb_iter + m;
    // Copy(r, p_0); Mlt(1 / normr, p_0)
    {
      const double inv = 1.0 / normr;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int Wd = decltype(wc)::value;
        Ents<Wd> ri = ldw<Wd>(v.r, i);
#pragma unroll
        for (int k = 0; k < Wd; k++) ri.v[k] = mul_rn(ri.v[k], inv);
        stw<Wd>(v.P, i, ri);
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    }
    int j = 0;
    for (;;) {
      // inner.Finished(r)
      reste = facteur * sqrt(rr);
      if (lead) hist_push(H, &hlen, nb_iter, reste);
      if (reste < it.tol || nb_iter >= inner_max) break;
      double* pj = v.P + (long long)j * ld;
      double* wj = v.W + (long long)j * ld;
      // w_j = M^{-1} A p_j; beta_j = (w_j, w_j); (w_j, r)
      {
        EpiGcrW epi{wj, v.r, A.diag, 0.0, 0.0};
        spmv_phase(A, pj, epi, s_prod, s_red);
        const double ww = block_sum<NT>(epi.ww, s_red);
        const double wr = block_sum<NT>(epi.wr, s_red);
        if (tid == 0) { s_vals[0] = ww; s_vals[1] = wr; }
        if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
      }
      const double beta_j = s_vals[0];
      if (beta_j == 0.0) { fail = 1; break; }
      if (tid == 0) s_beta[j] = beta_j;
      const double alpha = s_vals[1] / beta_j;
      // Add(alpha, p_j, x); Add(-alpha, w_j, r); ||r||^2
      {
        double a = 0.0;
        vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
          constexpr int Wd = decltype(wc)::value;
          if (alpha != 0.0) {
            Ents<Wd> xi = ldw<Wd>(v.x, i);
            const Ents<Wd> pi = ldw<Wd>(pj, i);
#pragma unroll
            for (int k = 0; k < Wd; k++) xi.v[k] = add_rn(xi.v[k], mul_rn(alpha, pi.v[k]));
            stw<Wd>(v.x, i, xi);
          }
          Ents<Wd> ri = ldw<Wd>(v.r, i);
          if (-alpha != 0.0) {
            const Ents<Wd> wi = ldw<Wd>(wj, i);
#pragma unroll
            for (int k = 0; k < Wd; k++) ri.v[k] = add_rn(ri.v[k], mul_rn(-alpha, wi.v[k]));
            stw<Wd>(v.r, i, ri);
          }
#pragma unroll
          for (int k = 0; k < Wd; k++) a = add_rn(a, mul_rn(ri.v[k], ri.v[k]));
        });
        a = block_sum<NT>(a, s_red);
        if (tid == 0) s_vals[0] = a;
        if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
        rr = s_vals[0];
      }
      nb_iter++;
      // q = M^{-1} A r; delta_i = -(w_i, q) / beta_i
      const int nd = j + 1;
      {
        EpiGcrQ epi{v.W, ld, A.diag, nd, {}};
        spmv_phase(A, v.r, epi, s_prod, s_red);
#pragma unroll
        for (int k = 0; k < kMaxRed; k++)
          if (k < nd) {
            const double d = block_sum<NT>(epi.acc[k], s_red);
            if (tid == 0) s_vals[k] = d;
          }
        if (!grid_sync<NT>(P, epoch, nd, s_vals, s_red)) return;
      }
      if (tid < nd) s_delta[tid] = -s_vals[tid] / s_beta[tid];
      __syncthreads();
      // Copy(r, p_{j+1}); Add(delta_i, p_i, p_{j+1}) for i = 0..j
      {
        double* pn = v.P + (long long)(j + 1) * ld;
        vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
          constexpr int Wd = decltype(wc)::value;
          Ents<Wd> pv = ldw<Wd>(v.r, i);
          for (int k = 0; k < nd; k++) {
            const double dk = s_delta[k];
            if (dk != 0.0) {
              const Ents<Wd> pk = ldw<Wd>(v.P + (long long)k * ld, i);
#pragma unroll
              for (int q = 0; q < Wd; q++) pv.v[q] = add_rn(pv.v[q], mul_rn(dk, pk.v[q]));
            }
          }
          stw<Wd>(pn, i, pv);
        });
        if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
      }
      nb_iter++;
      j++;
    }
    if (j == 0) break;  // the reference would repeat this cycle for ever
    normr = sqrt(rr);
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- BICGSTAB(L)

// Largest l of the persistent BiCgStabl: tau and the gammas live in shared
// memory, (l + 1)^2 + 3(l + 1) doubles.
constexpr int kBicglMax = 16;

struct BicglVecs {
  const double* b;
  double *x, *rt, *q;  // r0 (the shadow residual), M^{-1} of a product's operand
  double *R, *U;       // r_0 .. r_l and u_0 .. u_l, `ld` apart
  long long ld;
};

// epilogue of the initial residual: r_0 = b - A x, r0 = r_0, ||r_0||^2
struct EpiBiclInit {
  const double* b;
  double *r, *rt;
  double rr;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double v = add_rn(__ldg(b + i), -t);
    r[i] = v;
    rt[i] = v;
    rr = add_rn(rr, mul_rn(v, v));
  }
};

// BiCgStabl(l) (BiCgStabl.cxx:43-180), l = the restart parameter, right
// preconditioning.  A cycle: l BiCG steps of two products and four grid
// barriers each (the u and r updates ride the passes between products,
// (u_{j+1}, r0) and (r_{j+1}, r0) the products' epilogues), then the MR
// part's modified Gram-Schmidt over r_1 .. r_l (each axpy fused with the
// next dot), the small triangular solves for the gammas (every CTA the same,
// thread 0 into shared memory), and one update pass that also reduces the
// next test's ||r_0||^2 and (r_0, r0).  A breakdown ends the BiCG part only,
// as in the reference; tau and the gammas carry over between cycles.  x is
// mapped back by M^{-1} at the end.  Where the reference can repeat a cycle
// for ever (one that counts no iteration) the solve stops after it.
__global__ void __launch_bounds__(NT, 4) bicgstabl_fused_kernel(OpArgs A, BicglVecs v,
                                                             IterArgs it, Persist P, History H,
                                                             SolveOut* out) {
  SB2_SHARED_DECL;
  __shared__ double s_tau[(kBicglMax + 1) * (kBicglMax + 1)];
  __shared__ double s_g[kBicglMax + 1], s_gp[kBicglMax + 1], s_gt[kBicglMax + 1];
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const int l = it.restart;
  const int L1 = l + 1;
  const long long ld = v.ld;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  const bool jac = (A.diag != nullptr);
  unsigned epoch = 0;
  int hlen = 0;
  auto Rv = [&](int i) { return v.R + (long long)i * ld; };
  auto Uv = [&](int i) { return v.U + (long long)i * ld; };

  for (int k = tid; k < L1 * L1; k += NT) s_tau[k] = 0.0;
  for (int k = tid; k < L1; k += NT) s_g[k] = s_gp[k] = s_gt[k] = 0.0;
  // r_1..r_l and u_0..u_l start at zero; x = 0 for a null guess; ||b||
  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
    if (it.init_guess_null) v.x[i] = 0.0;
    for (int k = 0; k <= l; k++) {
      if (k > 0) Rv(k)[i] = 0.0;
      Uv(k)[i] = 0.0;
    }
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  // iter.Init(b) comes after r_0 in the reference; r_0 is not observable
  // when it fails, x (zeroed for a null guess) is
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;
  // r_0 = b - A x (or b); r0 = r_0
  double rr = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      const double bi = __ldg(v.b + i);
      Rv(0)[i] = bi;
      v.rt[i] = bi;
      rr = add_rn(rr, mul_rn(bi, bi));
    }
  } else {
    EpiBiclInit epi{v.b, Rv(0), v.rt, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    rr = epi.rr;
  }
  rr = block_sum<NT>(rr, s_red);
  if (tid == 0) s_vals[0] = rr;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  rr = s_vals[0];
  double rho_next = rr;  // (r_0, r0) with r0 = r_0
  double rho_0 = 1.0, alpha = 0.0, omega = 1.0;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * sqrt(rr);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    const int start = nb_iter;
    rho_0 = mul_rn(rho_0, -omega);
    // Bi-CG part
    for (int j = 0; j < l; j++) {
      const double rho_1 = rho_next;  // (r_j, r0)
      if (rho_0 == 0.0) { fail = 1; break; }
      const double beta = mul_rn(alpha, rho_1 / rho_0);
      rho_0 = rho_1;
      // u_i = r_i - beta u_i (Mlt(-beta, u_i); Add(1, r_i, u_i)), i <= j;
      // q = M^{-1} u_j
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        for (int k = 0; k <= j; k++) {
          Ents<W> u = ldw<W>(Uv(k), i);
          const Ents<W> r = ldw<W>(Rv(k), i);
#pragma unroll
          for (int e = 0; e < W; e++) u.v[e] = add_rn(mul_rn(u.v[e], -beta), r.v[e]);
          stw<W>(Uv(k), i, u);
          if (jac && k == j) stw<W>(v.q, i, precond_w<W>(A.diag, i, u));
        }
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
      // u_{j+1} = A q; sigma = (u_{j+1}, r0)
      {
        EpiStoreDot epi{Uv(j + 1), v.rt, 0.0};
        spmv_phase(A, jac ? v.q : Uv(j), epi, s_prod, s_red);
        const double d = block_sum<NT>(epi.acc, s_red);
        if (tid == 0) s_vals[0] = d;
        if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
      }
      nb_iter++;
      const double sigma = s_vals[0];
      if (sigma == 0.0) { fail = 2; break; }
      alpha = rho_1 / sigma;
      // Add(alpha, u_0, x); Add(-alpha, u_{i+1}, r_i), i <= j; q = M^{-1} r_j
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        if (alpha != 0.0) {
          Ents<W> xi = ldw<W>(v.x, i);
          const Ents<W> u0 = ldw<W>(Uv(0), i);
#pragma unroll
          for (int e = 0; e < W; e++) xi.v[e] = add_rn(xi.v[e], mul_rn(alpha, u0.v[e]));
          stw<W>(v.x, i, xi);
        }
        for (int k = 0; k <= j; k++) {
          Ents<W> r = ldw<W>(Rv(k), i);
          if (-alpha != 0.0) {
            const Ents<W> u = ldw<W>(Uv(k + 1), i);
#pragma unroll
            for (int e = 0; e < W; e++) r.v[e] = add_rn(r.v[e], mul_rn(-alpha, u.v[e]));
            stw<W>(Rv(k), i, r);
          }
          if (jac && k == j) stw<W>(v.q, i, precond_w<W>(A.diag, i, r));
        }
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
      // r_{j+1} = A q; the next step's rho = (r_{j+1}, r0)
      {
        EpiStoreDot epi{Rv(j + 1), v.rt, 0.0};
        spmv_phase(A, jac ? v.q : Rv(j), epi, s_prod, s_red);
        const double d = block_sum<NT>(epi.acc, s_red);
        if (tid == 0) s_vals[0] = d;
        if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
      }
      rho_next = s_vals[0];
      nb_iter++;
    }
    // MR part: for j = 1..l, tau(i, j) = (r_j, r_i) / gamma_i and
    // r_j -= tau(i, j) r_i for i < j with gamma_i != 0, each axpy fused with
    // the next dot; gamma_j = (r_j, r_j), gamma'_j = (r_0, r_j) / gamma_j
    for (int j = 1; j <= l; j++) {
      int pi = 0;          // pending axpy: r_j -= ptau r_pi (pi = 0: none)
      double ptau = 0.0;
      for (int i = 1; i <= j; i++) {
        const bool last = (i == j);
        if (!last && s_g[i] == 0.0) continue;
        double d0 = 0.0, d1 = 0.0;
        double* rj = Rv(j);
        const double* ri = Rv(last ? 0 : i);
        const double* rp = Rv(pi);
        vec_pass(n, gt, gs, true, [&](auto wc, long long e) {
          constexpr int W = decltype(wc)::value;
          Ents<W> a = ldw<W>(rj, e);
          if (pi > 0 && -ptau != 0.0) {
            const Ents<W> p = ldw<W>(rp, e);
#pragma unroll
            for (int k = 0; k < W; k++) a.v[k] = add_rn(a.v[k], mul_rn(-ptau, p.v[k]));
            stw<W>(rj, e, a);
          }
          const Ents<W> c = ldw<W>(ri, e);
#pragma unroll
          for (int k = 0; k < W; k++) {
            if (last) {
              d0 = add_rn(d0, mul_rn(a.v[k], a.v[k]));
              d1 = add_rn(d1, mul_rn(c.v[k], a.v[k]));
            } else {
              d0 = add_rn(d0, mul_rn(a.v[k], c.v[k]));
            }
          }
        });
        d0 = block_sum<NT>(d0, s_red);
        if (last) d1 = block_sum<NT>(d1, s_red);
        if (tid == 0) { s_vals[0] = d0; s_vals[1] = d1; }
        if (!grid_sync<NT>(P, epoch, last ? 2 : 1, s_vals, s_red)) return;
        if (!last) {
          ptau = s_vals[0] / s_g[i];
          if (tid == 0) s_tau[i * L1 + j] = ptau;
          pi = i;
        } else {
          const double gj = s_vals[0];
          const double gpj = s_vals[1];
          __syncthreads();  // every thread has read s_g before thread 0 writes
          if (tid == 0) {
            s_g[j] = gj;
            if (gj != 0.0) s_gp[j] = gpj / gj;
          }
          __syncthreads();
        }
      }
    }
    // gamma = tau^{-1} gamma'; gamma'' = T S gamma (thread 0, in order)
    if (tid == 0) {
      s_g[l] = s_gp[l];
      for (int j = l - 1; j >= 1; j--) {
        double sg = 0.0;
        for (int i = j + 1; i <= l; i++) sg = add_rn(sg, mul_rn(s_tau[j * L1 + i], s_g[i]));
        s_g[j] = add_rn(s_gp[j], -sg);
      }
      for (int j = 1; j <= l - 1; j++) {
        double sg = 0.0;
        for (int i = j + 1; i <= l - 1; i++)
          sg = add_rn(sg, mul_rn(s_tau[j * L1 + i], s_g[i + 1]));
        s_gt[j] = add_rn(s_g[j + 1], sg);
      }
    }
    __syncthreads();
    omega = s_g[l];
    // the update, with the next test's ||r_0||^2 and (r_0, r0)
    {
      double a0 = 0.0, a1 = 0.0;
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long e) {
        constexpr int W = decltype(wc)::value;
        Ents<W> xi = ldw<W>(v.x, e), r0e = ldw<W>(Rv(0), e), u0e = ldw<W>(Uv(0), e);
        const double g1 = s_g[1];
        if (g1 != 0.0)
#pragma unroll
          for (int k = 0; k < W; k++) xi.v[k] = add_rn(xi.v[k], mul_rn(g1, r0e.v[k]));
        {
          const double c = -s_gp[l];
          if (c != 0.0) {
            const Ents<W> t = ldw<W>(Rv(l), e);
#pragma unroll
            for (int k = 0; k < W; k++) r0e.v[k] = add_rn(r0e.v[k], mul_rn(c, t.v[k]));
          }
          const double cu = -s_g[l];
          if (cu != 0.0) {
            const Ents<W> t = ldw<W>(Uv(l), e);
#pragma unroll
            for (int k = 0; k < W; k++) u0e.v[k] = add_rn(u0e.v[k], mul_rn(cu, t.v[k]));
          }
        }
        for (int j = 1; j <= l - 1; j++) {
          const double cu = -s_g[j], cx = s_gt[j], cr = -s_gp[j];
          if (cu != 0.0) {
            const Ents<W> t = ldw<W>(Uv(j), e);
#pragma unroll
            for (int k = 0; k < W; k++) u0e.v[k] = add_rn(u0e.v[k], mul_rn(cu, t.v[k]));
          }
          if (cx != 0.0 || cr != 0.0) {
            const Ents<W> t = ldw<W>(Rv(j), e);
#pragma unroll
            for (int k = 0; k < W; k++) {
              if (cx != 0.0) xi.v[k] = add_rn(xi.v[k], mul_rn(cx, t.v[k]));
              if (cr != 0.0) r0e.v[k] = add_rn(r0e.v[k], mul_rn(cr, t.v[k]));
            }
          }
        }
        stw<W>(v.x, e, xi);
        stw<W>(Rv(0), e, r0e);
        stw<W>(Uv(0), e, u0e);
        const Ents<W> rte = ldw<W>(v.rt, e);
#pragma unroll
        for (int k = 0; k < W; k++) {
          a0 = add_rn(a0, mul_rn(r0e.v[k], r0e.v[k]));
          a1 = add_rn(a1, mul_rn(r0e.v[k], rte.v[k]));
        }
      });
      a0 = block_sum<NT>(a0, s_red);
      a1 = block_sum<NT>(a1, s_red);
      if (tid == 0) { s_vals[0] = a0; s_vals[1] = a1; }
      if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
      rr = s_vals[0];
      rho_next = s_vals[1];
    }
    if (nb_iter == start) break;  // the reference may repeat this cycle for ever
  }
  // change of coordinates (right preconditioning): x = M^{-1} x
  if (jac)
    for (long long i = gt; i < n; i += gs) v.x[i] = precond_val(A.diag, (int)i, __ldcg(v.x + i));
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- QCGS

struct QcgsVecs {
  const double* b;
  double *x, *r, *rt, *u, *p, *ph, *q, *v, *rq, *xq;
  double* uf;  // u = r_qcgs - r after the second product (its operand is u)
};

// epilogue of the product that follows Add(-alpha, ., r): r -= alpha t
// (A M^{-1} u, never stored), u = r_qcgs - r, and the projections (u, u),
// (u, v), (u, r), (v, r).  The new u goes to its own buffer: the product
// gathers the old one.
struct EpiQcgsFit {
  double *r, *u;
  const double *rq, *v;
  double malpha;
  double uu, uv, ur, vr;
  __device__ __forceinline__ void operator()(int i, double t) {
    double ri = __ldcg(r + i);
    if (malpha != 0.0) {
      ri = add_rn(ri, mul_rn(malpha, t));
      r[i] = ri;
    }
    const double ui = add_rn(__ldcg(rq + i), -ri);
    u[i] = ui;
    const double vi = __ldcg(v + i);
    uu = add_rn(uu, mul_rn(ui, ui));
    uv = add_rn(uv, mul_rn(ui, vi));
    ur = add_rn(ur, mul_rn(ui, ri));
    vr = add_rn(vr, mul_rn(vi, ri));
  }
};

// QCgs (QCgs.cxx:46-165): Cgs with a quasi-minimal smoothing step.  Five
// grid barriers per loop: the u, p, phat pass; v = A phat with (rtilde, v)
// and (v, v); the q, u, x pass; the second product with the r update, the
// new u = r_qcgs - r and four projections; the smoothing pass with
// ||r_qcgs||^2 and the next (rtilde, r).  x becomes M^{-1} x_qcgs at the
// end, breakdown or not, as in the reference.
__global__ void __launch_bounds__(NT, 4) qcgs_fused_kernel(OpArgs A, QcgsVecs v, IterArgs it,
                                                        Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  const bool jac = (A.diag != nullptr);
  double* ph = jac ? v.ph : v.p;  // identity: phat aliases its operand
  unsigned epoch = 0;
  int hlen = 0;

  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // r = b - A x (or x = 0, r = b)
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      v.x[i] = 0.0;
      v.r[i] = __ldg(v.b + i);
    }
  } else {
    EpiResidual epi{v.b, v.r, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
  }
  if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  // rtilde = r_qcgs = r; x_qcgs = x; q = p = 0; ||r||^2 (= (rtilde, r))
  double rr = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double ri = __ldcg(v.r + i);
    v.rt[i] = ri;
    v.rq[i] = ri;
    v.xq[i] = __ldcg(v.x + i);
    v.q[i] = 0.0;
    v.p[i] = 0.0;
    rr = add_rn(rr, mul_rn(ri, ri));
  }
  rr = block_sum<NT>(rr, s_red);
  if (tid == 0) s_vals[0] = rr;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  double rqq = s_vals[0], rho_2 = s_vals[0], rho_1 = 1.0;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * sqrt(rqq);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    if (rho_1 == 0.0) { fail = 1; break; }
    const double beta = rho_2 / rho_1;
    // Copy(r, u); Add(beta, q, u); Mlt(beta, p); Add(1, q, p); Mlt(beta, p);
    // Add(1, u, p); phat = M^{-1} p
    vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      const Ents<W> qi = ldw<W>(v.q, i);
      Ents<W> ui = ldw<W>(v.r, i), pi = ldw<W>(v.p, i);
#pragma unroll
      for (int j = 0; j < W; j++) {
        if (beta != 0.0) ui.v[j] = add_rn(ui.v[j], mul_rn(beta, qi.v[j]));
        pi.v[j] = add_rn(mul_rn(add_rn(mul_rn(pi.v[j], beta), qi.v[j]), beta), ui.v[j]);
      }
      stw<W>(v.u, i, ui);
      stw<W>(v.p, i, pi);
      if (jac) stw<W>(ph, i, precond_w<W>(A.diag, i, pi));
    });
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // v = A phat with sigma = (rtilde, v) and (v, v)
    {
      EpiStoreDot2 epi{v.v, v.rt, true, 0.0, 0.0};
      spmv_phase(A, ph, epi, s_prod, s_red);
      const double sg = block_sum<NT>(epi.acc0, s_red);
      const double vv = block_sum<NT>(epi.acc1, s_red);
      if (tid == 0) { s_vals[0] = sg; s_vals[1] = vv; }
      if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
    }
    nb_iter++;
    const double sigma = s_vals[0];
    const double b11 = s_vals[1];
    if (sigma == 0.0) { fail = 2; break; }
    const double alpha = rho_2 / sigma;
    // Copy(u, q); Add(-alpha, v, q); Add(1, q, u); Add(alpha, u, x);
    // phat = M^{-1} u
    vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      Ents<W> ui = ldw<W>(v.u, i), qi = ui;
      if (-alpha != 0.0) {
        const Ents<W> vi = ldw<W>(v.v, i);
#pragma unroll
        for (int j = 0; j < W; j++) qi.v[j] = add_rn(qi.v[j], mul_rn(-alpha, vi.v[j]));
      }
#pragma unroll
      for (int j = 0; j < W; j++) ui.v[j] = add_rn(ui.v[j], qi.v[j]);
      stw<W>(v.q, i, qi);
      stw<W>(v.u, i, ui);
      if (alpha != 0.0) {
        Ents<W> xi = ldw<W>(v.x, i);
#pragma unroll
        for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(alpha, ui.v[j]));
        stw<W>(v.x, i, xi);
      }
      if (jac) stw<W>(v.ph, i, precond_w<W>(A.diag, i, ui));
    });
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // u = A phat; Add(-alpha, u, r); u = r_qcgs - r; the four projections
    {
      EpiQcgsFit epi{v.r, v.uf, v.rq, v.v, -alpha, 0.0, 0.0, 0.0, 0.0};
      spmv_phase(A, jac ? v.ph : v.u, epi, s_prod, s_red);
      const double uu = block_sum<NT>(epi.uu, s_red);
      const double uv = block_sum<NT>(epi.uv, s_red);
      const double ur = block_sum<NT>(epi.ur, s_red);
      const double vr = block_sum<NT>(epi.vr, s_red);
      if (tid == 0) { s_vals[0] = uu; s_vals[1] = uv; s_vals[2] = ur; s_vals[3] = vr; }
      if (!grid_sync<NT>(P, epoch, 4, s_vals, s_red)) return;
    }
    const double b00 = s_vals[0], b10 = s_vals[1];
    // the symmetric 2 x 2 inverse (b(0,1) is b(1,0))
    const double delta = add_rn(mul_rn(b00, b11), -mul_rn(b10, b10));
    if (delta == 0.0) { fail = 3; break; }
    const double m00 = b11 / delta, m11 = b00 / delta, m10 = -b10 / delta;
    const double rn0 = -s_vals[2], rn1 = -s_vals[3];
    const double mu = add_rn(mul_rn(m00, rn0), mul_rn(m10, rn1));
    const double nu = add_rn(mul_rn(m10, rn0), mul_rn(m11, rn1));
    const double omu = 1.0 - mu;
    // r_qcgs = r + mu u + nu v; x_qcgs = mu x_qcgs + (1 - mu) x - nu p;
    // ||r_qcgs||^2 and the next (rtilde, r)
    {
      double a0 = 0.0, a1 = 0.0;
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> ri = ldw<W>(v.r, i), rti = ldw<W>(v.rt, i);
        Ents<W> rqi = ri, xqi = ldw<W>(v.xq, i);
        if (mu != 0.0) {
          const Ents<W> ui = ldw<W>(v.uf, i);
#pragma unroll
          for (int j = 0; j < W; j++) rqi.v[j] = add_rn(rqi.v[j], mul_rn(mu, ui.v[j]));
        }
        if (nu != 0.0) {
          const Ents<W> vi = ldw<W>(v.v, i);
#pragma unroll
          for (int j = 0; j < W; j++) rqi.v[j] = add_rn(rqi.v[j], mul_rn(nu, vi.v[j]));
        }
#pragma unroll
        for (int j = 0; j < W; j++) xqi.v[j] = mul_rn(xqi.v[j], mu);
        if (omu != 0.0) {
          const Ents<W> xi = ldw<W>(v.x, i);
#pragma unroll
          for (int j = 0; j < W; j++) xqi.v[j] = add_rn(xqi.v[j], mul_rn(omu, xi.v[j]));
        }
        if (-nu != 0.0) {
          const Ents<W> pi = ldw<W>(v.p, i);
#pragma unroll
          for (int j = 0; j < W; j++) xqi.v[j] = add_rn(xqi.v[j], mul_rn(-nu, pi.v[j]));
        }
        stw<W>(v.rq, i, rqi);
        stw<W>(v.xq, i, xqi);
#pragma unroll
        for (int j = 0; j < W; j++) {
          a0 = add_rn(a0, mul_rn(rqi.v[j], rqi.v[j]));
          a1 = add_rn(a1, mul_rn(rti.v[j], ri.v[j]));
        }
      });
      a0 = block_sum<NT>(a0, s_red);
      a1 = block_sum<NT>(a1, s_red);
      if (tid == 0) { s_vals[0] = a0; s_vals[1] = a1; }
      if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
      rqq = s_vals[0];
      rho_1 = rho_2;
      rho_2 = s_vals[1];
    }
    nb_iter++;
  }
  // x = M^{-1} x_qcgs (a Copy for the identity)
  for (long long i = gt; i < n; i += gs) v.x[i] = precond_val(A.diag, (int)i, __ldcg(v.xq + i));
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- BICG

struct BcgVecs {
  const double* b;
  double *x, *r, *rt, *p, *pt, *q, *qt;
  OpArgs AT;  // the transposed product: A itself for symmetric storage
};

// epilogue that only stores the product
struct EpiStore {
  double* y;
  __device__ __forceinline__ void operator()(int r, double t) { y[r] = t; }
  __device__ __forceinline__ void quad(int r, const double* t) {
    if (!al16(y + r)) {
      for (int j = 0; j < 4; j++) y[r + j] = t[j];
      return;
    }
    const double tv[4] = {t[0], t[1], t[2], t[3]};
    vst4(y + r, tv);
  }
};

// BiCg (BiCg.cxx:46-134): three grid barriers per loop -- the p and p~
// pass; the products q = A p (fused with (p~, q)) and q~ = A^T p~ in one
// phase, since neither reads what the other writes; the update pass with
// ||r||^2 and the next rho = (M^{-1} r, r~).  z and z~ are never stored:
// with the identity or Jacobi they are recomputed where they are read.
// Seldon's Mlt(SeldonTrans, ...) sums row i of the transpose in increasing
// index order (Functions_MatVect.cxx:1279-1317), which is what the product
// over the explicit transpose (or the expanded symmetric pattern) does.
__global__ void __launch_bounds__(NT, 4) bicg_fused_kernel(OpArgs A, BcgVecs v, IterArgs it,
                                                        Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // r = b - A x (or x = 0, r = b)
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      v.x[i] = 0.0;
      v.r[i] = __ldg(v.b + i);
    }
  } else {
    EpiResidual epi{v.b, v.r, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
  }
  if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  // r~ = r; ||r||^2 and rho = (M^{-1} r, r~)
  double rr = 0.0, rz = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double ri = __ldcg(v.r + i);
    v.rt[i] = ri;
    rr = add_rn(rr, mul_rn(ri, ri));
    rz = add_rn(rz, mul_rn(precond_val(A.diag, (int)i, ri), ri));
  }
  rr = block_sum<NT>(rr, s_red);
  rz = block_sum<NT>(rz, s_red);
  if (tid == 0) { s_vals[0] = rr; s_vals[1] = rz; }
  if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
  rr = s_vals[0];
  double rho_1 = s_vals[1], rho_2 = 0.0;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * sqrt(rr);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    if (rho_1 == 0.0) { fail = 1; break; }
    // p = z, p~ = z~ (first) | Mlt(beta, p); Add(1, z, p); the same for p~
    {
      const bool first = nb_iter == 0;
      const double beta = first ? 0.0 : rho_1 / rho_2;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> z = precond_w<W>(A.diag, i, ldw<W>(v.r, i));
        const Ents<W> zt = precond_w<W>(A.diag, i, ldw<W>(v.rt, i));
        if (first) {
          stw<W>(v.p, i, z);
          stw<W>(v.pt, i, zt);
        } else {
          Ents<W> pi = ldw<W>(v.p, i), pti = ldw<W>(v.pt, i);
#pragma unroll
          for (int j = 0; j < W; j++) {
            pi.v[j] = add_rn(mul_rn(pi.v[j], beta), z.v[j]);
            pti.v[j] = add_rn(mul_rn(pti.v[j], beta), zt.v[j]);
          }
          stw<W>(v.p, i, pi);
          stw<W>(v.pt, i, pti);
        }
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    }
    // q = A p with delta = (p~, q); q~ = A^T p~
    {
      EpiStoreDot e1{v.q, v.pt, 0.0};
      spmv_phase(A, v.p, e1, s_prod, s_red);
      EpiStore e2{v.qt};
      spmv_phase(v.AT, v.pt, e2, s_prod, s_red);
      const double d = block_sum<NT>(e1.acc, s_red);
      if (tid == 0) s_vals[0] = d;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    nb_iter++;
    const double delta = s_vals[0];
    if (delta == 0.0) { fail = 2; break; }
    const double alpha = rho_1 / delta;
    // Add(alpha, p, x); Add(-alpha, q, r); Add(-alpha, q~, r~); the next
    // ||r||^2 and rho
    {
      double a0 = 0.0, a1 = 0.0;
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        if (alpha != 0.0) {
          Ents<W> xi = ldw<W>(v.x, i);
          const Ents<W> pi = ldw<W>(v.p, i);
#pragma unroll
          for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(alpha, pi.v[j]));
          stw<W>(v.x, i, xi);
        }
        Ents<W> ri = ldw<W>(v.r, i), rti = ldw<W>(v.rt, i);
        if (-alpha != 0.0) {
          const Ents<W> qi = ldw<W>(v.q, i), qti = ldw<W>(v.qt, i);
#pragma unroll
          for (int j = 0; j < W; j++) {
            ri.v[j] = add_rn(ri.v[j], mul_rn(-alpha, qi.v[j]));
            rti.v[j] = add_rn(rti.v[j], mul_rn(-alpha, qti.v[j]));
          }
          stw<W>(v.r, i, ri);
          stw<W>(v.rt, i, rti);
        }
        const Ents<W> zi = precond_w<W>(A.diag, i, ri);
#pragma unroll
        for (int j = 0; j < W; j++) {
          a0 = add_rn(a0, mul_rn(ri.v[j], ri.v[j]));
          a1 = add_rn(a1, mul_rn(zi.v[j], rti.v[j]));
        }
      });
      a0 = block_sum<NT>(a0, s_red);
      a1 = block_sum<NT>(a1, s_red);
      if (tid == 0) { s_vals[0] = a0; s_vals[1] = a1; }
      if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
      rr = s_vals[0];
      rho_2 = rho_1;
      rho_1 = s_vals[1];
    }
    nb_iter++;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- CGNE

struct CgneVecs {
  const double* b;
  double *x, *r, *p, *q, *z;
  OpArgs AT;  // the transposed product: A itself for symmetric storage
};

// z = M^{-1} M^{-T} r (TransSolve then Solve; Jacobi divides twice)
__device__ __forceinline__ double cgne_z(const double* diag, int i, double r) {
  return precond_val(diag, i, precond_val(diag, i, r));
}

// epilogue of r = A^T (A x): Mlt(-1, r); Add(1, q, r); with (r, z)
struct EpiCgneInit {
  double* r;
  const double* q;
  const double* diag;
  double rz;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double ri = add_rn(-t, __ldcg(q + i));
    r[i] = ri;
    rz = add_rn(rz, mul_rn(ri, cgne_z(diag, i, ri)));
  }
};

// epilogue of q = A^T b: store q, with ||q||^2
struct EpiStoreNorm {
  double* y;
  double acc;
  __device__ __forceinline__ void operator()(int r, double t) {
    y[r] = t;
    acc = add_rn(acc, mul_rn(t, t));
  }
};

// Cgne (Cgne.cxx:40-127): CG on A^T A x = A^T b.  Four grid barriers per
// loop (two counted iterations): the p pass, with z = M^{-1} M^{-T} r
// recomputed where it is read; q = A p; z = A^T q fused with (p, z); the
// update pass with ||r||^2 and the next rho = (r, M^{-1} M^{-T} r).  The
// first test is on ||A^T b|| even from an initial guess, as in the
// reference.
__global__ void __launch_bounds__(NT, 4) cgne_fused_kernel(OpArgs A, CgneVecs v, IterArgs it,
                                                        Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  // q = A^T b; iter.Init(q)
  {
    EpiStoreNorm epi{v.q, 0.0};
    spmv_phase(v.AT, v.b, epi, s_prod, s_red);
    const double a = block_sum<NT>(epi.acc, s_red);
    if (tid == 0) s_vals[0] = a;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  }
  const double dq = sqrt(s_vals[0]);
  if (dq == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / dq;
  // r = q - A^T A x (or r = q, x = 0), with rho = (r, z)
  double rz = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      const double ri = __ldcg(v.q + i);
      v.r[i] = ri;
      v.x[i] = 0.0;
      rz = add_rn(rz, mul_rn(ri, cgne_z(A.diag, (int)i, ri)));
    }
  } else {
    EpiStore e1{v.p};
    spmv_phase(A, v.x, e1, s_prod, s_red);
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    EpiCgneInit e2{v.r, v.q, A.diag, 0.0};
    spmv_phase(v.AT, v.p, e2, s_prod, s_red);
    rz = e2.rz;
  }
  rz = block_sum<NT>(rz, s_red);
  if (tid == 0) s_vals[0] = rz;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  double rho = s_vals[0], rho_1 = 0.0;
  double dp = dq;  // Norm2(q)

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * dp;
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    if (rho == 0.0) { fail = 1; break; }
    // p = z (first) | Mlt(beta, p); Add(1, z, p)
    {
      const bool first = nb_iter == 0;
      const double beta = first ? 0.0 : rho / rho_1;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> z = precond_w<W>(A.diag, i, precond_w<W>(A.diag, i, ldw<W>(v.r, i)));
        if (first) {
          stw<W>(v.p, i, z);
        } else {
          Ents<W> pi = ldw<W>(v.p, i);
#pragma unroll
          for (int j = 0; j < W; j++) pi.v[j] = add_rn(mul_rn(pi.v[j], beta), z.v[j]);
          stw<W>(v.p, i, pi);
        }
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    }
    // q = A p
    {
      EpiStore e{v.q};
      spmv_phase(A, v.p, e, s_prod, s_red);
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    }
    // z = A^T q with delta = (p, z)
    {
      EpiStoreDot e{v.z, v.p, 0.0};
      spmv_phase(v.AT, v.q, e, s_prod, s_red);
      const double d = block_sum<NT>(e.acc, s_red);
      if (tid == 0) s_vals[0] = d;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    const double delta = s_vals[0];
    if (delta == 0.0) { fail = 2; break; }
    const double alpha = rho / delta;
    // Add(alpha, p, x); Add(-alpha, z, r); ||r||^2 and the next rho
    {
      double a0 = 0.0, a1 = 0.0;
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        if (alpha != 0.0) {
          Ents<W> xi = ldw<W>(v.x, i);
          const Ents<W> pi = ldw<W>(v.p, i);
#pragma unroll
          for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(alpha, pi.v[j]));
          stw<W>(v.x, i, xi);
        }
        Ents<W> ri = ldw<W>(v.r, i);
        if (-alpha != 0.0) {
          const Ents<W> zi = ldw<W>(v.z, i);
#pragma unroll
          for (int j = 0; j < W; j++) ri.v[j] = add_rn(ri.v[j], mul_rn(-alpha, zi.v[j]));
          stw<W>(v.r, i, ri);
        }
        const Ents<W> zn = precond_w<W>(A.diag, i, precond_w<W>(A.diag, i, ri));
#pragma unroll
        for (int j = 0; j < W; j++) {
          a0 = add_rn(a0, mul_rn(ri.v[j], ri.v[j]));
          a1 = add_rn(a1, mul_rn(ri.v[j], zn.v[j]));
        }
      });
      a0 = block_sum<NT>(a0, s_red);
      a1 = block_sum<NT>(a1, s_red);
      if (tid == 0) { s_vals[0] = a0; s_vals[1] = a1; }
      if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
      rho_1 = rho;
      rho = s_vals[1];
      dp = sqrt(s_vals[0]);
    }
    nb_iter += 2;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- Symmlq

struct SymmlqVecs {
  const double* b;
  double *x, *r, *z, *w, *w_bar, *u0, *u1, *v0, *v1;  // u, u_old and v, v_old by rotation
};

// Symmlq (Symmlq.cxx:45-161): Lanczos with an LQ factorisation, one product
// a step.  Three grid barriers a step: the update pass (v = r / beta,
// u = z / beta, w, w_bar, x += ceta w; the old u and v kept by pointer
// rotation); r = A u fused with alpha = (u, r); the pass z = M^{-1} r,
// r -= alpha v + beta v_old, z -= alpha u + beta u_old with (r, z).  The
// first test is on ||b|| even from an initial guess; x takes
// ceta_bar * w_bar after the loop, as in the reference.
__global__ void __launch_bounds__(NT, 4) symmlq_fused_kernel(OpArgs A, SymmlqVecs v, IterArgs it,
                                                          Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // r = b - A x (or x = 0, r = b)
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      v.x[i] = 0.0;
      v.r[i] = __ldg(v.b + i);
    }
  } else {
    EpiResidual epi{v.b, v.r, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
  }
  if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  // z = M^{-1} r; dp = (r, z)
  {
    double a0 = 0.0;
    for (long long i = gt; i < n; i += gs) {
      const double ri = __ldcg(v.r + i);
      const double zi = precond_val(A.diag, (int)i, ri);
      v.z[i] = zi;
      a0 = add_rn(a0, mul_rn(ri, zi));
    }
    a0 = block_sum<NT>(a0, s_red);
    if (tid == 0) s_vals[0] = a0;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  }
  double beta = sqrt(s_vals[0]);
  const double beta1 = beta;
  double sprod = fabs(beta1);
  double *u = v.u0, *u_old = v.u1, *vv = v.v0, *v_old = v.v1;
  // v = r / beta; u = z / beta; w_bar = u; u_old = v_old = 0
  {
    const double ib = 1.0 / beta;
    for (long long i = gt; i < n; i += gs) {
      const double ui = mul_rn(__ldcg(v.z + i), ib);
      vv[i] = mul_rn(__ldcg(v.r + i), ib);
      u[i] = ui;
      v.w_bar[i] = ui;
      u_old[i] = 0.0;
      v_old[i] = 0.0;
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  }
  double ceta = 0.0, ceta_old = 0.0, ceta_oold = 0.0;
  double c = 1.0, cold = 1.0, s = 0.0, sold = 0.0;
  double np = normb;

  int nb_iter = 0;
  double reste;
  for (;;) {
    reste = facteur * np;
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    if (nb_iter != 0) {
      // v_old = v; u_old = u (rotation); v = r / beta; u = z / beta;
      // w = c w_bar + s u; w_bar = -s w_bar + c u; x += ceta w
      double* t = v_old; v_old = vv; vv = t;
      t = u_old; u_old = u; u = t;
      const double ib = 1.0 / beta, cc = c, ss = s, ce = ceta;
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> ri = ldw<W>(v.r, i), zi = ldw<W>(v.z, i);
        Ents<W> vi, ui, wi, wb = ldw<W>(v.w_bar, i);
#pragma unroll
        for (int j = 0; j < W; j++) {
          vi.v[j] = mul_rn(ri.v[j], ib);
          ui.v[j] = mul_rn(zi.v[j], ib);
          wi.v[j] = mul_rn(wb.v[j], cc);
          if (ss != 0.0) wi.v[j] = add_rn(wi.v[j], mul_rn(ss, ui.v[j]));
          wb.v[j] = mul_rn(wb.v[j], -ss);
          if (cc != 0.0) wb.v[j] = add_rn(wb.v[j], mul_rn(cc, ui.v[j]));
        }
        stw<W>(vv, i, vi);
        stw<W>(u, i, ui);
        stw<W>(v.w, i, wi);
        stw<W>(v.w_bar, i, wb);
        if (ce != 0.0) {
          Ents<W> xi = ldw<W>(v.x, i);
#pragma unroll
          for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(ce, wi.v[j]));
          stw<W>(v.x, i, xi);
        }
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
      ceta_oold = ceta_old;
      ceta_old = ceta;
    }
    // r = A u with alpha = (u, r)
    {
      EpiStoreDot e{v.r, u, 0.0};
      spmv_phase(A, u, e, s_prod, s_red);
      const double a = block_sum<NT>(e.acc, s_red);
      if (tid == 0) s_vals[0] = a;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    const double alpha = s_vals[0];
    // z = M^{-1} r; Add(-alpha, v, r); Add(-alpha, u, z); Add(-beta, v_old, r);
    // Add(-beta, u_old, z); dp = (r, z)
    {
      double a0 = 0.0;
      const double na = -alpha, nbt = -beta;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        Ents<W> ri = ldw<W>(v.r, i);
        Ents<W> zi = precond_w<W>(A.diag, i, ri);
        if (na != 0.0) {
          const Ents<W> vi = ldw<W>(vv, i), ui = ldw<W>(u, i);
#pragma unroll
          for (int j = 0; j < W; j++) {
            ri.v[j] = add_rn(ri.v[j], mul_rn(na, vi.v[j]));
            zi.v[j] = add_rn(zi.v[j], mul_rn(na, ui.v[j]));
          }
        }
        if (nbt != 0.0) {
          const Ents<W> vo = ldw<W>(v_old, i), uo = ldw<W>(u_old, i);
#pragma unroll
          for (int j = 0; j < W; j++) {
            ri.v[j] = add_rn(ri.v[j], mul_rn(nbt, vo.v[j]));
            zi.v[j] = add_rn(zi.v[j], mul_rn(nbt, uo.v[j]));
          }
        }
        stw<W>(v.r, i, ri);
        stw<W>(v.z, i, zi);
#pragma unroll
        for (int j = 0; j < W; j++) a0 = add_rn(a0, mul_rn(ri.v[j], zi.v[j]));
      });
      a0 = block_sum<NT>(a0, s_red);
      if (tid == 0) s_vals[0] = a0;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    const double beta_old = beta;
    beta = sqrt(s_vals[0]);
    // the QR factorisation and the Givens rotation
    const double coold = cold, soold = sold;
    cold = c;
    sold = s;
    const double rho0 = add_rn(mul_rn(cold, alpha), -mul_rn(mul_rn(coold, sold), beta_old));
    const double rho1 = sqrt(add_rn(mul_rn(rho0, rho0), mul_rn(beta, beta)));
    const double rho2 = add_rn(mul_rn(sold, alpha), mul_rn(mul_rn(coold, cold), beta_old));
    const double rho3 = mul_rn(soold, beta_old);
    c = rho0 / rho1;
    s = beta / rho1;
    if (nb_iter == 0)
      ceta = beta1 / rho1;
    else
      ceta = -add_rn(mul_rn(rho2, ceta_old), mul_rn(rho3, ceta_oold)) / rho1;
    sprod = mul_rn(sprod, fabs(s));
    np = c == 0.0 ? mul_rn(sprod, 1e16) : sprod / fabs(c);
    nb_iter++;
  }
  // Add(ceta_bar, w_bar, x)
  const double ceta_bar = c == 0.0 ? mul_rn(ceta, 1e15) : ceta / c;
  if (ceta_bar != 0.0) {
    vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
      constexpr int W = decltype(wc)::value;
      Ents<W> xi = ldw<W>(v.x, i);
      const Ents<W> wb = ldw<W>(v.w_bar, i);
#pragma unroll
      for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(ceta_bar, wb.v[j]));
      stw<W>(v.x, i, xi);
    });
  }
  if (lead) write_out(out, nb_iter, it.max_iter, 0, facteur, reste, hlen);
}

// ----------------------------------------------------------------- QmrSym

struct QmrsVecs {
  const double* b;
  double *x, *r, *y, *v, *p, *pt, *d, *s;
};

// QmrSym (QmrSym.cxx:41-165): QMR for symmetric systems, one product a step.
// Four grid barriers a step: the p pass; pt = A p fused with ep = (p, pt);
// the v, y pass with ||y||^2; the d, s, x, r pass with ||r||^2, which also
// scales v and y by the new 1 / rho and reduces the next step's
// delta = (v, y) (the reference scales them at the top of its next step,
// after the test, which reads neither).  Fail codes 1, 3, 4, 5, 6 as in the
// reference.
__global__ void __launch_bounds__(NT, 4) qmrsym_fused_kernel(OpArgs A, QmrsVecs v, IterArgs it,
                                                          Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // r = b - A x (or x = 0, r = b)
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      v.x[i] = 0.0;
      v.r[i] = __ldg(v.b + i);
    }
  } else {
    EpiResidual epi{v.b, v.r, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
  }
  if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  // v = r; y = M^{-1} v; rho = ||y||; ||r||^2
  double rr, rho;
  {
    double a0 = 0.0, a1 = 0.0;
    for (long long i = gt; i < n; i += gs) {
      const double ri = __ldcg(v.r + i);
      const double yi = precond_val(A.diag, (int)i, ri);
      v.v[i] = ri;
      v.y[i] = yi;
      a0 = add_rn(a0, mul_rn(yi, yi));
      a1 = add_rn(a1, mul_rn(ri, ri));
    }
    a0 = block_sum<NT>(a0, s_red);
    a1 = block_sum<NT>(a1, s_red);
    if (tid == 0) { s_vals[0] = a0; s_vals[1] = a1; }
    if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
    rho = sqrt(s_vals[0]);
    rr = s_vals[1];
  }
  // Mlt(1 / rho, v); Mlt(1 / rho, y); delta = (v, y)
  double delta;
  {
    const double ir = 1. / rho;
    double a0 = 0.0;
    for (long long i = gt; i < n; i += gs) {
      const double vi = mul_rn(__ldcg(v.v + i), ir), yi = mul_rn(__ldcg(v.y + i), ir);
      v.v[i] = vi;
      v.y[i] = yi;
      a0 = add_rn(a0, mul_rn(vi, yi));
    }
    a0 = block_sum<NT>(a0, s_red);
    if (tid == 0) s_vals[0] = a0;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    delta = s_vals[0];
  }
  double ep = 0.0, theta = 0.0, gamma = 1.0, eta = -1.0;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * sqrt(rr);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    if (rho == 0.0) { fail = 1; break; }
    if (delta == 0.0) { fail = 3; break; }
    const bool first = nb_iter == 0;
    // p = y (first) | Mlt(-(rho delta / ep), p); Add(1, y, p)
    {
      const double c = first ? 0.0 : -(mul_rn(rho, delta) / ep);
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> yi = ldw<W>(v.y, i);
        if (first) {
          stw<W>(v.p, i, yi);
        } else {
          Ents<W> pi = ldw<W>(v.p, i);
#pragma unroll
          for (int j = 0; j < W; j++) pi.v[j] = add_rn(mul_rn(pi.v[j], c), yi.v[j]);
          stw<W>(v.p, i, pi);
        }
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    }
    // pt = A p with ep = (p, pt)
    {
      EpiStoreDot e{v.pt, v.p, 0.0};
      spmv_phase(A, v.p, e, s_prod, s_red);
      const double a = block_sum<NT>(e.acc, s_red);
      if (tid == 0) s_vals[0] = a;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    ep = s_vals[0];
    if (ep == 0.0) { fail = 4; break; }
    const double beta = ep / delta;
    if (beta == 0.0) { fail = 5; break; }
    // Mlt(-beta, v); Add(1, pt, v); y = M^{-1} v; rho = ||y||
    {
      double a0 = 0.0;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        Ents<W> vi = ldw<W>(v.v, i);
        const Ents<W> pti = ldw<W>(v.pt, i);
#pragma unroll
        for (int j = 0; j < W; j++) vi.v[j] = add_rn(mul_rn(vi.v[j], -beta), pti.v[j]);
        const Ents<W> yi = precond_w<W>(A.diag, i, vi);
        stw<W>(v.v, i, vi);
        stw<W>(v.y, i, yi);
#pragma unroll
        for (int j = 0; j < W; j++) a0 = add_rn(a0, mul_rn(yi.v[j], yi.v[j]));
      });
      a0 = block_sum<NT>(a0, s_red);
      if (tid == 0) s_vals[0] = a0;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    const double rho_1 = rho;
    rho = sqrt(s_vals[0]);
    const double gamma_1 = gamma, theta_1 = theta;
    theta = rho / mul_rn(gamma_1, beta);
    gamma = 1.0 / sqrt(add_rn(1.0, mul_rn(theta, theta)));
    if (gamma == 0.0) { fail = 6; break; }
    eta = mul_rn(mul_rn(mul_rn(-eta, rho_1), gamma), gamma) /
          mul_rn(mul_rn(beta, gamma_1), gamma_1);
    // d, s; Add(1, d, x); Add(-1, s, r) with ||r||^2; then the next step's
    // Mlt(1 / rho, v), Mlt(1 / rho, y) and delta = (v, y)
    {
      const double tmp = first ? 0.0 : mul_rn(mul_rn(mul_rn(theta_1, theta_1), gamma), gamma);
      const double ir = 1. / rho;
      const double et = eta;
      double a0 = 0.0, a1 = 0.0;
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        const Ents<W> pi = ldw<W>(v.p, i), pti = ldw<W>(v.pt, i);
        Ents<W> di, si;
        if (first) {
#pragma unroll
          for (int j = 0; j < W; j++) {
            di.v[j] = mul_rn(pi.v[j], et);
            si.v[j] = mul_rn(pti.v[j], et);
          }
        } else {
          di = ldw<W>(v.d, i);
          si = ldw<W>(v.s, i);
#pragma unroll
          for (int j = 0; j < W; j++) {
            di.v[j] = mul_rn(di.v[j], tmp);
            si.v[j] = mul_rn(si.v[j], tmp);
            if (et != 0.0) {
              di.v[j] = add_rn(di.v[j], mul_rn(et, pi.v[j]));
              si.v[j] = add_rn(si.v[j], mul_rn(et, pti.v[j]));
            }
          }
        }
        stw<W>(v.d, i, di);
        stw<W>(v.s, i, si);
        Ents<W> xi = ldw<W>(v.x, i), ri = ldw<W>(v.r, i), vi = ldw<W>(v.v, i), yi = ldw<W>(v.y, i);
#pragma unroll
        for (int j = 0; j < W; j++) {
          xi.v[j] = add_rn(xi.v[j], di.v[j]);
          ri.v[j] = add_rn(ri.v[j], -si.v[j]);
          vi.v[j] = mul_rn(vi.v[j], ir);
          yi.v[j] = mul_rn(yi.v[j], ir);
          a0 = add_rn(a0, mul_rn(ri.v[j], ri.v[j]));
          a1 = add_rn(a1, mul_rn(vi.v[j], yi.v[j]));
        }
        stw<W>(v.x, i, xi);
        stw<W>(v.r, i, ri);
        stw<W>(v.v, i, vi);
        stw<W>(v.y, i, yi);
      });
      a0 = block_sum<NT>(a0, s_red);
      a1 = block_sum<NT>(a1, s_red);
      if (tid == 0) { s_vals[0] = a0; s_vals[1] = a1; }
      if (!grid_sync<NT>(P, epoch, 2, s_vals, s_red)) return;
      rr = s_vals[0];
      delta = s_vals[1];
    }
    nb_iter++;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- Lsqr

struct LsqrVecs {
  const double* b;
  double *x, *u, *u1, *v, *v1, *w;
  OpArgs AT;  // the transposed product: A itself for symmetric storage
};

// epilogue of y = A x; Add(na, u, y) (skipped when na == 0, as Seldon's Add
// is); with ||y||^2
struct EpiAxpyNorm {
  double* y;
  const double* u;
  double na;
  double acc;
  __device__ __forceinline__ void operator()(int i, double t) {
    const double yi = na != 0.0 ? add_rn(t, mul_rn(na, __ldcg(u + i))) : t;
    y[i] = yi;
    acc = add_rn(acc, mul_rn(yi, yi));
  }
};

// Lsqr (Lsqr.cxx:40-135): Golub-Kahan bidiagonalisation; the preconditioner
// is not used.  The initial guess enters only the first test: x is zeroed
// and u starts from b either way, as in the reference.  Four grid barriers a
// loop (two counted iterations): u1 = A v - alpha u with ||u1||^2; u1 /=
// beta; v1 = A^T u1 - beta v with ||v1||^2; the pass that scales v1 and
// updates x and w.  u, u1 and v, v1 swap by pointer.
__global__ void __launch_bounds__(NT, 4) lsqr_fused_kernel(OpArgs A, LsqrVecs v, IterArgs it,
                                                        Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;
  // rnorm = ||b - A x|| (||b|| from a zero guess)
  double rnorm = normb;
  if (!it.init_guess_null) {
    EpiResidual epi{v.b, v.u, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    const double r2 = block_sum<NT>(epi.rr, s_red);
    if (tid == 0) s_vals[0] = r2;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    rnorm = sqrt(s_vals[0]);
  }
  // u = b / ||b||; x = 0
  {
    const double tb = 1.0 / normb;
    for (long long i = gt; i < n; i += gs) {
      v.u[i] = mul_rn(__ldg(v.b + i), tb);
      v.x[i] = 0.0;
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  }
  // v = A^T u, alpha = ||v||; v /= alpha; w = v
  double alpha;
  {
    EpiStoreNorm e{v.v, 0.0};
    spmv_phase(v.AT, v.u, e, s_prod, s_red);
    const double a = block_sum<NT>(e.acc, s_red);
    if (tid == 0) s_vals[0] = a;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    alpha = sqrt(s_vals[0]);
    const double ta = 1.0 / alpha;
    for (long long i = gt; i < n; i += gs) {
      const double vi = mul_rn(__ldcg(v.v + i), ta);
      v.v[i] = vi;
      v.w[i] = vi;
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  }
  double phi_bar = normb, rho_bar = alpha;
  double *u = v.u, *u1 = v.u1, *vv = v.v, *v1 = v.v1;

  int nb_iter = 0, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * rnorm;
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    // u1 = A v; Add(-alpha, u, u1); beta = ||u1||
    {
      EpiAxpyNorm e{u1, u, -alpha, 0.0};
      spmv_phase(A, vv, e, s_prod, s_red);
      const double a = block_sum<NT>(e.acc, s_red);
      if (tid == 0) s_vals[0] = a;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    const double beta = sqrt(s_vals[0]);
    if (beta == 0.0) { fail = 1; break; }
    // Mlt(1 / beta, u1)
    {
      const double tb = 1.0 / beta;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        Ents<W> ui = ldw<W>(u1, i);
#pragma unroll
        for (int j = 0; j < W; j++) ui.v[j] = mul_rn(ui.v[j], tb);
        stw<W>(u1, i, ui);
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    }
    // v1 = A^T u1; Add(-beta, v, v1); alpha = ||v1||
    {
      EpiAxpyNorm e{v1, vv, -beta, 0.0};
      spmv_phase(v.AT, u1, e, s_prod, s_red);
      const double a = block_sum<NT>(e.acc, s_red);
      if (tid == 0) s_vals[0] = a;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    alpha = sqrt(s_vals[0]);
    if (alpha == 0.0) { fail = 2; break; }
    const double rho = sqrt(add_rn(mul_rn(rho_bar, rho_bar), mul_rn(beta, beta)));
    if (rho == 0.0) { fail = 3; break; }
    const double c = rho_bar / rho, s = beta / rho;
    const double theta = mul_rn(s, alpha);
    rho_bar = mul_rn(-c, alpha);
    const double phi = mul_rn(c, phi_bar);
    phi_bar = mul_rn(s, phi_bar);
    // Mlt(1 / alpha, v1); Add(phi / rho, w, x); Mlt(-theta / rho, w); Add(1, v1, w)
    {
      const double ta = 1.0 / alpha, tx = phi / rho, tw = -theta / rho;
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        Ents<W> vi = ldw<W>(v1, i), wi = ldw<W>(v.w, i);
#pragma unroll
        for (int j = 0; j < W; j++) vi.v[j] = mul_rn(vi.v[j], ta);
        stw<W>(v1, i, vi);
        if (tx != 0.0) {
          Ents<W> xi = ldw<W>(v.x, i);
#pragma unroll
          for (int j = 0; j < W; j++) xi.v[j] = add_rn(xi.v[j], mul_rn(tx, wi.v[j]));
          stw<W>(v.x, i, xi);
        }
#pragma unroll
        for (int j = 0; j < W; j++) wi.v[j] = add_rn(mul_rn(wi.v[j], tw), vi.v[j]);
        stw<W>(v.w, i, wi);
      });
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    }
    rnorm = fabs(phi_bar);
    double* t = u1; u1 = u; u = t;
    t = v1; v1 = vv; vv = t;
    nb_iter += 2;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- BiCgcr

struct BcrVecs {
  const double* b;
  double *x, *v, *w, *s, *z, *p, *a;
};

// epilogue of a = A p: a stored, w = M^{-1} a, with ||v||^2, (w, v), (w, a)
struct EpiBcrA {
  double *a, *w;
  const double* v;
  const double* diag;
  double vv, wv, wa;
  __device__ __forceinline__ void operator()(int i, double t) {
    a[i] = t;
    const double wi = precond_val(diag, i, t);
    w[i] = wi;
    const double vi = __ldcg(v + i);
    vv = add_rn(vv, mul_rn(vi, vi));
    wv = add_rn(wv, mul_rn(wi, vi));
    wa = add_rn(wa, mul_rn(wi, t));
  }
};

// BiCgcr (BiCgcr.cxx:44-118): biconjugate conjugate residuals.  Three grid
// barriers a step: the x, v, s update pass; z = A s fused with tau = (w, z);
// the p, a, w pass with ||v||^2 and the next step's rho = (w, v) and
// mu = (w, a).  The count starts at 1: the reference counts the first
// product a = A p before its first test.
__global__ void __launch_bounds__(NT, 4) bicgcr_fused_kernel(OpArgs A, BcrVecs v, IterArgs it,
                                                          Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  double acc = 0.0;
  for (long long i = gt; i < n; i += gs) {
    const double bi = __ldg(v.b + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  acc = block_sum<NT>(acc, s_red);
  if (tid == 0) s_vals[0] = acc;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  const double normb = sqrt(s_vals[0]);
  if (normb == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / normb;

  // v = b - A x (or x = 0, v = b)
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      v.x[i] = 0.0;
      v.v[i] = __ldg(v.b + i);
    }
  } else {
    EpiResidual epi{v.b, v.v, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
  }
  if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  // s = M^{-1} v; p = s
  for (long long i = gt; i < n; i += gs) {
    const double si = precond_val(A.diag, (int)i, __ldcg(v.v + i));
    v.s[i] = si;
    v.p[i] = si;
  }
  if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
  // a = A p; w = M^{-1} a; ++iter
  double vv, wv, wa;
  {
    EpiBcrA e{v.a, v.w, v.v, A.diag, 0.0, 0.0, 0.0};
    spmv_phase(A, v.p, e, s_prod, s_red);
    vv = block_sum<NT>(e.vv, s_red);
    wv = block_sum<NT>(e.wv, s_red);
    wa = block_sum<NT>(e.wa, s_red);
    if (tid == 0) { s_vals[0] = vv; s_vals[1] = wv; s_vals[2] = wa; }
    if (!grid_sync<NT>(P, epoch, 3, s_vals, s_red)) return;
    vv = s_vals[0]; wv = s_vals[1]; wa = s_vals[2];
  }

  int nb_iter = 1, fail = 0;
  double reste;
  for (;;) {
    reste = facteur * sqrt(vv);
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    const double mu = wa;
    if (mu == 0.0) { fail = 1; break; }
    const double alpha = wv / mu;
    // Add(alpha, p, x); Add(-alpha, a, v); Add(-alpha, w, s)
    if (alpha != 0.0) {
      vec_pass(n, gt, gs, al16(v.x), [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        Ents<W> xi = ldw<W>(v.x, i), vi = ldw<W>(v.v, i), si = ldw<W>(v.s, i);
        const Ents<W> pi = ldw<W>(v.p, i), ai = ldw<W>(v.a, i), wi = ldw<W>(v.w, i);
#pragma unroll
        for (int j = 0; j < W; j++) {
          xi.v[j] = add_rn(xi.v[j], mul_rn(alpha, pi.v[j]));
          vi.v[j] = add_rn(vi.v[j], mul_rn(-alpha, ai.v[j]));
          si.v[j] = add_rn(si.v[j], mul_rn(-alpha, wi.v[j]));
        }
        stw<W>(v.x, i, xi);
        stw<W>(v.v, i, vi);
        stw<W>(v.s, i, si);
      });
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // z = A s with tau = (w, z)
    {
      EpiStoreDot e{v.z, v.w, 0.0};
      spmv_phase(A, v.s, e, s_prod, s_red);
      const double d = block_sum<NT>(e.acc, s_red);
      if (tid == 0) s_vals[0] = d;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    }
    const double tau = s_vals[0];
    if (tau == 0.0) { fail = 2; break; }
    const double nbeta = -(tau / mu);
    // Mlt(-beta, p); Add(1, s, p); Mlt(-beta, a); Add(1, z, a); w = M^{-1} a,
    // with ||v||^2, (w, v), (w, a)
    {
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      vec_pass(n, gt, gs, true, [&](auto wc, long long i) {
        constexpr int W = decltype(wc)::value;
        Ents<W> pi = ldw<W>(v.p, i), ai = ldw<W>(v.a, i);
        const Ents<W> si = ldw<W>(v.s, i), zi = ldw<W>(v.z, i), vi = ldw<W>(v.v, i);
#pragma unroll
        for (int j = 0; j < W; j++) {
          pi.v[j] = add_rn(mul_rn(nbeta, pi.v[j]), si.v[j]);
          ai.v[j] = add_rn(mul_rn(nbeta, ai.v[j]), zi.v[j]);
        }
        const Ents<W> wi = precond_w<W>(A.diag, i, ai);
        stw<W>(v.p, i, pi);
        stw<W>(v.a, i, ai);
        stw<W>(v.w, i, wi);
#pragma unroll
        for (int j = 0; j < W; j++) {
          a0 = add_rn(a0, mul_rn(vi.v[j], vi.v[j]));
          a1 = add_rn(a1, mul_rn(wi.v[j], vi.v[j]));
          a2 = add_rn(a2, mul_rn(wi.v[j], ai.v[j]));
        }
      });
      a0 = block_sum<NT>(a0, s_red);
      a1 = block_sum<NT>(a1, s_red);
      a2 = block_sum<NT>(a2, s_red);
      if (tid == 0) { s_vals[0] = a0; s_vals[1] = a1; s_vals[2] = a2; }
      if (!grid_sync<NT>(P, epoch, 3, s_vals, s_red)) return;
      vv = s_vals[0]; wv = s_vals[1]; wa = s_vals[2];
    }
    nb_iter++;
  }
  if (lead) write_out(out, nb_iter, it.max_iter, fail, facteur, reste, hlen);
}

// ----------------------------------------------------------------- GMRES

struct GmresVecs {
  const double* b;
  double *x, *r, *w, *V;  // V: (m+1) vectors of length n, `ld` apart
  long long ld;
};

// epilogue of u = A V_i: w_r = M^{-1} u_r, acc += V0_r * w_r (first MGS dot)
struct EpiPrecDot {
  double* w;
  const double* v0;
  const double* diag;
  double acc;
  __device__ __forceinline__ void operator()(int r, double t) {
    const double wr = precond_val(diag, r, t);
    w[r] = wr;
    acc = add_rn(acc, mul_rn(__ldcg(v0 + r), wr));
  }
  __device__ __forceinline__ void quad(int r, const double* t) {
    if (!al16(w + r) || !al16(v0 + r) || (diag && !al16(diag + r))) {
      for (int j = 0; j < 4; j++) (*this)(r + j, t[j]);
      return;
    }
    double vv[4], wv[4] = {t[0], t[1], t[2], t[3]};
    vld4_cg(v0 + r, vv);
    if (diag) {
      double dv[4];
      vld4_ldg(diag + r, dv);
#pragma unroll
      for (int j = 0; j < 4; j++) wv[j] = __ddiv_rn(t[j], dv[j]);
    }
    vst4(w + r, wv);
#pragma unroll
    for (int j = 0; j < 4; j++) acc = add_rn(acc, mul_rn(vv[j], wv[j]));
  }
};

__global__ void __launch_bounds__(NT, 4) gmres_fused_kernel(OpArgs A, GmresVecs v, IterArgs it,
                                                         Persist P, History H, SolveOut* out) {
  SB2_SHARED_DECL;
  extern __shared__ double s_dyn[];
  const int m = it.restart;
  const int ld = m + 1;
  double* Hm = s_dyn;            // (m+1) x (m+1), column-major
  double* sv = Hm + ld * ld;     // s(0..m)
  double* cs = sv + ld;          // rotations_cos
  double* sn = cs + ld;          // rotations_sin
  const int tid = threadIdx.x;
  const long long gt = (long long)blockIdx.x * NT + tid, gs = (long long)gridDim.x * NT;
  const int n = A.n;
  const size_t nn = (size_t)v.ld;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;

  for (int k = tid; k < ld * ld + 3 * ld; k += NT) s_dyn[k] = 0.0;

  // w = b (- A x); r = M^{-1} w; beta = ||r|| (Gmres.cxx:82-90)
  double rr = 0.0;
  if (it.init_guess_null) {
    for (long long i = gt; i < n; i += gs) {
      const double bi = __ldg(v.b + i);
      v.x[i] = 0.0;
      const double ri = precond_val(A.diag, (int)i, bi);
      v.r[i] = ri;
      rr = add_rn(rr, mul_rn(ri, ri));
    }
  } else {
    EpiResidual epi{v.b, v.w, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    for (long long i = gt; i < n; i += gs) {
      const double ri = precond_val(A.diag, (int)i, __ldcg(v.w + i));
      v.r[i] = ri;
      rr = add_rn(rr, mul_rn(ri, ri));
    }
  }
  rr = block_sum<NT>(rr, s_red);
  if (tid == 0) s_vals[0] = rr;
  if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
  double beta = sqrt(s_vals[0]);
  // outer.Init(r)
  if (beta == 0.0) {
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = 1.0 / beta;

  int nb_iter = 0;
  double reste;
  for (;;) {
    // while (!outer.Finished(beta))
    reste = facteur * beta;
    if (lead) hist_push(H, &hlen, nb_iter, reste);
    if (reste < it.tol || nb_iter >= it.max_iter) break;
    // V0 = r * (1/beta); s = beta e0
    const double inv_beta = 1.0 / beta;
    for (long long i = gt; i < n; i += gs) v.V[i] = mul_rn(__ldcg(v.r + i), inv_beta);
    if (tid == 0) {
      for (int k = 0; k < ld; k++) sv[k] = 0.0;
      sv[0] = beta;
    }
    const int inner_max = nb_iter + m;
    int i = 0;
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    for (;;) {
      double* Vi = v.V + (size_t)i * nn;
      // u = A V_i; w = M^{-1} u; h_{0,i} = (V_0, w)
      EpiPrecDot epi{v.w, v.V, A.diag, 0.0};
      spmv_phase(A, Vi, epi, s_prod, s_red);
      double d = block_sum<NT>(epi.acc, s_red);
      if (tid == 0) s_vals[0] = d;
      if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
      // modified Gram-Schmidt: H(k,i) = (V_k, w); Add(-H(k,i), V_k, w)
      for (int k = 0; k <= i; k++) {
        const double h = s_vals[0];
        if (tid == 0) Hm[k + i * ld] = h;
        const double* Vk = v.V + (size_t)k * nn;
        const double* Vn = (k < i) ? v.V + (size_t)(k + 1) * nn : nullptr;
        // paired 16-byte passes: 169 against 188 ms for the scalar form on
        // the 128^3 convection-diffusion operator with Jacobi and restart 30
        double acc = 0.0;
        vec_pass(n, gt, gs, true, [&](auto wc, long long e) {
          constexpr int W = decltype(wc)::value;
          Ents<W> we = ldw<W>(v.w, e);
          if (-h != 0.0) {
            const Ents<W> vke = ldw<W>(Vk, e);
#pragma unroll
            for (int j = 0; j < W; j++) we.v[j] = add_rn(we.v[j], mul_rn(-h, vke.v[j]));
            stw<W>(v.w, e, we);
          }
          const Ents<W> vne = Vn ? ldw<W>(Vn, e) : we;
#pragma unroll
          for (int j = 0; j < W; j++) acc = add_rn(acc, mul_rn(vne.v[j], we.v[j]));
        });
        acc = block_sum<NT>(acc, s_red);
        if (tid == 0) s_vals[0] = acc;
        if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
      }
      // h_{i+1,i} = ||w||; V_{i+1} = w / h
      double hi_ip1 = sqrt(s_vals[0]);
      double* Vn = v.V + (size_t)(i + 1) * nn;
      const double inv_h = (hi_ip1 != 0.0) ? 1.0 / hi_ip1 : 1.0;
      vec_pass(n, gt, gs, true, [&](auto wc, long long e) {
        constexpr int W = decltype(wc)::value;
        Ents<W> we = ldw<W>(v.w, e);
        if (hi_ip1 != 0.0) {
#pragma unroll
          for (int j = 0; j < W; j++) we.v[j] = mul_rn(we.v[j], inv_h);
        }
        stw<W>(Vn, e, we);
      });
      // rotations (every CTA computes the same scalars)
      if (tid == 0) {
        for (int k = 0; k < i; k++) apply_rot(Hm[k + i * ld], Hm[k + 1 + i * ld], cs[k], sn[k]);
        if (hi_ip1 != 0.0) {
          gen_rot(Hm[i + i * ld], hi_ip1, cs[i], sn[i]);
          apply_rot(sv[i], sv[i + 1], cs[i], sn[i]);
        }
      }
      i++;
      nb_iter++;
      __syncthreads();
      // inner.Finished(|s(i)|): inner counts alongside outer, max = start + m
      const double rin = facteur * fabs(sv[i]);
      if (lead) hist_push(H, &hlen, nb_iter, rin);
      reste = rin;
      const bool stop = (rin < it.tol) || (nb_iter >= inner_max);
      if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;  // V_{i} complete
      if (stop) break;
    }
    // Solve(H, s): netlib DTRSV column sweep on the leading i x i block
    if (tid == 0) {
      for (int j = i - 1; j >= 0; j--)
        if (sv[j] != 0.0) {
          sv[j] = sv[j] / Hm[j + j * ld];
          const double t = sv[j];
          for (int r = j - 1; r >= 0; r--) sv[r] = __dsub_rn(sv[r], mul_rn(t, Hm[r + j * ld]));
        }
    }
    __syncthreads();
    // x += sum_k s(k) V_k (Add skipped when s(k) == 0)
    for (long long e = gt; e < n; e += gs) {
      double xe = __ldcg(v.x + e);
      for (int k = 0; k < i; k++)
        if (sv[k] != 0.0) xe = add_rn(xe, mul_rn(sv[k], __ldcg(v.V + (size_t)k * nn + e)));
      v.x[e] = xe;
    }
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    // w = b - A x; r = M^{-1} w; beta = ||r||
    EpiResidual epi{v.b, v.w, nullptr, 0.0, 0.0};
    spmv_phase(A, v.x, epi, s_prod, s_red);
    if (!grid_sync<NT>(P, epoch, 0, s_vals, s_red)) return;
    rr = 0.0;
    for (long long e = gt; e < n; e += gs) {
      const double re = precond_val(A.diag, (int)e, __ldcg(v.w + e));
      v.r[e] = re;
      rr = add_rn(rr, mul_rn(re, re));
    }
    rr = block_sum<NT>(rr, s_red);
    if (tid == 0) s_vals[0] = rr;
    if (!grid_sync<NT>(P, epoch, 1, s_vals, s_red)) return;
    beta = sqrt(s_vals[0]);
  }
  if (lead) write_out(out, nb_iter, it.max_iter, 0, facteur, reste, hlen);
}

// ----------------------------------------------------------------- launch glue

struct DeviceBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~DeviceBuf() {
    if (p) cudaFreeAsync(p, s);
  }
};

struct SolveScratch {
  DeviceBuf vecs, state;
  double* vec = nullptr;
  GridSync* sync = nullptr;
  double* partials = nullptr;
  SolveOut* out = nullptr;
  double* hist = nullptr;
  int* hist_it = nullptr;
  int hist_cap = 0;
};

// Distance between the work vectors of one solve: n rounded up so that the
// vectors do not start a power of two apart (a solve streaming many of them
// at once, as GMRES's Gram-Schmidt passes do, would otherwise have its
// streams fall on the same L2 sets and DRAM channels when n is a power of
// two): 256 bytes past a multiple of 512.
size_t vector_stride(int n, size_t elem_bytes) {
  const size_t bytes = ((size_t)std::max(n, 1) * elem_bytes + 511) / 512 * 512 + 256;
  return bytes / elem_bytes;
}

static int alloc_scratch(cudaStream_t s, int n, int nvec, int grid, int hist_cap,
                         SolveScratch* S) {
  S->vecs.s = S->state.s = s;
  const size_t vbytes = sizeof(double) * vector_stride(n, sizeof(double)) * nvec;
  SB2_CUDA_TRY(pool_malloc((void**)&S->vecs.p, vbytes, s));
  S->vec = (double*)S->vecs.p;
  S->hist_cap = std::max(hist_cap, 1);
  const size_t sync_b = 256, part_b = sizeof(double) * kMaxRed * grid, out_b = 256;
  const size_t hist_b = sizeof(double) * S->hist_cap, hit_b = sizeof(int) * S->hist_cap;
  const size_t total = sync_b + ((part_b + 255) / 256) * 256 + out_b + ((hist_b + 255) / 256) * 256 + hit_b;
  SB2_CUDA_TRY(pool_malloc((void**)&S->state.p, total, s));
  char* c = (char*)S->state.p;
  S->sync = (GridSync*)c;
  c += sync_b;
  S->partials = (double*)c;
  c += ((part_b + 255) / 256) * 256;
  S->out = (SolveOut*)c;
  c += out_b;
  S->hist = (double*)c;
  c += ((hist_b + 255) / 256) * 256;
  S->hist_it = (int*)c;
  SB2_CUDA_TRY(cudaMemsetAsync(S->state.p, 0, sync_b + ((part_b + 255) / 256) * 256 + out_b, s));
  return SB2_OK;
}

static int coop_grid(const void* kernel, size_t smem, const sb2_csr* A) {
  const int dev = current_device();
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NT, smem) != cudaSuccess ||
      per_sm < 1)
    return 0;
  const int cap = per_sm * num_sms(dev);
  const int n = A->m;
  // enough CTAs to cover the work, no more: a small grid makes the barriers cheap
  const int want = std::max((n + NT * 4 - 1) / (NT * 4), (A->full.part.nblk + 1) / 2);
  return std::max(1, std::min(cap, want));
}

static int finish_solve(SolveScratch& S, cudaStream_t s, sb2_iter_result* res, double* hist,
                        int* hist_it, int hist_cap, int max_iter) {
  SolveOut o;
  GridSync gsync;
  SB2_CUDA_TRY(cudaMemcpyAsync(&o, S.out, sizeof(o), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaMemcpyAsync(&gsync, S.sync, sizeof(gsync), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  if (gsync.status != 0) return SB2_ERR_TIMEOUT;
  const int nh = std::min(o.hist_len, hist_cap);
  if (hist && nh > 0) SB2_CUDA_TRY(cudaMemcpy(hist, S.hist, sizeof(double) * nh, cudaMemcpyDeviceToHost));
  if (hist_it && nh > 0) SB2_CUDA_TRY(cudaMemcpy(hist_it, S.hist_it, sizeof(int) * nh, cudaMemcpyDeviceToHost));
  res->nb_iter = o.nb_iter;
  // a zero right-hand side returns ErrorCode() of an untouched Iteration
  res->error_code = o.init_failed ? (max_iter <= 0 ? -2 : 0) : o.error_code;
  res->init_failed = o.init_failed;
  res->hist_len = nh;
  res->facteur_reste = o.facteur_reste;
  res->last_residual = o.last_residual;
  return SB2_OK;
}

SellOp<double> sell_op(const CsrArrays& a);

static OpArgs op_args(const sb2_csr* A, const double* diag) {
  const CsrArrays& f = A->full;
  return OpArgs{f.d_ptr, f.d_ind, f.d_val, f.part.d_blk, f.part.d_kind, f.part.nblk, A->m, diag,
                sell_op(f)};
}

enum Solver {
  kCg = 0, kBicg = 1, kGmres = 2, kCgs = 3, kTfqmr = 4, kMinres = 5, kGcr = 6, kBicgl = 7,
  kQcgs = 8, kBcg = 9,  // kBicg is BiCgStab, kBcg BiCg
  kCgne = 10, kBcr = 11, kLsqr = 12, kQmrs = 13,  // kBcr BiCgcr, kQmrs QmrSym
  kSymm = 14                                     // Symmlq
};

static int fused_solve(int which, const sb2_csr* A, const double* diag, double* x,
                       const double* b, const sb2_iter_params* prm, sb2_iter_result* res,
                       double* hist, int* hist_it, int hist_cap, cudaStream_t s) {
  const int n = A->m;
  const int m = std::max(prm->restart, 1);
  const void* kern = nullptr;
  size_t smem = 0;
  int nvec = 0;
  if (which == kCg) { kern = (const void*)cg_fused_kernel; nvec = 3; }
  if (which == kBicg) { kern = (const void*)bicgstab_fused_kernel; nvec = 9; }
  if (which == kCgs) { kern = (const void*)cgs_fused_kernel; nvec = 8; }
  if (which == kTfqmr) { kern = (const void*)tfqmr_fused_kernel; nvec = 8; }
  if (which == kMinres) { kern = (const void*)minres_fused_kernel; nvec = 9; }
  if (which == kGcr) { kern = (const void*)gcr_fused_kernel; nvec = 1 + 2 * (std::max(prm->restart, 0) + 1); }
  if (which == kBicgl) { kern = (const void*)bicgstabl_fused_kernel; nvec = 2 + 2 * (prm->restart + 1); }
  if (which == kQcgs) { kern = (const void*)qcgs_fused_kernel; nvec = 10; }
  if (which == kBcr) { kern = (const void*)bicgcr_fused_kernel; nvec = 6; }
  if (which == kQmrs) { kern = (const void*)qmrsym_fused_kernel; nvec = 7; }
  if (which == kSymm) { kern = (const void*)symmlq_fused_kernel; nvec = 8; }
  if (which == kBcg || which == kCgne || which == kLsqr) {
    kern = which == kBcg    ? (const void*)bicg_fused_kernel
           : which == kCgne ? (const void*)cgne_fused_kernel
                            : (const void*)lsqr_fused_kernel;
    nvec = which == kBcg ? 6 : which == kCgne ? 4 : 5;
    if (!A->sym) SB2_TRY(ensure_transpose(A));
  }
  if (which == kGmres) {
    kern = (const void*)gmres_fused_kernel;
    nvec = 2 + (m + 1);
    smem = sizeof(double) * ((size_t)(m + 1) * (m + 1) + 3 * (m + 1));
    if (smem > 160 * 1024) return SB2_ERR_NOT_SUPPORTED;
    SB2_CUDA_TRY(cudaFuncSetAttribute(gmres_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  }
  const int grid = coop_grid(kern, smem, A);
  if (grid < 1) return SB2_ERR_CUDA;
  SolveScratch S;
  // history: every Finished() test; GMRES tests once per inner step and once
  // per restart
  const int hcap = std::max(hist_cap, 0) + 1;
  SB2_TRY(alloc_scratch(s, n, nvec, grid, hcap, &S));
  Persist P{S.sync, S.partials, barrier_wait_ns()};
  History H{S.hist, S.hist_it, hcap};
  IterArgs it{prm->tol, prm->max_iter,
              which == kGcr ? std::max(prm->restart, 0) : which == kBicgl ? prm->restart : m,
              prm->init_guess_null};
  OpArgs op = op_args(A, diag);
  const size_t nn = vector_stride(n, sizeof(double));
  double* V = S.vec;
  void* args[6];
  CgVecs cv;
  BicgVecs bv;
  GmresVecs gv;
  CgsVecs sv;
  TfqmrVecs tv;
  MinresVecs mv;
  GcrVecs rv;
  BicglVecs lv;
  QcgsVecs qv;
  BcgVecs gcv;
  CgneVecs nev;
  BcrVecs crv;
  LsqrVecs lsv;
  QmrsVecs qsv;
  SymmlqVecs syv;
  args[0] = &op;
  args[2] = &it;
  args[3] = &P;
  args[4] = &H;
  args[5] = &S.out;
  if (which == kCg) {
    cv = CgVecs{b, x, V, V + nn, V + 2 * nn};
    args[1] = &cv;
  } else if (which == kBicg) {
    bv = BicgVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn, V + 6 * nn,
                  V + 7 * nn};
    args[1] = &bv;
  } else if (which == kCgs) {
    sv = CgsVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn, V + 6 * nn,
                 V + 7 * nn};
    args[1] = &sv;
  } else if (which == kTfqmr) {
    tv = TfqmrVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn, V + 6 * nn,
                   V + 7 * nn};
    args[1] = &tv;
  } else if (which == kMinres) {
    mv = MinresVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn, V + 6 * nn,
                    V + 7 * nn, V + 8 * nn};
    args[1] = &mv;
  } else if (which == kGcr) {
    const int mg = std::max(prm->restart, 0);
    rv = GcrVecs{b, x, V, V + nn, V + (size_t)(mg + 2) * nn, (long long)nn};
    args[1] = &rv;
  } else if (which == kBicgl) {
    lv = BicglVecs{b, x, V, V + nn, V + 2 * nn, V + (size_t)(prm->restart + 3) * nn, (long long)nn};
    args[1] = &lv;
  } else if (which == kQcgs) {
    qv = QcgsVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn, V + 6 * nn,
                  V + 7 * nn, V + 8 * nn, V + 9 * nn};
    args[1] = &qv;
  } else if (which == kBcr) {
    crv = BcrVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn};
    args[1] = &crv;
  } else if (which == kSymm) {
    syv = SymmlqVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn, V + 6 * nn,
                     V + 7 * nn};
    args[1] = &syv;
  } else if (which == kQmrs) {
    qsv = QmrsVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn, V + 6 * nn};
    args[1] = &qsv;
  } else if (which == kBcg || which == kCgne || which == kLsqr) {
    // Seldon's transpose of RowSymSparse storage is the matrix itself
    const CsrArrays& t = A->sym ? A->full : A->trans;
    const OpArgs at{t.d_ptr, t.d_ind, t.d_val, t.part.d_blk, t.part.d_kind, t.part.nblk, A->m,
                    diag, sell_op(t)};
    if (which == kBcg) {
      gcv = BcgVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, V + 5 * nn, at};
      args[1] = &gcv;
    } else if (which == kCgne) {
      nev = CgneVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, at};
      args[1] = &nev;
    } else {
      lsv = LsqrVecs{b, x, V, V + nn, V + 2 * nn, V + 3 * nn, V + 4 * nn, at};
      args[1] = &lsv;
    }
  } else {
    gv = GmresVecs{b, x, V, V + nn, V + 2 * nn, (long long)nn};
    args[1] = &gv;
  }
  SB2_CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(NT), args, smem, s));
  return finish_solve(S, s, res, hist, hist_it, hcap - 1 > 0 ? hcap - 1 : 0, prm->max_iter);
}

// ----------------------------------------------------------------- host-driven drivers (SOR)

struct HostIter {
  double tol, facteur = 0.0;
  int max_iter, nb_iter = 0, fail = 0;
  std::vector<std::pair<int, double>> hist;
  bool finished(double res) {
    const double reste = facteur * res;
    hist.emplace_back(nb_iter, reste);
    return reste < tol || nb_iter >= max_iter;
  }
  int code() const { return nb_iter >= max_iter ? -2 : fail; }
};

struct Ops {
  const sb2_csr* A;
  const sb2_precond* M;
  cudaStream_t s;
  int n;
  RedScratch* rs = nullptr;
  int dot(const double* x, const double* y, double* out) { return sb2_dot(n, x, y, out, s); }
  int nrm(const double* x, double* out) { return sb2_nrm2(n, x, out, s); }
  int axpy(double a, const double* x, double* y) { return sb2_axpy(n, a, x, y, s); }
  int scal(double a, double* x) { return sb2_scal(n, a, x, s); }
  int copy(const double* x, double* y) { return sb2_copy(n, x, y, s); }
  int mlt(const double* x, double* y) { return sb2_mlt(A, 0, 1.0, x, y, s); }
  int residual(const double* b, const double* x, double* r) {
    SB2_TRY(copy(b, r));
    return sb2_spmv(A, 0, -1.0, x, 1.0, r, s);
  }
  // no handle is the identity (Preconditioner_Base::Solve is a Copy): Gcr
  // with a restart above the persistent kernel's reaches this loop with it
  int prec(const double* r, double* z) {
    return M ? precond_apply(M, false, r, z, s) : copy(r, z);
  }
  int prect(const double* r, double* z) {  // TransSolve
    return M ? precond_apply(M, true, r, z, s) : copy(r, z);
  }
  int mltt(const double* x, double* y) { return sb2_mlt(A, 1, 1.0, x, y, s); }
};

static int host_cg(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                   HostIter& it, double* V, int* init_failed) {
  const int n = o.n;
  double *p = V, *q = V + n, *r = V + 2 * (size_t)n, *z = V + 3 * (size_t)n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, r));
  else { SB2_TRY(o.copy(b, r)); SB2_TRY(sb2_fill(n, 0.0, x, o.s)); }
  double rho = 1.0, rho_1 = 1.0, res;
  for (;;) {
    SB2_TRY(o.nrm(r, &res));
    if (it.finished(res)) break;
    SB2_TRY(o.prec(r, z));
    SB2_TRY(o.dot(r, z, &rho));
    if (rho == 0.0) { it.fail = 1; break; }
    if (it.nb_iter == 0) SB2_TRY(o.copy(z, p));
    else {
      SB2_TRY(o.scal(rho / rho_1, p));
      SB2_TRY(o.axpy(1.0, z, p));
    }
    SB2_TRY(o.mlt(p, q));
    double delta;
    SB2_TRY(o.dot(p, q, &delta));
    if (delta == 0.0) { it.fail = 2; break; }
    const double alpha = rho / delta;
    SB2_TRY(o.axpy(alpha, p, x));
    SB2_TRY(o.axpy(-alpha, q, r));
    rho_1 = rho;
    it.nb_iter++;
  }
  return SB2_OK;
}

static int host_bicgstab(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                         HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *p = V, *phat = V + n, *s = V + 2 * n, *shat = V + 3 * n, *t = V + 4 * n,
         *v = V + 5 * n, *r = V + 6 * n, *rt = V + 7 * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, r));
  else { SB2_TRY(o.copy(b, r)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(o.copy(r, rt));
  double rho_1, rho_2 = 0.0, alpha = 0.0, omega = 0.0, res;
  for (;;) {
    SB2_TRY(o.nrm(r, &res));
    if (it.finished(res)) break;
    SB2_TRY(o.dot(rt, r, &rho_1));
    if (rho_1 == 0.0) { it.fail = 1; break; }
    if (it.nb_iter == 0) SB2_TRY(o.copy(r, p));
    else {
      if (omega == 0.0) { it.fail = 2; break; }
      const double beta = (rho_1 / rho_2) * (alpha / omega);
      SB2_TRY(o.axpy(-omega, v, p));
      SB2_TRY(o.scal(beta, p));
      SB2_TRY(o.axpy(1.0, r, p));
    }
    SB2_TRY(o.prec(p, phat));
    SB2_TRY(o.mlt(phat, v));
    double sigma;
    SB2_TRY(o.dot(rt, v, &sigma));
    if (sigma == 0.0) { it.fail = 3; break; }
    alpha = rho_1 / sigma;
    SB2_TRY(o.copy(r, s));
    SB2_TRY(o.axpy(-alpha, v, s));
    it.nb_iter++;
    SB2_TRY(o.nrm(s, &res));
    if (it.finished(res)) {
      SB2_TRY(o.axpy(alpha, phat, x));
      break;
    }
    SB2_TRY(o.prec(s, shat));
    SB2_TRY(o.mlt(shat, t));
    double ts, tt;
    SB2_TRY(o.dot(t, s, &ts));
    SB2_TRY(o.dot(t, t, &tt));
    omega = ts / tt;
    SB2_TRY(o.axpy(alpha, phat, x));
    SB2_TRY(o.axpy(omega, shat, x));
    SB2_TRY(o.copy(s, r));
    SB2_TRY(o.axpy(-omega, t, r));
    rho_2 = rho_1;
    it.nb_iter++;
  }
  return SB2_OK;
}

static int host_cgs(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                    HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *p = V, *phat = V + n, *q = V + 2 * n, *qhat = V + 3 * n, *vhat = V + 4 * n,
         *u = V + 5 * n, *uhat = V + 6 * n, *r = V + 7 * n, *rt = V + 8 * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, r));
  else { SB2_TRY(o.copy(b, r)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(o.copy(r, rt));
  double rho_1, rho_2 = 0.0, res;
  for (;;) {
    SB2_TRY(o.nrm(r, &res));
    if (it.finished(res)) break;
    SB2_TRY(o.dot(rt, r, &rho_1));
    if (rho_1 == 0.0) { it.fail = 1; break; }
    if (it.nb_iter == 0) {
      SB2_TRY(o.copy(r, u));
      SB2_TRY(o.copy(u, p));
    } else {
      const double beta = rho_1 / rho_2;
      SB2_TRY(o.copy(r, u));
      SB2_TRY(o.axpy(beta, q, u));
      SB2_TRY(o.scal(beta, p));
      SB2_TRY(o.axpy(1.0, q, p));
      SB2_TRY(o.scal(beta, p));
      SB2_TRY(o.axpy(1.0, u, p));
    }
    SB2_TRY(o.prec(p, phat));
    SB2_TRY(o.mlt(phat, vhat));
    it.nb_iter++;
    double delta;
    SB2_TRY(o.dot(rt, vhat, &delta));
    if (delta == 0.0) { it.fail = 2; break; }
    const double alpha = rho_1 / delta;
    SB2_TRY(o.copy(u, q));
    SB2_TRY(o.axpy(-alpha, vhat, q));
    SB2_TRY(o.axpy(1.0, q, u));
    SB2_TRY(o.prec(u, uhat));
    SB2_TRY(o.axpy(alpha, uhat, x));
    SB2_TRY(o.mlt(uhat, qhat));
    SB2_TRY(o.axpy(-alpha, qhat, r));
    rho_2 = rho_1;
    it.nb_iter++;
  }
  return SB2_OK;
}

static int host_tfqmr(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                      HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *tmp = V, *r0 = V + n, *v = V + 2 * n, *h = V + 3 * n, *w = V + 4 * n,
         *y1 = V + 5 * n, *g = V + 6 * n, *y0 = V + 7 * n, *rt = V + 8 * n, *d = V + 9 * n;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, tmp));
  else { SB2_TRY(o.copy(b, tmp)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(o.prec(tmp, r0));
  double tau;
  SB2_TRY(o.nrm(r0, &tau));
  if (tau == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / tau;
  SB2_TRY(o.copy(r0, w));
  SB2_TRY(o.copy(r0, y1));
  SB2_TRY(o.mlt(y1, tmp));
  SB2_TRY(o.prec(tmp, v));
  SB2_TRY(o.copy(v, g));
  SB2_TRY(sb2_fill(o.n, 0.0, d, o.s));
  SB2_TRY(o.copy(r0, rt));
  double rho, sigma, theta = 0.0, eta = 0.0;
  SB2_TRY(o.dot(rt, r0, &rho));
  for (;;) {
    SB2_TRY(o.dot(rt, v, &sigma));
    if (sigma == 0.0) { it.fail = 1; break; }
    const double alpha = rho / sigma;
    SB2_TRY(o.copy(y1, y0));
    SB2_TRY(o.axpy(-alpha, v, y0));
    SB2_TRY(o.mlt(y0, tmp));
    SB2_TRY(o.prec(tmp, h));
    SB2_TRY(o.axpy(-alpha, g, w));
    if (alpha == 0.0) { it.fail = 2; break; }
    SB2_TRY(o.scal(theta * theta * eta / alpha, d));
    SB2_TRY(o.axpy(1.0, y1, d));
    if (tau == 0.0) { it.fail = 3; break; }
    double nw;
    SB2_TRY(o.nrm(w, &nw));
    theta = nw / tau;
    double c = 1.0 / std::sqrt(1.0 + theta * theta);
    tau = tau * c * theta;
    eta = c * c * alpha;
    SB2_TRY(o.axpy(eta, d, x));
    if (it.finished(tau * std::sqrt(2. * (it.nb_iter + 1)))) break;
    it.nb_iter++;
    SB2_TRY(o.copy(h, g));
    SB2_TRY(o.axpy(-alpha, g, w));
    SB2_TRY(o.scal(theta * theta * eta / alpha, d));
    SB2_TRY(o.axpy(1.0, y0, d));
    if (tau == 0.0) { it.fail = 4; break; }
    SB2_TRY(o.nrm(w, &nw));
    theta = nw / tau;
    c = 1.0 / std::sqrt(1.0 + theta * theta);
    tau = tau * c * theta;
    eta = c * c * alpha;
    SB2_TRY(o.axpy(eta, d, x));
    if (it.finished(tau * std::sqrt(2. * (it.nb_iter + 1) + 1.))) break;
    const double rho0 = rho;
    SB2_TRY(o.dot(rt, w, &rho));
    if (rho0 == 0.0) { it.fail = 5; break; }
    const double beta = rho / rho0;
    SB2_TRY(o.copy(w, y1));
    SB2_TRY(o.axpy(beta, y0, y1));
    SB2_TRY(o.mlt(y1, tmp));
    SB2_TRY(o.prec(tmp, g));
    SB2_TRY(o.scal(beta * beta, v));
    SB2_TRY(o.axpy(beta, h, v));
    SB2_TRY(o.axpy(1.0, g, v));
    it.nb_iter++;
  }
  return SB2_OK;
}

static int host_minres(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                       HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *u_old = V, *u = V + n, *r = V + 2 * n, *v_old = V + 3 * n, *v = V + 4 * n,
         *w_old = V + 5 * n, *w = V + 6 * n, *z = V + 7 * n, *w_oold = V + 8 * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, r));
  else { SB2_TRY(o.copy(b, r)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  for (double* p : {u_old, v_old, w_old, w, w_oold}) SB2_TRY(sb2_fill(o.n, 0.0, p, o.s));
  SB2_TRY(o.prec(r, z));
  double dp;
  SB2_TRY(o.dot(r, z, &dp));
  double beta = std::sqrt(dp), eta = beta;
  SB2_TRY(o.copy(r, v));
  SB2_TRY(o.copy(z, u));
  double ibeta = 1.0 / beta;
  SB2_TRY(o.scal(ibeta, v));
  SB2_TRY(o.scal(ibeta, u));
  double c = 1.0, s = 0.0, cold = 1.0, sold = 0.0, np = nb;
  for (;;) {
    if (it.finished(np)) break;
    SB2_TRY(o.mlt(u, r));
    double alpha;
    SB2_TRY(o.dot(r, u, &alpha));
    SB2_TRY(o.prec(r, z));
    SB2_TRY(o.axpy(-alpha, v, r));
    SB2_TRY(o.axpy(-alpha, u, z));
    SB2_TRY(o.axpy(-beta, v_old, r));
    SB2_TRY(o.axpy(-beta, u_old, z));
    const double beta_old = beta;
    SB2_TRY(o.dot(r, z, &dp));
    beta = std::sqrt(dp);
    const double coold = cold, soold = sold;
    cold = c;
    sold = s;
    volatile double t0 = cold * alpha, t1 = coold * sold, t2 = t1 * beta_old;
    const double rho0 = t0 - t2;
    volatile double q0 = rho0 * rho0, q1 = beta * beta;
    const double rho1 = std::sqrt(q0 + q1);
    volatile double a0 = sold * alpha, a1 = coold * cold, a2 = a1 * beta_old;
    const double rho2 = a0 + a2;
    const double rho3 = soold * beta_old;
    if (rho1 == 0.0) { it.fail = 1; break; }
    c = rho0 / rho1;
    s = beta / rho1;
    SB2_TRY(o.copy(w_old, w_oold));
    SB2_TRY(o.copy(w, w_old));
    SB2_TRY(o.copy(u, w));
    SB2_TRY(o.axpy(-rho2, w_old, w));
    SB2_TRY(o.axpy(-rho3, w_oold, w));
    SB2_TRY(o.scal(1. / rho1, w));
    const double ceta = c * eta;
    SB2_TRY(o.axpy(ceta, w, x));
    eta = -s * eta;
    SB2_TRY(o.copy(v, v_old));
    SB2_TRY(o.copy(u, u_old));
    SB2_TRY(o.copy(r, v));
    SB2_TRY(o.copy(z, u));
    if (beta == 0.0) { it.fail = 2; break; }
    ibeta = 1.0 / beta;
    SB2_TRY(o.scal(ibeta, v));
    SB2_TRY(o.scal(ibeta, u));
    np *= std::fabs(s);
    it.nb_iter++;
  }
  return SB2_OK;
}

static int host_gcr(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                    HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  const int m = std::max(prm->restart, 0);
  double *r = V, *q = V + n, *u = V + 2 * n, *Pv = V + 3 * n, *Wv = V + (size_t)(m + 4) * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, u));
  else { SB2_TRY(o.copy(b, u)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(o.prec(u, r));
  std::vector<double> beta(m + 1, 0.0);
  double normr, res;
  SB2_TRY(o.nrm(r, &normr));
  for (;;) {
    SB2_TRY(o.nrm(r, &res));
    if (it.finished(res)) break;
    HostIter inner = it;
    inner.max_iter = it.nb_iter + m;
    SB2_TRY(o.copy(r, Pv));
    SB2_TRY(o.scal(1.0 / normr, Pv));
    int j = 0;
    for (;;) {
      SB2_TRY(o.nrm(r, &res));
      if (inner.finished(res)) break;
      double *pj = Pv + (size_t)j * n, *wj = Wv + (size_t)j * n;
      SB2_TRY(o.mlt(pj, u));
      SB2_TRY(o.prec(u, wj));
      SB2_TRY(o.dot(wj, wj, &beta[j]));
      if (beta[j] == 0.0) { it.fail = 1; break; }
      double wr;
      SB2_TRY(o.dot(wj, r, &wr));
      const double alpha = wr / beta[j];
      SB2_TRY(o.axpy(alpha, pj, x));
      SB2_TRY(o.axpy(-alpha, wj, r));
      inner.nb_iter++;
      it.nb_iter++;
      SB2_TRY(o.mlt(r, u));
      SB2_TRY(o.prec(u, q));
      double* pn = Pv + (size_t)(j + 1) * n;
      SB2_TRY(o.copy(r, pn));
      for (int i = 0; i <= j; i++) {
        double d;
        SB2_TRY(o.dot(Wv + (size_t)i * n, q, &d));
        SB2_TRY(o.axpy(-d / beta[i], Pv + (size_t)i * n, pn));
      }
      inner.nb_iter++;
      it.nb_iter++;
      j++;
    }
    it.hist = inner.hist;
    if (j == 0) break;  // the reference would repeat this cycle for ever
    SB2_TRY(o.nrm(r, &normr));
  }
  return SB2_OK;
}

static int host_bicgstabl(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                          HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  const int l = prm->restart;
  double *q = V, *r0 = V + n, *Rb = V + 2 * n, *Ub = V + (size_t)(l + 3) * n;
  auto R = [&](int i) { return Rb + (size_t)i * n; };
  auto U = [&](int i) { return Ub + (size_t)i * n; };
  const int L1 = l + 1;
  std::vector<double> tau((size_t)L1 * L1, 0.0), g(L1, 0.0), gp(L1, 0.0), gt(L1, 0.0);
  for (int i = 0; i <= l; i++) {
    SB2_TRY(sb2_fill(o.n, 0.0, R(i), o.s));
    SB2_TRY(sb2_fill(o.n, 0.0, U(i), o.s));
  }
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, R(0)));
  else { SB2_TRY(o.copy(b, R(0))); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  SB2_TRY(o.copy(R(0), r0));
  double rho_0 = 1.0, rho_1, alpha = 0.0, omega = 1.0, sigma, res;
  for (;;) {
    SB2_TRY(o.nrm(R(0), &res));
    if (it.finished(res)) break;
    const int start = it.nb_iter;
    rho_0 *= -omega;
    for (int j = 0; j < l; j++) {
      SB2_TRY(o.dot(R(j), r0, &rho_1));
      if (rho_0 == 0.0) { it.fail = 1; break; }
      const double beta = alpha * (rho_1 / rho_0);
      rho_0 = rho_1;
      for (int i = 0; i <= j; i++) {
        SB2_TRY(o.scal(-beta, U(i)));
        SB2_TRY(o.axpy(1.0, R(i), U(i)));
      }
      SB2_TRY(o.prec(U(j), q));
      SB2_TRY(o.mlt(q, U(j + 1)));
      it.nb_iter++;
      SB2_TRY(o.dot(U(j + 1), r0, &sigma));
      if (sigma == 0.0) { it.fail = 2; break; }
      alpha = rho_1 / sigma;
      SB2_TRY(o.axpy(alpha, U(0), x));
      for (int i = 0; i <= j; i++) SB2_TRY(o.axpy(-alpha, U(i + 1), R(i)));
      SB2_TRY(o.prec(R(j), q));
      SB2_TRY(o.mlt(q, R(j + 1)));
      it.nb_iter++;
    }
    for (int j = 1; j <= l; j++) {
      for (int i = 1; i < j; i++)
        if (g[i] != 0.0) {
          double d;
          SB2_TRY(o.dot(R(j), R(i), &d));
          tau[(size_t)i * L1 + j] = d / g[i];
          SB2_TRY(o.axpy(-tau[(size_t)i * L1 + j], R(i), R(j)));
        }
      SB2_TRY(o.dot(R(j), R(j), &g[j]));
      if (g[j] != 0.0) {
        double d;
        SB2_TRY(o.dot(R(0), R(j), &d));
        gp[j] = d / g[j];
      }
    }
    g[l] = gp[l];
    omega = g[l];
    for (int j = l - 1; j >= 1; j--) {
      double sg = 0.0;
      for (int i = j + 1; i <= l; i++) {
        volatile double t = tau[(size_t)j * L1 + i] * g[i];
        sg += t;
      }
      g[j] = gp[j] - sg;
    }
    for (int j = 1; j <= l - 1; j++) {
      double sg = 0.0;
      for (int i = j + 1; i <= l - 1; i++) {
        volatile double t = tau[(size_t)j * L1 + i] * g[i + 1];
        sg += t;
      }
      gt[j] = g[j + 1] + sg;
    }
    SB2_TRY(o.axpy(g[1], R(0), x));
    SB2_TRY(o.axpy(-gp[l], R(l), R(0)));
    SB2_TRY(o.axpy(-g[l], U(l), U(0)));
    for (int j = 1; j <= l - 1; j++) {
      SB2_TRY(o.axpy(-g[j], U(j), U(0)));
      SB2_TRY(o.axpy(gt[j], R(j), x));
      SB2_TRY(o.axpy(-gp[j], R(j), R(0)));
    }
    if (it.nb_iter == start) break;  // the reference may repeat this cycle for ever
  }
  SB2_TRY(o.copy(x, q));
  return o.prec(q, x);
}

static int host_qcgs(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                     HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *p = V, *q = V + n, *r = V + 2 * n, *rt = V + 3 * n, *u = V + 4 * n,
         *ph = V + 5 * n, *rq = V + 6 * n, *xq = V + 7 * n, *v = V + 8 * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, r));
  else { SB2_TRY(o.copy(b, r)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(o.copy(r, rt));
  SB2_TRY(sb2_fill(o.n, 0.0, q, o.s));
  SB2_TRY(sb2_fill(o.n, 0.0, p, o.s));
  SB2_TRY(o.copy(r, rq));
  SB2_TRY(o.copy(x, xq));
  double rho_1 = 1.0, rho_2, res;
  for (;;) {
    SB2_TRY(o.nrm(rq, &res));
    if (it.finished(res)) break;
    SB2_TRY(o.dot(rt, r, &rho_2));
    if (rho_1 == 0.0) { it.fail = 1; break; }
    const double beta = rho_2 / rho_1;
    SB2_TRY(o.copy(r, u));
    SB2_TRY(o.axpy(beta, q, u));
    SB2_TRY(o.scal(beta, p));
    SB2_TRY(o.axpy(1.0, q, p));
    SB2_TRY(o.scal(beta, p));
    SB2_TRY(o.axpy(1.0, u, p));
    SB2_TRY(o.prec(p, ph));
    SB2_TRY(o.mlt(ph, v));
    it.nb_iter++;
    double sigma;
    SB2_TRY(o.dot(rt, v, &sigma));
    if (sigma == 0.0) { it.fail = 2; break; }
    const double alpha = rho_2 / sigma;
    SB2_TRY(o.copy(u, q));
    SB2_TRY(o.axpy(-alpha, v, q));
    SB2_TRY(o.axpy(1.0, q, u));
    SB2_TRY(o.axpy(alpha, u, x));
    SB2_TRY(o.prec(u, ph));
    SB2_TRY(o.mlt(ph, u));
    SB2_TRY(o.axpy(-alpha, u, r));
    SB2_TRY(o.copy(rq, u));
    SB2_TRY(o.axpy(-1.0, r, u));
    double b00, b11, b10, ur, vr;
    SB2_TRY(o.dot(u, u, &b00));
    SB2_TRY(o.dot(v, v, &b11));
    SB2_TRY(o.dot(u, v, &b10));
    volatile double d0 = b00 * b11, d1 = b10 * b10;
    const double delta = d0 - d1;
    if (delta == 0.0) { it.fail = 3; break; }
    const double m00 = b11 / delta, m11 = b00 / delta, m10 = -b10 / delta;
    SB2_TRY(o.dot(u, r, &ur));
    SB2_TRY(o.dot(v, r, &vr));
    const double rn0 = -ur, rn1 = -vr;
    volatile double e0 = m00 * rn0, e1 = m10 * rn1, f0 = m10 * rn0, f1 = m11 * rn1;
    const double mu = e0 + e1, nu = f0 + f1;
    SB2_TRY(o.copy(r, rq));
    SB2_TRY(o.axpy(mu, u, rq));
    SB2_TRY(o.axpy(nu, v, rq));
    SB2_TRY(o.scal(mu, xq));
    SB2_TRY(o.axpy(1.0 - mu, x, xq));
    SB2_TRY(o.axpy(-nu, p, xq));
    rho_1 = rho_2;
    it.nb_iter++;
  }
  return o.prec(xq, x);
}

static int host_bicg(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                     HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *r = V, *z = V + n, *p = V + 2 * n, *q = V + 3 * n, *rt = V + 4 * n, *zt = V + 5 * n,
         *pt = V + 6 * n, *qt = V + 7 * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, r));
  else { SB2_TRY(o.copy(b, r)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(o.copy(r, rt));
  double rho_1, rho_2 = 0.0, res;
  for (;;) {
    SB2_TRY(o.nrm(r, &res));
    if (it.finished(res)) break;
    SB2_TRY(o.prec(r, z));
    SB2_TRY(o.prect(rt, zt));
    SB2_TRY(o.dot(z, rt, &rho_1));
    if (rho_1 == 0.0) { it.fail = 1; break; }
    if (it.nb_iter == 0) {
      SB2_TRY(o.copy(z, p));
      SB2_TRY(o.copy(zt, pt));
    } else {
      const double beta = rho_1 / rho_2;
      SB2_TRY(o.scal(beta, p));
      SB2_TRY(o.axpy(1.0, z, p));
      SB2_TRY(o.scal(beta, pt));
      SB2_TRY(o.axpy(1.0, zt, pt));
    }
    SB2_TRY(o.mlt(p, q));
    it.nb_iter++;
    SB2_TRY(o.mltt(pt, qt));
    double delta;
    SB2_TRY(o.dot(pt, q, &delta));
    if (delta == 0.0) { it.fail = 2; break; }
    const double alpha = rho_1 / delta;
    SB2_TRY(o.axpy(alpha, p, x));
    SB2_TRY(o.axpy(-alpha, q, r));
    SB2_TRY(o.axpy(-alpha, qt, rt));
    rho_2 = rho_1;
    it.nb_iter++;
  }
  return SB2_OK;
}

static int host_symmlq(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                       HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *r = V, *z = V + n, *w = V + 2 * n, *w_bar = V + 3 * n, *u = V + 4 * n,
         *u_old = V + 5 * n, *v = V + 6 * n, *v_old = V + 7 * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, r));
  else { SB2_TRY(o.copy(b, r)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(sb2_fill(o.n, 0.0, u_old, o.s));
  SB2_TRY(sb2_fill(o.n, 0.0, v_old, o.s));
  double ceta = 0.0, ceta_old = 0.0, ceta_oold = 0.0, c = 1.0, cold = 1.0, s = 0.0, sold = 0.0;
  SB2_TRY(o.prec(r, z));
  double dp;
  SB2_TRY(o.dot(r, z, &dp));
  double beta = std::sqrt(dp);
  const double beta1 = beta;
  double s_prod = std::fabs(beta1);
  SB2_TRY(o.copy(r, v));
  SB2_TRY(o.copy(z, u));
  SB2_TRY(o.scal(1.0 / beta, v));
  SB2_TRY(o.scal(1.0 / beta, u));
  SB2_TRY(o.copy(u, w_bar));
  double np = nb;
  it.nb_iter = 0;
  for (;;) {
    if (it.finished(np)) break;
    if (it.nb_iter != 0) {
      SB2_TRY(o.copy(v, v_old));
      SB2_TRY(o.copy(u, u_old));
      const double ib = 1.0 / beta;
      SB2_TRY(o.copy(r, v));
      SB2_TRY(o.scal(ib, v));
      SB2_TRY(o.copy(z, u));
      SB2_TRY(o.scal(ib, u));
      SB2_TRY(o.copy(w_bar, w));
      SB2_TRY(o.scal(c, w));
      SB2_TRY(o.axpy(s, u, w));
      SB2_TRY(o.scal(-s, w_bar));
      SB2_TRY(o.axpy(c, u, w_bar));
      SB2_TRY(o.axpy(ceta, w, x));
      ceta_oold = ceta_old;
      ceta_old = ceta;
    }
    SB2_TRY(o.mlt(u, r));
    double alpha;
    SB2_TRY(o.dot(u, r, &alpha));
    SB2_TRY(o.prec(r, z));
    SB2_TRY(o.axpy(-alpha, v, r));
    SB2_TRY(o.axpy(-alpha, u, z));
    SB2_TRY(o.axpy(-beta, v_old, r));
    SB2_TRY(o.axpy(-beta, u_old, z));
    const double beta_old = beta;
    SB2_TRY(o.dot(r, z, &dp));
    beta = std::sqrt(dp);
    const double coold = cold, soold = sold;
    cold = c;
    sold = s;
    const double rho0 = cold * alpha - coold * sold * beta_old;
    const double rho1 = std::sqrt(rho0 * rho0 + beta * beta);
    const double rho2 = sold * alpha + coold * cold * beta_old;
    const double rho3 = soold * beta_old;
    c = rho0 / rho1;
    s = beta / rho1;
    if (it.nb_iter == 0) ceta = beta1 / rho1;
    else ceta = -(rho2 * ceta_old + rho3 * ceta_oold) / rho1;
    s_prod *= std::fabs(s);
    np = c == 0.0 ? s_prod * 1e16 : s_prod / std::fabs(c);
    it.nb_iter++;
  }
  const double ceta_bar = c == 0.0 ? ceta * 1e15 : ceta / c;
  SB2_TRY(o.axpy(ceta_bar, w_bar, x));
  return SB2_OK;
}

static int host_qmrsym(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                       HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *r = V, *y = V + n, *v = V + 2 * n, *p = V + 3 * n, *pt = V + 4 * n, *d = V + 5 * n,
         *s = V + 6 * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, r));
  else { SB2_TRY(o.copy(b, r)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(o.copy(r, v));
  SB2_TRY(o.prec(v, y));
  double rho, ep = 0.0, theta = 0.0, gamma = 1.0, eta = -1.0;
  SB2_TRY(o.nrm(y, &rho));
  it.nb_iter = 0;
  for (;;) {
    double res;
    SB2_TRY(o.nrm(r, &res));
    if (it.finished(res)) break;
    if (rho == 0.0) { it.fail = 1; break; }
    SB2_TRY(o.scal(1. / rho, v));
    SB2_TRY(o.scal(1. / rho, y));
    double delta;
    SB2_TRY(o.dot(v, y, &delta));
    if (delta == 0.0) { it.fail = 3; break; }
    const bool first = it.nb_iter == 0;
    if (first) SB2_TRY(o.copy(y, p));
    else {
      SB2_TRY(o.scal(-(rho * delta / ep), p));
      SB2_TRY(o.axpy(1.0, y, p));
    }
    SB2_TRY(o.mlt(p, pt));
    SB2_TRY(o.dot(p, pt, &ep));
    if (ep == 0.0) { it.fail = 4; break; }
    const double beta = ep / delta;
    if (beta == 0.0) { it.fail = 5; break; }
    SB2_TRY(o.scal(-beta, v));
    SB2_TRY(o.axpy(1.0, pt, v));
    SB2_TRY(o.prec(v, y));
    const double rho_1 = rho;
    SB2_TRY(o.nrm(y, &rho));
    const double gamma_1 = gamma, theta_1 = theta;
    theta = rho / (gamma_1 * beta);
    gamma = 1.0 / std::sqrt(1.0 + theta * theta);
    if (gamma == 0.0) { it.fail = 6; break; }
    eta = -eta * rho_1 * gamma * gamma / (beta * gamma_1 * gamma_1);
    if (first) {
      SB2_TRY(o.copy(p, d));
      SB2_TRY(o.scal(eta, d));
      SB2_TRY(o.copy(pt, s));
      SB2_TRY(o.scal(eta, s));
    } else {
      const double tmp = theta_1 * theta_1 * gamma * gamma;
      SB2_TRY(o.scal(tmp, d));
      SB2_TRY(o.axpy(eta, p, d));
      SB2_TRY(o.scal(tmp, s));
      SB2_TRY(o.axpy(eta, pt, s));
    }
    SB2_TRY(o.axpy(1.0, d, x));
    SB2_TRY(o.axpy(-1.0, s, r));
    it.nb_iter++;
  }
  return SB2_OK;
}

static int host_bicgcr(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                       HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *v = V, *w = V + n, *s = V + 2 * n, *z = V + 3 * n, *p = V + 4 * n, *a = V + 5 * n;
  double nb;
  SB2_TRY(o.nrm(b, &nb));
  if (nb == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / nb;
  if (!prm->init_guess_null) SB2_TRY(o.residual(b, x, v));
  else { SB2_TRY(o.copy(b, v)); SB2_TRY(sb2_fill(o.n, 0.0, x, o.s)); }
  SB2_TRY(o.prec(v, s));
  SB2_TRY(o.copy(s, p));
  SB2_TRY(o.mlt(p, a));
  SB2_TRY(o.prec(a, w));
  it.nb_iter = 1;
  for (;;) {
    double res;
    SB2_TRY(o.nrm(v, &res));
    if (it.finished(res)) break;
    double rho, mu;
    SB2_TRY(o.dot(w, v, &rho));
    SB2_TRY(o.dot(w, a, &mu));
    if (mu == 0.0) { it.fail = 1; break; }
    const double alpha = rho / mu;
    SB2_TRY(o.axpy(alpha, p, x));
    SB2_TRY(o.axpy(-alpha, a, v));
    SB2_TRY(o.axpy(-alpha, w, s));
    SB2_TRY(o.mlt(s, z));
    double tau;
    SB2_TRY(o.dot(w, z, &tau));
    if (tau == 0.0) { it.fail = 2; break; }
    const double beta = tau / mu;
    SB2_TRY(o.scal(-beta, p));
    SB2_TRY(o.axpy(1.0, s, p));
    SB2_TRY(o.scal(-beta, a));
    SB2_TRY(o.axpy(1.0, z, a));
    SB2_TRY(o.prec(a, w));
    it.nb_iter++;
  }
  return SB2_OK;
}

static int host_cgne(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                     HostIter& it, double* V, int* init_failed) {
  const size_t n = o.n;
  double *p = V, *q = V + n, *r = V + 2 * n, *z = V + 3 * n;
  SB2_TRY(o.mltt(b, q));
  double dp;
  SB2_TRY(o.nrm(q, &dp));
  if (dp == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / dp;
  if (!prm->init_guess_null) {
    SB2_TRY(o.mlt(x, p));
    SB2_TRY(o.mltt(p, r));
    SB2_TRY(o.scal(-1.0, r));
    SB2_TRY(o.axpy(1.0, q, r));
  } else {
    SB2_TRY(o.copy(q, r));
    SB2_TRY(sb2_fill(o.n, 0.0, x, o.s));
  }
  double rho = 1.0, rho_1 = 0.0;
  for (;;) {
    if (it.finished(dp)) break;
    SB2_TRY(o.prect(r, q));
    SB2_TRY(o.prec(q, z));
    SB2_TRY(o.dot(r, z, &rho));
    if (rho == 0.0) { it.fail = 1; break; }
    if (it.nb_iter == 0) SB2_TRY(o.copy(z, p));
    else {
      SB2_TRY(o.scal(rho / rho_1, p));
      SB2_TRY(o.axpy(1.0, z, p));
    }
    SB2_TRY(o.mlt(p, q));
    SB2_TRY(o.mltt(q, z));
    double delta;
    SB2_TRY(o.dot(p, z, &delta));
    if (delta == 0.0) { it.fail = 2; break; }
    const double alpha = rho / delta;
    SB2_TRY(o.axpy(alpha, p, x));
    SB2_TRY(o.axpy(-alpha, z, r));
    rho_1 = rho;
    SB2_TRY(o.nrm(r, &dp));
    it.nb_iter += 2;
  }
  return SB2_OK;
}

static void host_genrot(double& a_in, double& b_in, double& c_, double& s_) {
  const double a = a_in, b = b_in;
  const double roe = (std::fabs(a) > std::fabs(b)) ? a : b;
  const double scal = std::fabs(a) + std::fabs(b);
  double r, z;
  if (scal != 0.0) {
    volatile double a_scl = a / scal, b_scl = b / scal;
    volatile double aa = a_scl * a_scl, bb = b_scl * b_scl;
    r = scal * std::sqrt(aa + bb);
    if (roe < 0.0) r *= -1.0;
    c_ = a / r;
    s_ = b / r;
    z = 1.0;
    if (std::fabs(a) > std::fabs(b)) z = s_;
    else if (std::fabs(b) >= std::fabs(a) && c_ != 0.0) z = 1.0 / c_;
  } else {
    c_ = 1.0; s_ = 0.0; r = 0.0; z = 0.0;
  }
  a_in = r;
  b_in = z;
}

static void host_applyrot(double& x, double& y, double c, double s) {
  volatile double cx = c * x, sy = s * y, cy = c * y, sx = s * x;
  const double temp = cx + sy;
  y = cy - sx;
  x = temp;
}

static int host_gmres(Ops& o, double* x, const double* b, const sb2_iter_params* prm,
                      HostIter& it, double* Vbuf, int* init_failed) {
  const size_t n = o.n;
  const int m = std::max(prm->restart, 1);
  const int ld = m + 1;
  double *w = Vbuf, *r = Vbuf + n, *u = Vbuf + 2 * n, *V = Vbuf + 3 * n;
  std::vector<double> Hm((size_t)ld * ld, 0.0), s(ld, 0.0), cs(ld, 0.0), sn(ld, 0.0);
  SB2_TRY(o.copy(b, w));
  if (!prm->init_guess_null) SB2_TRY(sb2_spmv(o.A, 0, -1.0, x, 1.0, w, o.s));
  else SB2_TRY(sb2_fill(o.n, 0.0, x, o.s));
  SB2_TRY(o.prec(w, r));
  double beta;
  SB2_TRY(o.nrm(r, &beta));
  if (beta == 0.0) { *init_failed = 1; return SB2_OK; }
  it.facteur = 1.0 / beta;
  it.nb_iter = 0;
  while (!it.finished(beta)) {
    SB2_TRY(o.copy(r, V));
    SB2_TRY(o.scal(1.0 / beta, V));
    std::fill(s.begin(), s.end(), 0.0);
    s[0] = beta;
    int i = 0;
    HostIter inner = it;
    inner.max_iter = it.nb_iter + m;
    bool stop;
    do {
      SB2_TRY(o.mlt(V + i * n, u));
      SB2_TRY(o.prec(u, w));
      for (int k = 0; k <= i; k++) {
        double h;
        SB2_TRY(o.dot(V + k * n, w, &h));
        Hm[k + (size_t)i * ld] = h;
        SB2_TRY(o.axpy(-h, V + k * n, w));
      }
      double hi;
      SB2_TRY(o.nrm(w, &hi));
      SB2_TRY(o.copy(w, V + (i + 1) * n));
      if (hi != 0.0) SB2_TRY(o.scal(1.0 / hi, V + (i + 1) * n));
      for (int k = 0; k < i; k++) host_applyrot(Hm[k + (size_t)i * ld], Hm[k + 1 + (size_t)i * ld], cs[k], sn[k]);
      if (hi != 0.0) {
        host_genrot(Hm[i + (size_t)i * ld], hi, cs[i], sn[i]);
        host_applyrot(s[i], s[i + 1], cs[i], sn[i]);
      }
      inner.nb_iter++;
      it.nb_iter++;
      i++;
      stop = inner.finished(std::fabs(s[i]));
    } while (!stop);
    it.hist = inner.hist;
    for (int j = i - 1; j >= 0; j--)
      if (s[j] != 0.0) {
        s[j] = s[j] / Hm[j + (size_t)j * ld];
        const double t = s[j];
        for (int q = j - 1; q >= 0; q--) {
          volatile double tq = t * Hm[q + (size_t)j * ld];
          s[q] = s[q] - tq;
        }
      }
    for (int k = 0; k < i; k++) SB2_TRY(o.axpy(s[k], V + k * n, x));
    SB2_TRY(o.copy(b, w));
    SB2_TRY(sb2_spmv(o.A, 0, -1.0, x, 1.0, w, o.s));
    SB2_TRY(o.prec(w, r));
    SB2_TRY(o.nrm(r, &beta));
  }
  return SB2_OK;
}

static int host_solve(int which, const sb2_csr* A, const sb2_precond* M, double* x,
                      const double* b, const sb2_iter_params* prm, sb2_iter_result* res,
                      double* hist, int* hist_it, int hist_cap, cudaStream_t s) {
  const int n = A->m;
  const int m = std::max(prm->restart, 1);
  const int nvec = which == kCg ? 4
                   : which == kBicg ? 8
                   : which == kCgs ? 9
                   : which == kTfqmr ? 10
                   : which == kMinres ? 9
                   : which == kGcr ? 3 + 2 * (std::max(prm->restart, 0) + 1)
                   : which == kBicgl ? 2 + 2 * (std::max(prm->restart, 0) + 1)
                   : which == kQcgs ? 9
                   : which == kBcg ? 8
                   : which == kCgne ? 4
                   : which == kBcr ? 6
                   : which == kQmrs ? 7
                   : which == kSymm ? 8
                                      : 3 + m + 1;
  DeviceBuf buf;
  buf.s = s;
  SB2_CUDA_TRY(pool_malloc((void**)&buf.p, sizeof(double) * (size_t)std::max(n, 1) * nvec, s));
  Ops o{A, M, s, n};
  HostIter it;
  it.tol = prm->tol;
  it.max_iter = prm->max_iter;
  int init_failed = 0;
  double* V = (double*)buf.p;
  if (which == kCg) SB2_TRY(host_cg(o, x, b, prm, it, V, &init_failed));
  else if (which == kBicg) SB2_TRY(host_bicgstab(o, x, b, prm, it, V, &init_failed));
  else if (which == kCgs) SB2_TRY(host_cgs(o, x, b, prm, it, V, &init_failed));
  else if (which == kTfqmr) SB2_TRY(host_tfqmr(o, x, b, prm, it, V, &init_failed));
  else if (which == kMinres) SB2_TRY(host_minres(o, x, b, prm, it, V, &init_failed));
  else if (which == kGcr) SB2_TRY(host_gcr(o, x, b, prm, it, V, &init_failed));
  else if (which == kBicgl) SB2_TRY(host_bicgstabl(o, x, b, prm, it, V, &init_failed));
  else if (which == kQcgs) SB2_TRY(host_qcgs(o, x, b, prm, it, V, &init_failed));
  else if (which == kBcg) SB2_TRY(host_bicg(o, x, b, prm, it, V, &init_failed));
  else if (which == kCgne) SB2_TRY(host_cgne(o, x, b, prm, it, V, &init_failed));
  else if (which == kBcr) SB2_TRY(host_bicgcr(o, x, b, prm, it, V, &init_failed));
  else if (which == kQmrs) SB2_TRY(host_qmrsym(o, x, b, prm, it, V, &init_failed));
  else if (which == kSymm) SB2_TRY(host_symmlq(o, x, b, prm, it, V, &init_failed));
  else SB2_TRY(host_gmres(o, x, b, prm, it, V, &init_failed));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  res->init_failed = init_failed;
  res->nb_iter = init_failed ? 0 : it.nb_iter;
  res->error_code = init_failed ? (prm->max_iter <= 0 ? -2 : 0) : it.code();
  res->facteur_reste = it.facteur;
  res->last_residual = it.hist.empty() ? 0.0 : it.hist.back().second;
  const int nh = std::min((int)it.hist.size(), std::max(hist_cap, 0));
  for (int k = 0; k < nh; k++) {
    if (hist) hist[k] = it.hist[k].second;
    if (hist_it) hist_it[k] = it.hist[k].first;
  }
  res->hist_len = nh;
  return SB2_OK;
}

template <typename VT>
long long chain_part_slots(const SellOp<VT>& S, int n);
template <typename T, typename VT>
int chain_cg(const SellOp<VT>& S, int n, const T* diag, T* x, const T* b, T* work,
             ChainState<T>* st, T* part, double* hist, int* hist_it, int hist_cap, double tol,
             int max_iter, int init_guess_null, cudaStream_t s, ChainState<T>* out);

// Systems at least this large run CG as a chain of full-occupancy kernels;
// smaller ones as one persistent kernel, where an iteration is latency-bound
// and grid barriers cost less than launches.  On a B200 the two cross near
// 3.5e6 rows (7-point Poisson, identity, us per iteration persistent /
// chained: 93.4 / 102.9 at 3.0e6 rows, 132.2 / 125.5 at 4.1e6, 224.6 / 211.9
// at 7.1e6).  BiCgStab crosses over at three times that size: its
// persistent kernel is still the faster at 7.1e6 rows (convection-diffusion,
// identity: 126.7 / 132.6 at 4.1e6, 206.2 / 210.2 at 7.1e6).
// sb2_krylov_set_config changes it.
static std::atomic<int> g_chain_min_n{3500000};
// Systems that fit one thread-block cluster's shared memory run CG there.
static std::atomic<int> g_cluster_cg{1};
static std::atomic<int> g_cluster_cap{16};  // most CTAs a cluster may take
// Cg with SOR or ILUT preconditioning runs as a device-resident chain (1) or
// host-driven, one library call per operation (0): sb2_krylov_set_pcg.
static std::atomic<int> g_pcg_device{1};

// ----------------------------------------------------------------- cluster-resident CG
//
// Small systems: the whole solve in one thread-block cluster (up to 16 CTAs on
// 16 SMs).  Each CTA keeps its block of rows of the matrix and its slice of
// every vector in shared memory; the product reads the other CTAs' slices of
// p through distributed shared memory, and the reductions exchange per-CTA
// partials through it after a hardware cluster barrier.  Every CTA sums the
// partials in rank order, so all of them take the same (deterministic)
// decisions.  The arithmetic is cg_fused_kernel's, step for step (Cg.cxx:
// 45-116): each row summed in stored order, the same fused reductions.

constexpr int NTC = 512;           // threads per CTA of the cluster kernel
constexpr int kClusterMaxRanks = 16;

struct ClusterCgArgs {
  const int* ptr;
  const int* ind;
  const double* val;
  const double* diag;  // nullptr: identity, else Jacobi
  const double* b;
  double* x;
  int n, rpc, nnz_max;  // rows per CTA, largest slice
  IterArgs it;
  History H;
  SolveOut* out;
};

__global__ void __launch_bounds__(NTC, 1) cg_cluster_kernel(ClusterCgArgs a) {
  namespace cgr = cooperative_groups;
  cgr::cluster_group cl = cgr::this_cluster();
  const int rank = (int)cl.block_rank(), C = (int)cl.num_blocks();
  const int tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double s_red[NTC / 32];
  __shared__ double s_bc[2];
  // shared layout (the same offsets in every CTA)
  double* sval = reinterpret_cast<double*>(smem);
  double* xv = sval + a.nnz_max;
  double* rv = xv + a.rpc;
  double* pv = rv + a.rpc;
  double* qv = pv + a.rpc;
  double* dg = qv + a.rpc;
  double* red = dg + a.rpc;  // [2 phases][2 values]
  int* sidx = reinterpret_cast<int*>(red + 4);  // packed (owner << 24 | local row)
  int* lptr = sidx + a.nnz_max;
  const int r0 = rank * a.rpc;
  const int nr = max(0, min(a.n, r0 + a.rpc) - r0);
  const int e0 = nr > 0 ? __ldg(a.ptr + r0) : 0;
  for (int i = tid; i <= nr; i += NTC) lptr[i] = nr > 0 ? __ldg(a.ptr + r0 + i) - e0 : 0;
  __syncthreads();
  const int nnz_l = lptr[nr];
  for (int k = tid; k < nnz_l; k += NTC) {
    const int j = __ldg(a.ind + e0 + k);
    const int q = j / a.rpc;
    sval[k] = __ldg(a.val + e0 + k);
    sidx[k] = (q << 24) | (j - q * a.rpc);
  }
  for (int i = tid; i < nr; i += NTC) {
    dg[i] = a.diag ? __ldg(a.diag + r0 + i) : 1.0;
    xv[i] = a.it.init_guess_null ? 0.0 : a.x[r0 + i];
  }
  int phase = 0;
  // sum of two per-thread values over the cluster, the same in every CTA
  auto reduce = [&](double v0, double v1, double& o0, double& o1) {
    v0 = block_sum<NTC>(v0, s_red);
    v1 = block_sum<NTC>(v1, s_red);
    double* slot = red + 2 * phase;
    if (tid == 0) {
      slot[0] = v0;
      slot[1] = v1;
    }
    cl.sync();
    if (tid == 0) {
      double t0 = 0.0, t1 = 0.0;
      for (int q = 0; q < C; q++) {
        const double* rs = cl.map_shared_rank(slot, q);
        t0 = add_rn(t0, rs[0]);
        t1 = add_rn(t1, rs[1]);
      }
      s_bc[0] = t0;
      s_bc[1] = t1;
    }
    __syncthreads();
    o0 = s_bc[0];
    o1 = s_bc[1];
    phase ^= 1;
  };
  // row i of A times the vector whose local slices are `vec`
  auto row_dot = [&](const double* vec, int i) {
    double t = 0.0;
    for (int k = lptr[i]; k < lptr[i + 1]; k++) {
      const int w = sidx[k];
      const int q = w >> 24, jj = w & 0xffffff;
      const double xj = (q == rank) ? vec[jj] : *cl.map_shared_rank(vec + jj, q);
      t = add_rn(t, mul_rn(sval[k], xj));
    }
    return t;
  };
  auto zval = [&](int i, double r) { return a.diag ? __ddiv_rn(r, dg[i]) : r; };
  const bool lead = (rank == 0 && tid == 0);
  int hlen = 0;

  // iter.Init(b): facteur_reste = 1/||b|| (Iterative.cxx:235-249)
  double acc = 0.0, unused;
  for (int i = tid; i < nr; i += NTC) {
    const double bi = __ldg(a.b + r0 + i);
    acc = add_rn(acc, mul_rn(bi, bi));
  }
  cl.sync();  // every slice is in place before any CTA reads another's
  double nb2;
  reduce(acc, 0.0, nb2, unused);
  const double normb = sqrt(nb2);
  if (normb == 0.0) {
    if (lead) {
      a.out->init_failed = 1;
      a.out->hist_len = 0;
    }
    cl.sync();
    return;
  }
  const double facteur = 1.0 / normb;
  // r = b - A x (or r = b with x = 0), with ||r||^2 and (r, z)
  double rr = 0.0, rz = 0.0;
  for (int i = tid; i < nr; i += NTC) {
    const double bi = __ldg(a.b + r0 + i);
    const double ri = a.it.init_guess_null ? bi : add_rn(bi, -row_dot(xv, i));
    rv[i] = ri;
    rr = add_rn(rr, mul_rn(ri, ri));
    rz = add_rn(rz, mul_rn(ri, zval(i, ri)));
  }
  reduce(rr, rz, rr, rz);
  double rho = rz, rho_1 = 1.0, reste;
  int nb_iter = 0, fail = 0;
  for (;;) {
    // while (!iter.Finished(r))
    reste = facteur * sqrt(rr);
    if (lead) hist_push(a.H, &hlen, nb_iter, reste);
    if (reste < a.it.tol || nb_iter >= a.it.max_iter) break;
    if (rho == 0.0) {
      fail = 1;
      break;
    }
    // p = z (first) | p = beta*p + z
    const double beta = rho / rho_1;
    for (int i = tid; i < nr; i += NTC) {
      const double z = zval(i, rv[i]);
      pv[i] = nb_iter == 0 ? z : add_rn(mul_rn(pv[i], beta), z);
    }
    cl.sync();  // p complete in every CTA before the product reads it
    // q = A p fused with delta = (p, q)
    double d = 0.0;
    for (int i = tid; i < nr; i += NTC) {
      const double t = row_dot(pv, i);
      qv[i] = t;
      d = add_rn(d, mul_rn(pv[i], t));
    }
    double delta;
    reduce(d, 0.0, delta, unused);
    if (delta == 0.0) {
      fail = 2;
      break;
    }
    const double alpha = rho / delta;
    rr = 0.0;
    rz = 0.0;
    for (int i = tid; i < nr; i += NTC) {
      if (alpha != 0.0) xv[i] = add_rn(xv[i], mul_rn(alpha, pv[i]));
      double ri = rv[i];
      if (-alpha != 0.0) {
        ri = add_rn(ri, mul_rn(-alpha, qv[i]));
        rv[i] = ri;
      }
      rr = add_rn(rr, mul_rn(ri, ri));
      rz = add_rn(rz, mul_rn(ri, zval(i, ri)));
    }
    reduce(rr, rz, rr, rz);
    rho_1 = rho;
    rho = rz;
    nb_iter++;
  }
  for (int i = tid; i < nr; i += NTC) a.x[r0 + i] = xv[i];
  if (lead) write_out(a.out, nb_iter, a.it.max_iter, fail, facteur, reste, hlen);
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// Shared memory of one CTA for `rpc` rows and a largest slice of `nnz_max`.
static size_t cluster_smem(int rpc, int nnz_max) {
  return sizeof(double) * ((size_t)nnz_max + 5 * (size_t)rpc + 4) +
         sizeof(int) * ((size_t)nnz_max + (size_t)rpc + 1);
}

// Plan (ranks, rows per CTA, largest slice) for A, from its row pointer;
// ranks = 0 when A does not fit one cluster.
static int cluster_plan(const sb2_csr* A, int* ranks, int* rpc, int* nnz_max) {
  sb2_csr* M = const_cast<sb2_csr*>(A);
  std::lock_guard<std::mutex> g(M->mu);
  const int cap = g_cluster_cap.load();
  if (M->cl_ranks < 0 || M->cl_cap != cap) {
    M->cl_ranks = 0;
    M->cl_cap = cap;
    const int n = A->m;
    if (n >= 256 && n <= kClusterMaxRanks * 4096) {
      std::vector<int> ptr(n + 1);
      SB2_CUDA_TRY(cudaMemcpy(ptr.data(), A->full.d_ptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
      int dev_smem = 0;
      cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, current_device());
      const size_t limit = (size_t)std::max(dev_smem - 1024, 0);  // static shared memory
      for (int c = std::min(kClusterMaxRanks, cap); c >= 2; c /= 2) {
        const int r = (n + c - 1) / c;
        int mx = 0;
        for (int q = 0; q < c; q++) {
          const int a0 = std::min(n, q * r), a1 = std::min(n, (q + 1) * r);
          mx = std::max(mx, ptr[a1] - ptr[a0]);
        }
        if (r < (1 << 24) && cluster_smem(r, mx) <= limit) {
          // the most SMs whose shared memory holds the system
          M->cl_ranks = c;
          M->cl_rpc = r;
          M->cl_nnz_max = mx;
          break;
        }
      }
    }
  }
  *ranks = M->cl_ranks;
  *rpc = M->cl_rpc;
  *nnz_max = M->cl_nnz_max;
  return SB2_OK;
}

static int cluster_cg_solve(const sb2_csr* A, const double* diag, double* x, const double* b,
                            const sb2_iter_params* prm, sb2_iter_result* res, double* hist,
                            int* hist_it, int hist_cap, cudaStream_t s) {
  int C = 0, rpc = 0, nnz_max = 0;
  SB2_TRY(cluster_plan(A, &C, &rpc, &nnz_max));
  if (C < 2) return SB2_ERR_NOT_SUPPORTED;
  const size_t smem = cluster_smem(rpc, nnz_max);
  SB2_CUDA_TRY(cudaFuncSetAttribute(cg_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  SB2_CUDA_TRY(cudaFuncSetAttribute(cg_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(NTC);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, cg_cluster_kernel, &cfg) != cudaSuccess ||
      clusters < 1) {
    cudaGetLastError();
    return SB2_ERR_NOT_SUPPORTED;
  }
  SolveScratch S;
  const int hcap = std::max(hist_cap, 0) + 1;
  SB2_TRY(alloc_scratch(s, A->m, 0, 1, hcap, &S));
  ClusterCgArgs args{A->full.d_ptr, A->full.d_ind, A->full.d_val, diag, b, x, A->m, rpc, nnz_max,
                     IterArgs{prm->tol, prm->max_iter, 1, prm->init_guess_null},
                     History{S.hist, S.hist_it, hcap}, S.out};
  SB2_CUDA_TRY(cudaLaunchKernelEx(&cfg, cg_cluster_kernel, args));
  return finish_solve(S, s, res, hist, hist_it, hcap - 1 > 0 ? hcap - 1 : 0, prm->max_iter);
}

static int chain_cg_solve(const sb2_csr* A, const double* diag, double* x, const double* b,
                          const sb2_iter_params* prm, sb2_iter_result* res, double* hist,
                          int* hist_it, int hist_cap, cudaStream_t s) {
  const SellOp<double> S = sell_op(A->full);
  const int n = A->m;
  const long long slots = chain_part_slots(S, n);
  const int hcap = std::max(hist_cap, 1);
  const size_t vb = sizeof(double) * 3 * (size_t)n;
  const size_t sb = 256, pb = sizeof(double) * slots, hb = sizeof(double) * hcap, ib = sizeof(int) * hcap;
  DeviceBuf buf;
  buf.s = s;
  SB2_CUDA_TRY(pool_malloc((void**)&buf.p, vb + sb + pb + hb + ib + 64, s));
  char* c = (char*)buf.p;
  double* work = (double*)c;
  ChainState<double>* st = (ChainState<double>*)(c + vb);
  double* part = (double*)(c + vb + sb);
  double* dh = (double*)(c + vb + sb + pb);
  int* dhi = (int*)(c + vb + sb + pb + hb);
  ChainState<double> o;
  SB2_TRY((chain_cg<double, double>(S, n, diag, x, b, work, st, part, dh, dhi, hcap, prm->tol,
                                    prm->max_iter, prm->init_guess_null, s, &o)));
  const int nh = std::min(o.hist_len, std::max(hist_cap, 0));
  if (hist && nh > 0) SB2_CUDA_TRY(cudaMemcpy(hist, dh, sizeof(double) * nh, cudaMemcpyDeviceToHost));
  if (hist_it && nh > 0) SB2_CUDA_TRY(cudaMemcpy(hist_it, dhi, sizeof(int) * nh, cudaMemcpyDeviceToHost));
  res->init_failed = o.init_failed;
  res->nb_iter = o.init_failed ? 0 : o.nb_iter;
  res->error_code = o.init_failed ? (prm->max_iter <= 0 ? -2 : 0)
                                  : (o.nb_iter >= prm->max_iter ? -2 : o.fail);
  res->hist_len = nh;
  res->facteur_reste = o.facteur;
  res->last_residual = o.reste;
  return SB2_OK;
}

int chain_pcg(const SellOp<double>& S, int n, const PrecondLaunch& apply, double* x,
              const double* b, double* work, ChainState<double>* st, double* part, double* hist,
              int* hist_it, int hist_cap, double tol, int max_iter, int init_guess_null,
              cudaStream_t s, ChainState<double>* out);

int PrecondLaunch::operator()(const double* r, double* z, cudaStream_t s) const {
  return precond_apply(M, trans, r, z, s);
}

// Cg with an SOR or ILUT preconditioner: the chained passes with the
// preconditioner's own launches between them, scalars on the device.
int chain_pbicgstab(const SellOp<double>& S, int n, const PrecondLaunch& apply, double* x,
                    const double* b, double* work, ChainState<double>* st, double* part,
                    double* hist, int* hist_it, int hist_cap, double tol, int max_iter,
                    int init_guess_null, cudaStream_t s, ChainState<double>* out);

int chain_pgmres(const SellOp<double>& S, int n, int m, const PrecondLaunch& apply, double* x,
                 const double* b, double* work, long long ldv, ChainState<double>* st,
                 GmresChainExtra* ex, double* hbuf, double* part, double* hist, int* hist_it,
                 int hist_cap, double tol, int max_iter, int init_guess_null, cudaStream_t s,
                 ChainState<double>* out);

// Cg, BiCgStab or Gmres with SOR or ILUT as a device-resident chain around
// the preconditioner's launches.
static int pcg_solve(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
                     const sb2_iter_params* prm, sb2_iter_result* res, double* hist,
                     int* hist_it, int hist_cap, cudaStream_t s, int which = kCg) {
  const SellOp<double> S = sell_op(A->full);
  const int n = A->m;
  const long long slots = chain_part_slots(S, n);
  const int hcap = std::max(hist_cap, 1);
  const int m = std::max(prm->restart, 1);
  const long long ldv = (long long)vector_stride(n, sizeof(double));
  // Gmres: w, r, u, V_0..V_m, then H, s, cos, sin and the extra scalars
  const size_t gh = sizeof(double) * ((size_t)(m + 1) * (m + 1) + 3 * (size_t)(m + 1)) +
                    sizeof(GmresChainExtra);
  const size_t vb = which == kGmres
                        ? sizeof(double) * (size_t)ldv * (m + 4) + (gh + 255) / 256 * 256
                        : sizeof(double) * (which == kBicg ? 8 : 4) * (size_t)n;
  const size_t sb = 256, pb = sizeof(double) * slots, hb = sizeof(double) * hcap, ib = sizeof(int) * hcap;
  DeviceBuf buf;
  buf.s = s;
  SB2_CUDA_TRY(pool_malloc((void**)&buf.p, vb + sb + pb + hb + ib + 64, s));
  char* c = (char*)buf.p;
  double* work = (double*)c;
  ChainState<double>* st = (ChainState<double>*)(c + vb);
  double* part = (double*)(c + vb + sb);
  double* dh = (double*)(c + vb + sb + pb);
  int* dhi = (int*)(c + vb + sb + pb + hb);
  ChainState<double> o;
  if (which == kGmres) {
    double* hb = work + (size_t)ldv * (m + 4);
    GmresChainExtra* ex = reinterpret_cast<GmresChainExtra*>(
        hb + (size_t)(m + 1) * (m + 1) + 3 * (size_t)(m + 1));
    SB2_TRY(chain_pgmres(S, n, m, PrecondLaunch{M, false}, x, b, work, ldv, st, ex, hb, part, dh,
                         dhi, hcap, prm->tol, prm->max_iter, prm->init_guess_null, s, &o));
  } else if (which == kBicg) {
    SB2_TRY(chain_pbicgstab(S, n, PrecondLaunch{M, false}, x, b, work, st, part, dh, dhi, hcap,
                            prm->tol, prm->max_iter, prm->init_guess_null, s, &o));
  } else {
    SB2_TRY(chain_pcg(S, n, PrecondLaunch{M, false}, x, b, work, st, part, dh, dhi, hcap,
                      prm->tol, prm->max_iter, prm->init_guess_null, s, &o));
  }
  const int nh = std::min(o.hist_len, std::max(hist_cap, 0));
  if (hist && nh > 0) SB2_CUDA_TRY(cudaMemcpy(hist, dh, sizeof(double) * nh, cudaMemcpyDeviceToHost));
  if (hist_it && nh > 0) SB2_CUDA_TRY(cudaMemcpy(hist_it, dhi, sizeof(int) * nh, cudaMemcpyDeviceToHost));
  res->init_failed = o.init_failed;
  res->nb_iter = o.init_failed ? 0 : o.nb_iter;
  res->error_code = o.init_failed ? (prm->max_iter <= 0 ? -2 : 0)
                                  : (o.nb_iter >= prm->max_iter ? -2 : o.fail);
  res->hist_len = o.init_failed ? 0 : nh;
  res->facteur_reste = o.facteur;
  res->last_residual = o.reste;
  return SB2_OK;
}

static int solve_entry(int which, const sb2_csr* A, const sb2_precond* M, double* x,
                       const double* b, const sb2_iter_params* prm, sb2_iter_result* res,
                       double* hist, int* hist_it, int hist_cap, cudaStream_t s) {
  if (!A || !prm || !res || A->m != A->n) return SB2_ERR_INVALID_VALUE;
  if (A->m > 0 && (!x || !b || x == b)) return SB2_ERR_INVALID_VALUE;
  *res = sb2_iter_result{};
  // Solvers return 0 for an empty system before touching anything (Cg.cxx:50-51)
  if (A->m <= 0) return SB2_OK;
  const int kind = M ? precond_kind(M) : SB2_PRECOND_IDENTITY;
  // ILUT holds its own factor: it may be bound to no matrix, but its order
  // must be the system's
  if (kind == SB2_PRECOND_ILUT) {
    if ((precond_matrix(M) && precond_matrix(M) != A) || precond_n(M) != A->m)
      return SB2_ERR_INVALID_VALUE;
  } else if (M && precond_matrix(M) != A) {
    return SB2_ERR_INVALID_VALUE;
  }
  if ((kind == SB2_PRECOND_SOR || kind == SB2_PRECOND_ILUT) && A->full.sell.nslice >= 0 &&
      g_pcg_device && which <= kGmres)
    return pcg_solve(A, M, x, b, prm, res, hist, hist_it, hist_cap, s, which);
  // Lsqr uses no preconditioner (Lsqr.cxx:40-135): one kernel for every kind
  if (which == kLsqr)
    return fused_solve(which, A, nullptr, x, b, prm, res, hist, hist_it, hist_cap, s);
  // l = 0 reads past the reference's one-entry gamma vector (BiCgStabl.cxx:167)
  if (which == kBicgl && prm->restart < 1) return SB2_ERR_INVALID_VALUE;
  if (kind == SB2_PRECOND_SOR || kind == SB2_PRECOND_ILUT)
    return host_solve(which, A, M, x, b, prm, res, hist, hist_it, hist_cap, s);
  // a Gcr step reduces ceil(m / 2) projections in one barrier; BiCgStabl's
  // tau lives in shared memory
  if ((which == kGcr && prm->restart > kGcrMaxRestart) ||
      (which == kBicgl && prm->restart > kBicglMax))
    return host_solve(which, A, M, x, b, prm, res, hist, hist_it, hist_cap, s);
  const double* diag = nullptr;
  if (kind == SB2_PRECOND_JACOBI) {
    SB2_TRY(ensure_diag(A));
    diag = A->d_diag;
  }
  if (which == kCg && A->m >= g_chain_min_n && A->full.sell.nslice >= 0)
    return chain_cg_solve(A, diag, x, b, prm, res, hist, hist_it, hist_cap, s);
  if (which == kBicg && (long long)A->m >= 3LL * g_chain_min_n && A->full.sell.nslice >= 0)
    return pcg_solve(A, kind == SB2_PRECOND_IDENTITY ? nullptr : M, x, b, prm, res, hist, hist_it,
                     hist_cap, s, kBicg);
  if (which == kCg && g_cluster_cg) {
    const int st = cluster_cg_solve(A, diag, x, b, prm, res, hist, hist_it, hist_cap, s);
    if (st != SB2_ERR_NOT_SUPPORTED) return st;
  }
  return fused_solve(which, A, diag, x, b, prm, res, hist, hist_it, hist_cap, s);
}

}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_krylov_set_cluster(int on) try {
  const int old = g_cluster_cg ? g_cluster_cap.load() : 0;
  g_cluster_cg = on ? 1 : 0;
  if (on >= 2) {
    int c = 2;
    while (c * 2 <= std::min(on, kClusterMaxRanks)) c *= 2;
    g_cluster_cap = c;
  } else if (on == 1) {
    g_cluster_cap = kClusterMaxRanks;
  }
  return old;
} SB2_CATCH

int sb2_krylov_set_pcg(int device_resident) try {
  const int old = g_pcg_device;
  g_pcg_device = device_resident ? 1 : 0;
  return old;
} SB2_CATCH

int sb2_krylov_set_config(int chain_min_n) try {
  if (chain_min_n < 0) return SB2_ERR_INVALID_VALUE;
  const int old = g_chain_min_n;
  g_chain_min_n = chain_min_n;
  return old;
} SB2_CATCH

int sb2_cg(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
           const sb2_iter_params* params, sb2_iter_result* result, double* hist, int* hist_it,
           int hist_cap, void* stream) try {
  SB2_TRACE("sb2_cg");
  return solve_entry(kCg, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_bicgstab(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
                 const sb2_iter_params* params, sb2_iter_result* result, double* hist,
                 int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_bicgstab");
  return solve_entry(kBicg, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_gmres(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
              const sb2_iter_params* params, sb2_iter_result* result, double* hist,
              int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_gmres");
  return solve_entry(kGmres, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_cgs(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
            const sb2_iter_params* params, sb2_iter_result* result, double* hist, int* hist_it,
            int hist_cap, void* stream) try {
  SB2_TRACE("sb2_cgs");
  return solve_entry(kCgs, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_tfqmr(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
              const sb2_iter_params* params, sb2_iter_result* result, double* hist,
              int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_tfqmr");
  return solve_entry(kTfqmr, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_minres(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
               const sb2_iter_params* params, sb2_iter_result* result, double* hist,
               int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_minres");
  return solve_entry(kMinres, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_gcr(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
            const sb2_iter_params* params, sb2_iter_result* result, double* hist, int* hist_it,
            int hist_cap, void* stream) try {
  SB2_TRACE("sb2_gcr");
  return solve_entry(kGcr, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

// CoCg (CoCg.cxx:45-116) in real arithmetic is Cg step for step (the same
// dots without conjugation, the same updates and tests), so it runs Cg's
// engines; the two give the same bits in the reference too.
int sb2_cocg(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_cocg");
  return solve_entry(kCg, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_symmlq(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
               const sb2_iter_params* params, sb2_iter_result* result, double* hist,
               int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_symmlq");
  return solve_entry(kSymm, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_qmrsym(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
               const sb2_iter_params* params, sb2_iter_result* result, double* hist,
               int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_qmrsym");
  return solve_entry(kQmrs, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_lsqr(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_lsqr");
  return solve_entry(kLsqr, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_bicgcr(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
               const sb2_iter_params* params, sb2_iter_result* result, double* hist,
               int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_bicgcr");
  return solve_entry(kBcr, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_cgne(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_cgne");
  return solve_entry(kCgne, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_bicg(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_bicg");
  return solve_entry(kBcg, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_qcgs(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_qcgs");
  return solve_entry(kQcgs, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

int sb2_bicgstabl(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
                  const sb2_iter_params* params, sb2_iter_result* result, double* hist,
                  int* hist_it, int hist_cap, void* stream) try {
  SB2_TRACE("sb2_bicgstabl");
  return solve_entry(kBicgl, A, M, x, b, params, result, hist, hist_it, hist_cap,
                     (cudaStream_t)stream);
} SB2_CATCH

}  // extern "C"

// ----------------------------------------------------------------- no-allocation CG

namespace sb2 {

// Scratch of sb2_cg_noalloc: the three work vectors, the reduction slots, the
// barrier word and the result record, for systems of up to kNoAllocMaxN
// rows.  It is a file-scope device array, so it exists on every GPU that
// loads this library (about 3.2 MB each) until the process exits, and every
// call on a GPU reuses the same array.
constexpr int kNoAllocMaxN = 131072;
constexpr int kNoAllocMaxGrid = 2048;
constexpr size_t kNoAllocVec = 3 * (size_t)kNoAllocMaxN;
constexpr size_t kNoAllocPart = (size_t)kMaxRed * kNoAllocMaxGrid;
constexpr size_t kNoAllocDoubles = kNoAllocVec + kNoAllocPart + 64 + 64 + 16;
static __device__ __align__(256) double g_cg_noalloc_scratch[kNoAllocDoubles];

// Device address of the scratch on the current device.  Host code cannot use
// the array's name as a device address, so the address is looked up once per
// device (with that device current) and remembered.
static int cg_noalloc_scratch(double** out) {
  static std::mutex mu;
  static double* addr[128] = {};
  const int dev = current_device();
  if (dev < 0 || dev >= 128) return SB2_ERR_INVALID_VALUE;
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_cg_noalloc_scratch);
    if (e != cudaSuccess) return map_cuda_error(e);
    addr[dev] = static_cast<double*>(p);
  }
  *out = addr[dev];
  return SB2_OK;
}

static int cg_noalloc(const sb2_csr* A, double* x, const double* b, const sb2_iter_params* prm,
                      sb2_iter_result* res, cudaStream_t s) {
  if (!A || !prm || !res || A->m != A->n) return SB2_ERR_INVALID_VALUE;
  if (A->m > kNoAllocMaxN) return SB2_ERR_INVALID_VALUE;  // beyond the scratch
  if (A->m > 0 && (!x || !b || x == b)) return SB2_ERR_INVALID_VALUE;
  *res = sb2_iter_result{};
  if (A->m <= 0) return SB2_OK;
  const int grid = coop_grid((const void*)cg_fused_kernel, 0, A);
  if (grid < 1) return SB2_ERR_CUDA;
  if (grid > kNoAllocMaxGrid) return SB2_ERR_NOT_SUPPORTED;
  double* base = nullptr;
  SB2_TRY(cg_noalloc_scratch(&base));
  const size_t n = (size_t)A->m;
  double* vec = base;
  double* partials = base + kNoAllocVec;
  GridSync* sync = reinterpret_cast<GridSync*>(partials + kNoAllocPart);
  SolveOut* out = reinterpret_cast<SolveOut*>(partials + kNoAllocPart + 64);
  double* hist = partials + kNoAllocPart + 128;
  int* hist_it = reinterpret_cast<int*>(hist + 8);
  // the barrier word and the result record must start at zero on every call
  SB2_CUDA_TRY(cudaMemsetAsync(sync, 0, sizeof(double) * 128, s));
  Persist P{sync, partials, barrier_wait_ns()};
  History H{hist, hist_it, 1};
  IterArgs it{prm->tol, prm->max_iter, std::max(prm->restart, 1), prm->init_guess_null};
  OpArgs op = op_args(A, nullptr);
  CgVecs cv{b, x, vec, vec + n, vec + 2 * n};
  void* args[6] = {&op, &cv, &it, &P, &H, &out};
  SB2_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)cg_fused_kernel, dim3(grid), dim3(NT),
                                           args, 0, s));
  SolveOut o;
  GridSync gs;
  SB2_CUDA_TRY(cudaMemcpyAsync(&o, out, sizeof(o), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaMemcpyAsync(&gs, sync, sizeof(gs), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  if (gs.status != 0) return SB2_ERR_TIMEOUT;
  res->nb_iter = o.nb_iter;
  res->error_code = o.init_failed ? (prm->max_iter <= 0 ? -2 : 0) : o.error_code;
  res->init_failed = o.init_failed;
  res->hist_len = 0;
  res->facteur_reste = o.facteur_reste;
  res->last_residual = o.last_residual;
  return SB2_OK;
}

}  // namespace sb2

extern "C" int sb2_cg_noalloc(const sb2_csr* A, double* x, const double* b,
                              const sb2_iter_params* params, sb2_iter_result* result,
                              void* stream) try {
  return sb2::cg_noalloc(A, x, b, params, result, (cudaStream_t)stream);
} SB2_CATCH
