// Restarted GMRES(m) with classical Gram-Schmidt applied twice (CGS2), the
// second projection delayed by one step, as one cooperative persistent
// kernel, in two precisions:
//
//   VT = double  the FP64 solver (sb2_gmres_cgs2): Seldon's Gmres (Gmres.cxx:
//                44-183) with its modified Gram-Schmidt loop (:127-132)
//                replaced by two classical projections.  Same restarts,
//                Givens rotations, back-solve and stopping rule.
//   VT = float   the GMRES inner solve of the iterative refinement
//                (sb2_ir_solve, solver 1): the Arnoldi products, basis,
//                projections and their per-thread sums in FP32; the residual
//                b - A x, the solution update x += V y, the Hessenberg
//                matrix, its rotations and back-solve in FP64.  Each restart
//                is a refinement step: the cycle's FP32 Krylov space corrects
//                the FP64 x, and the next cycle starts from the FP64 residual.
//
// One Arnoldi step reads the basis twice and takes two grid barriers, where
// the modified Gram-Schmidt order reads it about once (the second touch of
// each vector comes from L2) but takes i + 2 barriers, and CGS2 done in
// order reads it three times behind three barriers.  A step projects the new
// product once and finishes the previous vector's second projection, whose
// coefficients come out of the same reduction (the low-synchronization
// DCGS2 scheme of Bielich, Langou, Thomas, Swirydowicz, Yamazaki and Boman,
// Parallel Computing 2022); the kernel's loop states the algebra.
//
// Every vector pass walks the rows each thread owns in the product (the rows
// of its SELL quad, or the warp- or CTA-bin row its product epilogue wrote),
// so a pass that reads what the product wrote needs no barrier before it.
// Grid sums are deterministic: CTA partials summed in CTA order by the last
// CTA to arrive; every wait is bounded (SB2_ERR_TIMEOUT).
#include <algorithm>
#include <cmath>

#include "givens.cuh"
#include "persist.cuh"
#include "sell.cuh"

namespace sb2 {

constexpr int NTG = 256;        // threads per CTA
constexpr int kCgs2MaxK = 32;   // basis vectors one projection covers (restart <= 32)
constexpr int kWarpsG = NTG / 32;
constexpr int kWide = 2 * kCgs2MaxK + 2;  // values one wide barrier reduces

SellOp<double> sell_op(const CsrArrays& a);
size_t vector_stride(int n, size_t elem_bytes);
int ensure_fp32(const sb2_csr* A, bool need_diag);
SellOp<float> sell_op32(const sb2_csr* A);

struct Cgs2Out {
  int nb_iter;     // Arnoldi steps (Seldon's iteration count)
  int cycles;      // restarts begun
  int error_code;  // 0, or -2 (iteration limit)
  int init_failed; // zero initial residual (FP64 form) / zero b (refinement)
  int hist_len;
  int pad;
  double facteur_reste;  // 1 / ||M^{-1} r0||
  double last_residual;  // relative residual of the last Finished() test
  double true_rel;       // ||b - A x|| / ||b|| at the last restart
};

template <typename VT>
struct Cgs2Args {
  SellOp<double> A64;    // FP64 operator: the residual b - A x
  SellOp<VT> Ain;        // the Arnoldi products' operator (same slices, VT values)
  const double* diag64;  // Jacobi diagonal (FP64), nullptr: identity
  const VT* diag_in;     // the same in VT
  const double* b;
  double* x;
  VT* V;                 // (m+1) basis vectors, `ldv` apart
  VT* w;
  VT* u;
  double* wide;          // [kWide] results of the last wide barrier
  long long ldv;
  int n, m;
  double tol, inner_tol;
  int max_iter, max_cycles, init_guess_null;
  int ir;                // 1: refinement form (see cgs2_solve)
};

#ifdef __CUDACC__

// Grid barrier that reduces K <= kWide values: each CTA deposits s_vals[0..K)
// (threads 0..K-1, one value each), the last CTA to arrive sums every value
// over the CTAs in CTA order (warp k % 8 takes value k, lanes stride over the
// CTAs, a fixed shuffle tree combines them), publishes the K sums and
// releases the grid.  On return s_vals holds the K sums in every CTA.  The
// wait is bounded like grid_sync's; false when it ran out here or elsewhere.
__device__ __forceinline__ bool grid_sync_wide(const Persist& P, double* wide, unsigned& epoch,
                                               int K, double* s_vals) {
  __shared__ int s_last, s_ok;
  const int tid = threadIdx.x;
  const unsigned G = gridDim.x;
  if (tid < K) {
    P.partials[(size_t)tid * G + blockIdx.x] = s_vals[tid];
    __threadfence();
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&P.sync->count, 1u);
    s_last = (prev == G - 1) ? 1 : 0;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    const int lane = tid & 31, warp = tid >> 5;
    for (int k = warp; k < K; k += kWarpsG) {
      const double* pv = P.partials + (size_t)k * G;
      // every load of a lane issued before the first add waits on one: one
      // round trip per value up to 512 CTAs
      double v = 0.0;
      for (unsigned g0 = lane; g0 < G; g0 += 32 * 16) {
        double part[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
          const unsigned g = g0 + 32u * q;
          part[q] = g < G ? __ldcg(pv + g) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 16; q++) v = add_rn(v, part[q]);
      }
      v = warp_sum(v);
      if (lane == 0) wide[k] = v;
    }
    if (lane == 0) __threadfence();
    __syncthreads();
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
    __threadfence();  // as grid_sync: the next phase gathers through L1
  }
  // thread 0's acquire, then the CTA barrier, orders every thread's reads
  // of the published sums after the release
  __syncthreads();
  if (tid < K) s_vals[tid] = __ldcg(wide + tid);
  if (tid == 0) s_ok = (*((volatile int*)&P.sync->status) == 0) ? 1 : 0;
  __syncthreads();
  epoch++;
  return s_ok != 0;
}

// The rows this thread writes in a product over S with (blockIdx.x,
// gridDim.x): f.quad(r0) for a lane's 4 consecutive rows r0..r0+3 with
// r0 % 4 == 0, f.row(r) for any other row.  Mirrors sell_spmv's assignment.
template <typename VT, class F>
__device__ __forceinline__ void own_rows(const SellOp<VT>& S, F& f) {
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)blockIdx.x * kWarpsG + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * kWarpsG;
  for (long long s = gw; s < S.nslice; s += nw) {
    const size_t q = (size_t)s * 32 + lane;
    const uint2 inf = __ldg(S.qinfo + q);
    if (!(inf.x & kQuadScattered)) {
      const int r0 = (int)inf.x;
      if ((r0 & 3) == 0) {
        f.quad(r0);
      } else {
        f.row(r0);
        f.row(r0 + 1);
        f.row(r0 + 2);
        f.row(r0 + 3);
      }
    } else {
      const int4 rr = __ldg(S.qrows + q);
      if (rr.x >= 0) f.row(rr.x);
      if (rr.y >= 0) f.row(rr.y);
      if (rr.z >= 0) f.row(rr.z);
      if (rr.w >= 0) f.row(rr.w);
    }
  }
  if (lane == 0)
    for (long long r = gw; r < S.nwarp_rows; r += nw) f.row(__ldg(S.wrows + r));
  if (threadIdx.x == 0)
    for (int r = blockIdx.x; r < S.ncta_rows; r += gridDim.x) f.row(__ldg(S.crows + r));
}

template <typename VT>
__device__ __forceinline__ VT precond_v(const VT* diag, int i, VT r) {
  if (!diag) return r;
  if constexpr (sizeof(VT) == 8) return __ddiv_rn(r, diag[i]);
  else return __fdiv_rn(r, diag[i]);
}

// Delayed form, product epilogue: w = M^{-1} A u (u unnormalized).
template <typename VT>
struct EpiPrecond {
  VT* w;
  const VT* diag;
  __device__ __forceinline__ void operator()(int r, VT t) { w[r] = precond_v(diag, r, t); }
  __device__ __forceinline__ void quad(int r, const VT* t) {
    VT wq[4];
#pragma unroll
    for (int j = 0; j < 4; j++) wq[j] = precond_v(diag, r + j, t[j]);
    vst4(w + r, wq);
  }
};

// Delayed form, the step's one update pass on the owned rows:
//   V_i = (u - sum_{k<i} s_k V_k) / rho        (u's delayed second projection)
//   u   = w / rho - sum_{k<=i} d_k V_k         (w's first projection, scaled)
// where V_i in the last term is the value just formed.
template <typename VT>
struct PassDelayed {
  const VT* V;
  VT* vi;
  VT* u;
  const VT* w;
  const double* sc;  // s_k (shared)
  const double* dc;  // d_k (shared)
  long long ldv;
  int i;
  VT inv_rho;
  __device__ __forceinline__ void quad(int r) {
    VT a[4], b[4], wq[4];
    vld4_cg(u + r, a);
    vld4_cg(w + r, wq);
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = mul_rn(wq[q], inv_rho);
#pragma unroll 4
    for (int k = 0; k < i; k++) {
      const VT sk = (VT)sc[k], dk = (VT)dc[k];
      VT v[4];
      vld4_cg(V + k * ldv + r, v);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        a[q] = add_rn(a[q], -mul_rn(sk, v[q]));
        b[q] = add_rn(b[q], -mul_rn(dk, v[q]));
      }
    }
    const VT di = (VT)dc[i];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      a[q] = mul_rn(a[q], inv_rho);
      b[q] = add_rn(b[q], -mul_rn(di, a[q]));
    }
    vst4(vi + r, a);
    vst4(u + r, b);
  }
  __device__ __forceinline__ void row(int r) {
    VT a = __ldcg(u + r);
    VT b = mul_rn(__ldcg(w + r), inv_rho);
#pragma unroll 4
    for (int k = 0; k < i; k++) {
      const VT v = __ldcg(V + k * ldv + r);
      a = add_rn(a, -mul_rn((VT)sc[k], v));
      b = add_rn(b, -mul_rn((VT)dc[k], v));
    }
    a = mul_rn(a, inv_rho);
    b = add_rn(b, -mul_rn((VT)dc[i], a));
    vi[r] = a;
    u[r] = b;
  }
};

// x += sum_{k < cnt} y_k V_k in FP64 on the owned rows (Add skipped for y_k == 0)
template <typename VT>
struct PassUpdate {
  const VT* V;
  double* x;
  const double* y;  // shared memory
  long long ldv;
  int cnt;
  __device__ __forceinline__ void row(int r) {
    double xr = x[r];
    for (int k = 0; k < cnt; k++)
      if (y[k] != 0.0) xr = add_rn(xr, mul_rn(y[k], (double)__ldcg(V + k * ldv + r)));
    x[r] = xr;
  }
  __device__ __forceinline__ void quad(int r) {
    row(r);
    row(r + 1);
    row(r + 2);
    row(r + 3);
  }
};

// Residual epilogue (FP64): v = b - A x; z = M^{-1} v; u = VT(z); sums of z^2, v^2
template <typename VT>
struct EpiResidualCgs2 {
  const double* b;
  const double* diag;
  VT* u;
  double zz, vv;
  __device__ __forceinline__ void operator()(int r, double t) {
    const double v = add_rn(__ldg(b + r), -t);
    const double z = diag ? __ddiv_rn(v, __ldg(diag + r)) : v;
    u[r] = (VT)z;
    zz = add_rn(zz, mul_rn(z, z));
    vv = add_rn(vv, mul_rn(v, v));
  }
};

// Null initial guess: x = 0, v = b on the owned rows
template <typename VT>
struct PassNullGuess {
  const double* b;
  const double* diag;
  double* x;
  VT* u;
  double zz, vv;
  __device__ __forceinline__ void row(int r) {
    const double v = __ldg(b + r);
    x[r] = 0.0;
    const double z = diag ? __ddiv_rn(v, __ldg(diag + r)) : v;
    u[r] = (VT)z;
    zz = add_rn(zz, mul_rn(z, z));
    vv = add_rn(vv, mul_rn(v, v));
  }
  __device__ __forceinline__ void quad(int r) {
    row(r);
    row(r + 1);
    row(r + 2);
    row(r + 3);
  }
};

// Basis vectors one pass of a step's dots covers: 8 with the FP32 basis, 4
// with FP64 (its registers then allow three CTAs per SM, which measured
// faster than two CTAs with 8)
template <typename VT>
constexpr int del_chunk() { return sizeof(VT) == 4 ? 8 : 4; }

// Delayed form, dots of one step over the owned rows: acc[2j] += (V_k, u)
// and acc[2j+1] += (V_k, w) for k = k0 + j < kend (j < del_chunk); with
// `norms`, nrm[0] += (u, u) and nrm[1] += (u, w).  Without W the w terms
// are skipped (the cycle's last step has no product).
template <typename VT, bool W>
struct PassDotsUW {
  static constexpr int kChunk = del_chunk<VT>();
  const VT* V;
  const VT* u;
  const VT* w;
  long long ldv;
  int k0, kend;
  bool norms;
  VT acc[2 * kChunk];
  VT nrm[2];
  __device__ __forceinline__ void quad(int r) {
    VT uq[4], wq[4];
    vld4_cg(u + r, uq);
    if constexpr (W) vld4_cg(w + r, wq);
    if (norms) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        nrm[0] = add_rn(nrm[0], mul_rn(uq[q], uq[q]));
        if constexpr (W) nrm[1] = add_rn(nrm[1], mul_rn(uq[q], wq[q]));
      }
    }
#pragma unroll
    for (int j = 0; j < kChunk; j++) {
      if (k0 + j < kend) {
        VT v[4];
        vld4_cg(V + (k0 + j) * ldv + r, v);
        VT a = acc[2 * j], c = acc[2 * j + 1];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          a = add_rn(a, mul_rn(v[q], uq[q]));
          if constexpr (W) c = add_rn(c, mul_rn(v[q], wq[q]));
        }
        acc[2 * j] = a;
        acc[2 * j + 1] = c;
      }
    }
  }
  __device__ __forceinline__ void row(int r) {
    const VT ur = __ldcg(u + r);
    const VT wr = W ? __ldcg(w + r) : VT(0);
    if (norms) {
      nrm[0] = add_rn(nrm[0], mul_rn(ur, ur));
      if constexpr (W) nrm[1] = add_rn(nrm[1], mul_rn(ur, wr));
    }
#pragma unroll
    for (int j = 0; j < kChunk; j++) {
      if (k0 + j < kend) {
        const VT v = __ldcg(V + (k0 + j) * ldv + r);
        acc[2 * j] = add_rn(acc[2 * j], mul_rn(v, ur));
        if constexpr (W) acc[2 * j + 1] = add_rn(acc[2 * j + 1], mul_rn(v, wr));
      }
    }
  }
};

// Delayed form, the step's reductions into s_vals (CTA sums): [2k] = (V_k, u),
// [2k+1] = (V_k, w) for k < i, [2i] = (u, u), [2i+1] = (u, w).  The basis
// goes in chunks of del_chunk vectors, one pass over the owned rows each;
// after a chunk every warp folds its lanes' sums (shuffle tree) into its own
// row of s_part and goes on, and the CTA adds the warps' rows in warp order
// once, at the end.  (Tried and slower: each warp of the CTA taking a share
// of the basis over all the CTA's rows, one pass, u and w re-read through
// L1; and lane k summing V_k over rows staged by its warp, whose loads touch
// 32 vectors at once.)
template <typename VT, bool W>
__device__ __forceinline__ void delayed_dots(const Cgs2Args<VT>& a, int i, double* s_part,
                                             double* s_vals) {
  constexpr int kChunk = del_chunk<VT>();
  const int lane = threadIdx.x & 31;
  double* mp = s_part + (threadIdx.x >> 5) * kWide;
  for (int k0 = 0; k0 < max(i, 1); k0 += kChunk) {
    PassDotsUW<VT, W> f{a.V, a.u, a.w, a.ldv, k0, i, k0 == 0, {}, {}};
    own_rows(a.Ain, f);
    const int cnt = 2 * min(kChunk, i - k0);
#pragma unroll
    for (int j = 0; j < 2 * kChunk; j++) {
      if (j < cnt) {
        const VT v = warp_sum(f.acc[j]);
        if (lane == 0) mp[2 * k0 + j] = (double)v;
      }
    }
    if (k0 == 0) {
      const VT v0 = warp_sum(f.nrm[0]), v1 = warp_sum(f.nrm[1]);
      if (lane == 0) {
        mp[2 * i] = (double)v0;
        mp[2 * i + 1] = (double)v1;
      }
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < 2 * i + 2) {
    double t = 0.0;
    for (int w = 0; w < kWarpsG; w++) t = add_rn(t, s_part[w * kWide + threadIdx.x]);
    s_vals[threadIdx.x] = t;
  }
  __syncthreads();
}

__device__ __forceinline__ void cgs2_hist(const History& h, int* len, int it, double res) {
  if (*len < h.cap) {
    h.res[*len] = res;
    h.it[*len] = it;
  }
  (*len)++;
}

static_assert(kWide <= NTG, "a wide barrier deposits one value per thread");

template <typename VT>
__global__ void __launch_bounds__(NTG, 3)
    gmres_cgs2_kernel(Cgs2Args<VT> a, Persist P, History H, Cgs2Out* out) {
  __shared__ double s_red[kWarpsG];
  __shared__ VT s_redv[kWarpsG];
  __shared__ double s_part[kWarpsG * kWide];  // every CTA reduction uses it
  __shared__ double s_vals[kWide];
  __shared__ double s_h1[kCgs2MaxK];
  __shared__ double s_h2[kCgs2MaxK + 1];
  __shared__ double s_rho[2];
  extern __shared__ double s_dyn[];
  const int m = a.m, ld = m + 1;
  double* Hm = s_dyn;         // (m+1) x (m+1), column-major, rotated in place
  double* sv = Hm + ld * ld;  // s(0..m)
  double* cs = sv + ld;       // rotations_cos
  double* sn = cs + ld;       // rotations_sin
  double* Hr = sn + ld;        // the Hessenberg matrix as built, unrotated
  const int tid = threadIdx.x;
  const bool lead = (blockIdx.x == 0 && tid == 0);
  unsigned epoch = 0;
  int hlen = 0;
  for (int k = tid; k < 2 * ld * ld + 3 * ld; k += NTG) s_dyn[k] = 0.0;

  // ||b||^2: the refinement form stops on ||b - A x|| / ||b||
  double nb = 1.0;
  if (a.ir) {
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * NTG + tid; i < a.n; i += (long long)gridDim.x * NTG) {
      const double bi = __ldg(a.b + i);
      acc = add_rn(acc, mul_rn(bi, bi));
    }
    acc = block_sum<NTG>(acc, s_red);
    if (tid == 0) s_vals[0] = acc;
    __syncthreads();
    if (!grid_sync_wide(P, a.wide, epoch, 1, s_vals)) return;
    nb = sqrt(s_vals[0]);
    if (nb == 0.0) {
      if (lead) { out->init_failed = 1; out->hist_len = 0; }
      return;
    }
  }

  // r = M^{-1}(b - A x) in FP64 (x = 0: M^{-1} b); u = r in VT; beta = ||r||
  auto residual = [&](bool null_guess, double& zz, double& vv) -> bool {
    if (null_guess) {
      PassNullGuess<VT> f{a.b, a.diag64, a.x, a.u, 0.0, 0.0};
      own_rows(a.A64, f);
      zz = f.zz;
      vv = f.vv;
    } else {
      EpiResidualCgs2<VT> e{a.b, a.diag64, a.u, 0.0, 0.0};
      XLoadCa<double> xl{a.x};
      sell_spmv<NTG, double, double>(a.A64, xl, e, s_red, blockIdx.x, gridDim.x);
      zz = e.zz;
      vv = e.vv;
    }
    zz = block_sum<NTG>(zz, s_red);
    vv = block_sum<NTG>(vv, s_red);
    if (tid == 0) { s_vals[0] = zz; s_vals[1] = vv; }
    __syncthreads();
    if (!grid_sync_wide(P, a.wide, epoch, 2, s_vals)) return false;
    zz = s_vals[0];
    vv = s_vals[1];
    return true;
  };

  double zz, vv;
  if (!residual(a.init_guess_null != 0, zz, vv)) return;
  double beta = sqrt(zz);
  if (!a.ir && beta == 0.0) {  // outer.Init(r)
    if (lead) { out->init_failed = 1; out->hist_len = 0; }
    return;
  }
  const double facteur = beta != 0.0 ? 1.0 / beta : 0.0;
  int nb_iter = 0, cycles = 0;
  double reste, true_rel = sqrt(vv) / nb;
  for (;;) {
    // outer.Finished(beta); the refinement form tests the FP64 true residual
    reste = a.ir ? true_rel : facteur * beta;
    if (lead) cgs2_hist(H, &hlen, nb_iter, reste);
    if (reste < a.tol || nb_iter >= a.max_iter || (a.ir && cycles >= a.max_cycles) || beta == 0.0)
      break;
    cycles++;
    if (tid == 0) {
      for (int k = 0; k < ld; k++) sv[k] = 0.0;
      sv[0] = beta;
    }
    const double beta_cycle = beta;
    const int inner_max = nb_iter + m;
    int i = 0;
    {
      // Delayed reorthogonalization.  Entering step i, V_0..V_{i-1} are
      // final and u is the next vector projected once, not normalized
      // (u = r at i = 0).  Step i:
      //   A. w = M^{-1} A u and the 2i+2 dots (V_k, u), (V_k, w), (u, u), (u, w)
      //      in one pass                                          -> barrier
      //      s_k = (V_k, u) is u's second projection, rho^2 = (u,u) - |s|^2;
      //      column i-1 of H becomes h + s with H(i,i-1) = rho, and its
      //      rotation gives the residual estimate of step i-1 (the stopping
      //      test, one step late: a converged cycle wastes one product);
      //   B. V_i = (u - V s) / rho and u = (w - V z - e V_i) / rho in one
      //      pass, z_k = (V_k, w), e = (V_i, w)                       -> barrier
      //      Column i's first coefficients are h_k = (z_k - t_k) / rho and
      //      h_i = (e - t_i) / rho, with t = H(:, 0..i-1) s: A V_i equals
      //      (w - A V s) / rho and A V_{0..i-1} = V H, so the projection
      //      of w stands for that of A V_i.
      // Step m has no product: it only finalizes column m-1.
      for (;;) {
        const bool prod = i < m;
        if (prod) {
          EpiPrecond<VT> e{a.w, a.diag_in};
          XLoadCa<VT> xl{a.u};
          sell_spmv<NTG, VT, VT>(a.Ain, xl, e, s_redv, blockIdx.x, gridDim.x);
          delayed_dots<VT, true>(a, i, s_part, s_vals);
        } else {
          delayed_dots<VT, false>(a, i, s_part, s_vals);
        }
        if (!grid_sync_wide(P, a.wide, epoch, 2 * i + 2, s_vals)) return;
        if (tid == 0) {
          double ss = 0.0, sz = 0.0;
          for (int k = 0; k < i; k++) {
            ss = add_rn(ss, mul_rn(s_vals[2 * k], s_vals[2 * k]));
            sz = add_rn(sz, mul_rn(s_vals[2 * k], s_vals[2 * k + 1]));
          }
          const double rho = i == 0 ? beta_cycle : sqrt(fmax(add_rn(s_vals[2 * i], -ss), 0.0));
          s_rho[0] = rho;
          s_rho[1] = (prod && rho != 0.0) ? add_rn(s_vals[2 * i + 1], -sz) / rho : 0.0;
          if (i >= 1) {  // column i-1 final: H(k,c) = h_k + s_k, H(i,c) = rho
            const int c = i - 1;
            for (int k = 0; k <= c; k++) Hr[k + c * ld] = add_rn(Hr[k + c * ld], s_vals[2 * k]);
            Hr[i + c * ld] = rho;
            for (int k = 0; k <= i; k++) Hm[k + c * ld] = Hr[k + c * ld];
            for (int k = 0; k < c; k++) apply_rot(Hm[k + c * ld], Hm[k + 1 + c * ld], cs[k], sn[k]);
            if (rho != 0.0) {
              double hc = rho;
              gen_rot(Hm[c + c * ld], hc, cs[c], sn[c]);
              apply_rot(sv[c], sv[c + 1], cs[c], sn[c]);
            }
          }
        }
        if (tid < i) s_h1[tid] = s_vals[2 * tid];
        __syncthreads();
        const double rho = s_rho[0];
        if (i >= 1) {  // inner.Finished(|s(i)|) of step i-1
          nb_iter++;
          const double rin = fabs(sv[i]);
          reste = facteur * rin;
          if (lead && !a.ir) cgs2_hist(H, &hlen, nb_iter, reste);
          bool stop = (reste < a.tol) || (nb_iter >= inner_max) || (rho == 0.0);
          if (a.ir) stop = stop || (rin <= a.inner_tol * beta_cycle) || (nb_iter >= a.max_iter);
          if (stop) break;
        }
        // column i's first coefficients (into Hr) and the update's d_k (s_h2)
        if (tid <= i) {
          double t = 0.0;
          for (int k = max(tid - 1, 0); k < i; k++) t = add_rn(t, mul_rn(Hr[tid + k * ld], s_h1[k]));
          const double zk = tid < i ? s_vals[2 * tid + 1] : s_rho[1];
          Hr[tid + i * ld] = add_rn(zk, -t) / rho;
          s_h2[tid] = zk / rho;
        }
        __syncthreads();
        {
          PassDelayed<VT> f{a.V, a.V + (long long)i * a.ldv, a.u, a.w, s_h1, s_h2, a.ldv, i,
                            (VT)(1.0 / rho)};
          own_rows(a.Ain, f);
          __syncthreads();
          if (!grid_sync_wide(P, a.wide, epoch, 0, s_vals)) return;
        }
        i++;
      }
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
    // x += sum_k s(k) V_k (FP64)
    {
      PassUpdate<VT> f{a.V, a.x, sv, a.ldv, i};
      own_rows(a.A64, f);
      __syncthreads();
      if (!grid_sync_wide(P, a.wide, epoch, 0, s_vals)) return;
    }
    if (!residual(false, zz, vv)) return;
    beta = sqrt(zz);
    true_rel = sqrt(vv) / nb;
  }
  if (lead) {
    out->nb_iter = nb_iter;
    out->cycles = cycles;
    // Iteration::ErrorCode (Iterative.cxx:344-354); the refinement form
    // reports whether its FP64 residual met tol
    out->error_code = a.ir ? ((reste < a.tol) ? 0 : -2) : ((nb_iter >= a.max_iter) ? -2 : 0);
    out->init_failed = 0;
    out->hist_len = hlen;
    out->facteur_reste = facteur;
    out->last_residual = reste;
    out->true_rel = true_rel;
  }
}

#endif  // __CUDACC__

// ----------------------------------------------------------------- host side

template <typename VT>
static int cgs2_grid(size_t smem, const SellOp<VT>& S, int n) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gmres_cgs2_kernel<VT>, NTG,
                                                    smem) !=
          cudaSuccess ||
      per_sm < 1)
    return 0;
  const int cap = per_sm * num_sms(current_device());
  // enough CTAs to cover the work, no more: a small grid makes the barriers cheap
  const long long want = std::max<long long>(((long long)n + NTG * 4 - 1) / (NTG * 4),
                                             (long long)S.ncta_rows);
  return (int)std::max<long long>(1, std::min<long long>(cap, want));
}

// One solve.  ir = 0: Seldon's Gmres stopping rule (outer test on
// ||M^{-1} r|| / ||M^{-1} r0||, max_iter on the iteration count; max_cycles
// and inner_tol unused).  ir = 1: the refinement form: stop when the FP64
// ||b - A x|| / ||b|| < tol at a restart, after max_iter Arnoldi steps or
// max_cycles restarts; a cycle also ends when its FP32 residual estimate has
// dropped by inner_tol.
template <typename VT>
static int cgs2_solve(const sb2_csr* A, const SellOp<VT>& Ain, const double* diag64,
                      const VT* diag_in, double* x, const double* b, int m, double tol,
                      double inner_tol, int max_iter, int max_cycles, int init_guess_null, int ir,
                      Cgs2Out* o, double* hist, int* hist_it, int hist_cap, cudaStream_t s) {
  const int n = A->m;
  // the Hessenberg matrix rotated and as built, s and the rotations
  const size_t smem = sizeof(double) * (2 * (size_t)(m + 1) * (m + 1) + 3 * (size_t)(m + 1));
  SB2_CUDA_TRY(cudaFuncSetAttribute(gmres_cgs2_kernel<VT>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = cgs2_grid<VT>(smem, Ain, n);
  if (grid < 1) return SB2_ERR_CUDA;
  const long long ldv = (long long)vector_stride(n, sizeof(VT));
  const int hcap = std::max(hist_cap, 0) + 1;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_vec = take(sizeof(VT) * (size_t)ldv * (size_t)(m + 3));
  const size_t o_sync = take(sizeof(GridSync));
  const size_t o_part = take(sizeof(double) * (size_t)kWide * grid);
  const size_t o_wide = take(sizeof(double) * kWide);
  const size_t o_out = take(sizeof(Cgs2Out));
  const size_t o_h = take(sizeof(double) * hcap), o_hi = take(sizeof(int) * hcap);
  struct Buf {
    void* p = nullptr;
    cudaStream_t s;
    ~Buf() {
      if (p) cudaFreeAsync(p, s);
    }
  } buf;
  buf.s = s;
  SB2_CUDA_TRY(pool_malloc(&buf.p, off, s));
  char* base = static_cast<char*>(buf.p);
  SB2_CUDA_TRY(cudaMemsetAsync(base + o_sync, 0, o_h - o_sync, s));
  VT* vec = reinterpret_cast<VT*>(base + o_vec);
  Cgs2Args<VT> args{sell_op(A->full), Ain, diag64, diag_in, b, x,
                    vec, vec + (size_t)ldv * (m + 1), vec + (size_t)ldv * (m + 2),
                    reinterpret_cast<double*>(base + o_wide), ldv, n, m, tol, inner_tol,
                    max_iter, max_cycles, init_guess_null, ir};
  Persist P{reinterpret_cast<GridSync*>(base + o_sync), reinterpret_cast<double*>(base + o_part),
            barrier_wait_ns()};
  History H{reinterpret_cast<double*>(base + o_h), reinterpret_cast<int*>(base + o_hi), hcap};
  Cgs2Out* d_out = reinterpret_cast<Cgs2Out*>(base + o_out);
  void* kargs[4] = {&args, &P, &H, &d_out};
  SB2_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)gmres_cgs2_kernel<VT>, dim3(grid),
                                           dim3(NTG), kargs, smem, s));
  GridSync gs;
  SB2_CUDA_TRY(cudaMemcpyAsync(o, d_out, sizeof(Cgs2Out), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaMemcpyAsync(&gs, base + o_sync, sizeof(gs), cudaMemcpyDeviceToHost, s));
  SB2_CUDA_TRY(cudaStreamSynchronize(s));
  if (gs.status != 0) return SB2_ERR_TIMEOUT;
  const int nh = std::min(o->hist_len, std::max(hist_cap, 0));
  if (hist && nh > 0)
    SB2_CUDA_TRY(cudaMemcpy(hist, base + o_h, sizeof(double) * nh, cudaMemcpyDeviceToHost));
  if (hist_it && nh > 0)
    SB2_CUDA_TRY(cudaMemcpy(hist_it, base + o_hi, sizeof(int) * nh, cudaMemcpyDeviceToHost));
  o->hist_len = nh;
  return SB2_OK;
}

// FP64 GMRES with CGS2 orthogonalization (identity or Jacobi).
static int gmres_cgs2(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
                      const sb2_iter_params* prm, sb2_iter_result* res, double* hist,
                      int* hist_it, int hist_cap, cudaStream_t s) {
  if (!A || !prm || !res || A->m != A->n) return SB2_ERR_INVALID_VALUE;
  if (A->m > 0 && (!x || !b || x == b)) return SB2_ERR_INVALID_VALUE;
  *res = sb2_iter_result{};
  if (A->m <= 0) return SB2_OK;
  const int kind = M ? precond_kind(M) : SB2_PRECOND_IDENTITY;
  if (kind != SB2_PRECOND_IDENTITY && kind != SB2_PRECOND_JACOBI) return SB2_ERR_NOT_SUPPORTED;
  if (M && precond_matrix(M) != A) return SB2_ERR_INVALID_VALUE;
  const int m = std::max(prm->restart, 1);
  if (m > kCgs2MaxK || A->full.sell.nslice < 0) return SB2_ERR_NOT_SUPPORTED;
  const double* diag = nullptr;
  if (kind == SB2_PRECOND_JACOBI) {
    SB2_TRY(ensure_diag(A));
    diag = A->d_diag;
  }
  Cgs2Out o{};
  SB2_TRY(cgs2_solve<double>(A, sell_op(A->full), diag, diag, x, b, m, prm->tol, 0.0,
                             prm->max_iter, 1 << 30, prm->init_guess_null, 0, &o, hist, hist_it,
                             hist_cap, s));
  res->init_failed = o.init_failed;
  res->nb_iter = o.init_failed ? 0 : o.nb_iter;
  res->error_code = o.init_failed ? (prm->max_iter <= 0 ? -2 : 0)
                                  : (o.nb_iter >= prm->max_iter ? -2 : 0);
  res->hist_len = o.init_failed ? 0 : o.hist_len;
  res->facteur_reste = o.facteur_reste;
  res->last_residual = o.last_residual;
  return SB2_OK;
}

// Iterative refinement with the GMRES inner solve (sb2_ir_solve, solver 1).
int ir_gmres_solve(const sb2_csr* A, bool jacobi, double* x, const double* b,
                   const sb2_ir_params* prm, sb2_ir_result* res, double* hist, int hist_cap,
                   cudaStream_t s) {
  const int m = prm->restart > 0 ? prm->restart : 30;
  if (m > kCgs2MaxK || A->full.sell.nslice < 0) return SB2_ERR_NOT_SUPPORTED;
  SB2_TRY(ensure_fp32(A, jacobi));
  Cgs2Out o{};
  SB2_TRY(cgs2_solve<float>(A, sell_op32(A), jacobi ? A->d_diag : nullptr,
                            jacobi ? A->d_diag32 : nullptr, x, b, m, prm->tol, prm->inner_tol,
                            prm->max_inner, prm->max_outer, prm->init_guess_null, 1, &o, hist,
                            nullptr, hist_cap, s));
  res->init_failed = o.init_failed;
  res->outer_iter = o.init_failed ? 0 : o.cycles;
  res->inner_iter = o.init_failed ? 0 : o.nb_iter;
  res->rel_residual = o.init_failed ? 0.0 : o.true_rel;
  res->error_code = o.init_failed ? 0 : (o.true_rel < prm->tol ? 0 : -2);
  res->hist_len = o.init_failed ? 0 : o.hist_len;
  return SB2_OK;
}

}  // namespace sb2

extern "C" int sb2_gmres_cgs2(const sb2_csr* A, const sb2_precond* M, double* x,
                              const double* b, const sb2_iter_params* params,
                              sb2_iter_result* result, double* hist, int* hist_it, int hist_cap,
                              void* stream) try {
  SB2_TRACE("sb2_gmres_cgs2");
  return sb2::gmres_cgs2(A, M, x, b, params, result, hist, hist_it, hist_cap,
                         (cudaStream_t)stream);
} SB2_CATCH
