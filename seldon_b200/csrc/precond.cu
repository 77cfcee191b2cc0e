// Preconditioners: identity, Jacobi, level-scheduled SOR and the ILUT apply.
//
// SOR reproduces the reference's strictly sequential sweeps
// (Relaxation_MatVect.cxx:41-95 RowSparse, :176-298 RowSymSparse) bit for
// bit: rows are grouped into wavefront levels such that every value a row
// reads is the one the sequential order would have read (true dependencies on
// already-updated rows AND anti-dependencies on rows that must still hold
// their old value), and each row repeats the reference's own operation order
// with separately rounded products.
//
// The ILUT apply runs Seldon's SolveLU (computation/solver/SparseSolver.cxx:
// 533-611 and 852-882) on a factor computed on the host.  Its loops are
// either row gathers (x_i -= v * x_c over row i) or column scatters
// (x_c -= v * x_i for each entry of row i).  Every sweep is put in gather
// form: target j collects its updates in the order the sequential loop
// would have applied them (the scatter sources in increasing or decreasing
// row order, each row's entries in stored order), and the rows are grouped
// into levels on their dependencies.  Each row then repeats the reference's
// own operations with separately rounded products, so the result is the
// reference's bit for bit.
#include <algorithm>
#include <vector>

#include "sb2_internal.cuh"

namespace sb2 {

struct LevelPlan {
  int nlev = 0;
  std::vector<int> h_lvl;      // [nlev+1] offsets into rows
  int* d_rows = nullptr;       // rows ordered by level
  int* d_lvl = nullptr;        // device copy of h_lvl
  void release() {
    cudaFree(d_rows);
    cudaFree(d_lvl);
    d_rows = d_lvl = nullptr;
    h_lvl.clear();
    nlev = 0;
  }
};

static int upload_plan(const std::vector<int>& level, int n, LevelPlan* P,
                       std::vector<int>* order = nullptr) {
  int nlev = 0;
  for (int i = 0; i < n; i++) nlev = std::max(nlev, level[i] + 1);
  P->nlev = nlev;
  P->h_lvl.assign(nlev + 1, 0);
  for (int i = 0; i < n; i++) P->h_lvl[level[i] + 1]++;
  for (int l = 0; l < nlev; l++) P->h_lvl[l + 1] += P->h_lvl[l];
  std::vector<int> rows(std::max(n, 1)), fill(P->h_lvl.begin(), P->h_lvl.end() - 1);
  for (int i = 0; i < n; i++) rows[fill[level[i]]++] = i;  // increasing row in a level
  SB2_CUDA_TRY(cudaMalloc(&P->d_rows, sizeof(int) * std::max(n, 1)));
  SB2_CUDA_TRY(cudaMalloc(&P->d_lvl, sizeof(int) * (nlev + 1)));
  SB2_CUDA_TRY(cudaMemcpy(P->d_rows, rows.data(), sizeof(int) * std::max(n, 1), cudaMemcpyHostToDevice));
  SB2_CUDA_TRY(cudaMemcpy(P->d_lvl, P->h_lvl.data(), sizeof(int) * (nlev + 1), cudaMemcpyHostToDevice));
  if (order) order->assign(rows.begin(), rows.begin() + n);
  return SB2_OK;
}

// Levels of a sequential sweep over rows in `order` (forward: increasing,
// backward: decreasing).  Row j reads x(k) for every stored k: it must come
// after k when k precedes j in the sweep (k is read updated) and before k
// when k follows j (k is read old).
static void sweep_levels(int n, const int* ptr, const int* ind, bool forward,
                         std::vector<int>& level) {
  level.assign(n, 0);
  std::vector<int> req(n, 0);
  for (int s = 0; s < n; s++) {
    const int j = forward ? s : n - 1 - s;
    int lev = req[j];
    for (int k = ptr[j]; k < ptr[j + 1]; k++) {
      const int c = ind[k];
      const bool before = forward ? (c < j) : (c > j);
      if (before) lev = std::max(lev, level[c] + 1);
    }
    level[j] = lev;
    for (int k = ptr[j]; k < ptr[j + 1]; k++) {
      const int c = ind[k];
      const bool after = forward ? (c > j) : (c < j);
      if (after) req[c] = std::max(req[c], lev + 1);
    }
  }
}

// Levels of a triangular solve: row j depends on the entries of `ptr/ind`
// on the solved side (lower: c < j, upper: c > j).
static void tri_levels(int n, const int* ptr, const int* ind, bool lower,
                       std::vector<int>& level) {
  level.assign(n, 0);
  for (int s = 0; s < n; s++) {
    const int j = lower ? s : n - 1 - s;
    int lev = 0;
    for (int k = ptr[j]; k < ptr[j + 1]; k++) {
      const int c = ind[k];
      if (lower ? (c < j) : (c > j)) lev = std::max(lev, level[c] + 1);
    }
    level[j] = lev;
  }
}

// ------------------------------------------------------------------ row ops

#ifdef __CUDACC__
// Plain loads: within one CTA (all levels in one launch) the SM's L1 holds
// the CTA's own stores, and across launches every write is visible.
__device__ __forceinline__ double ldx(const double* p) { return *p; }

// RowSparse sweep, one row (Relaxation_MatVect.cxx:69-77 / :83-91).
struct RowSparseSor {
  const int* ptr; const int* ind; const double* val; const double* diag;
  const double* b; double* x; double omega;
  __device__ void operator()(int j) const {
    double temp = 0.0;
    const double ajj = diag[j];
    for (int k = ptr[j]; k < ptr[j + 1]; k++) temp = add_rn(temp, mul_rn(val[k], ldx(x + ind[k])));
    const double xj = ldx(x + j);
    temp = add_rn(__dsub_rn(b[j], temp), mul_rn(ajj, xj));
    x[j] = add_rn(mul_rn(__dsub_rn(1.0, omega), xj), __ddiv_rn(mul_rn(omega, temp), ajj));
  }
};

__device__ __forceinline__ double sym_diag(const int* uptr, const int* uind, const double* uval, int j) {
  double ajj = 0.0;
  for (int k = uptr[j]; k < uptr[j + 1]; k++)
    if (uind[k] == j) ajj = add_rn(ajj, uval[k]);
  return ajj;
}

// RowSymSparse forward, first loop (Relaxation_MatVect.cxx:214-230):
// t_j = ((1-w)/w * ajj) * x_j + (b_j - sum_{p != j} a_jp x_p), x read old.
struct SymFwd1 {
  const int* uptr; const int* uind; const double* uval;
  const double* b; const double* x; double* t; double omega;
  __device__ void operator()(int j) const {
    double temp = 0.0, ajj = 0.0;
    for (int k = uptr[j]; k < uptr[j + 1]; k++) {
      const int p = uind[k];
      if (p == j) ajj = add_rn(ajj, uval[k]);
      else temp = add_rn(temp, mul_rn(uval[k], ldx(x + p)));
    }
    temp = __dsub_rn(b[j], temp);
    const double c = __ddiv_rn(__dsub_rn(1.0, omega), omega);
    t[j] = add_rn(mul_rn(mul_rn(c, ajj), ldx(x + j)), temp);
  }
};

// RowSymSparse forward, second loop as a gather (:232-249): x_j =
// (t_j - a_{k1 j} x_{k1} - a_{k2 j} x_{k2} ...) * (w / ajj), k increasing.
// fptr/find/fval: the full row, whose entries with column < j come first in
// increasing column order (they mirror the strict upper part).
struct SymFwd2 {
  const int* fptr; const int* find; const double* fval;
  const int* uptr; const int* uind; const double* uval;
  const double* t; double* x; double omega;
  __device__ void operator()(int j) const {
    double v = t[j];
    for (int k = fptr[j]; k < fptr[j + 1]; k++) {
      const int c = find[k];
      if (c >= j) break;
      v = __dsub_rn(v, mul_rn(fval[k], ldx(x + c)));
    }
    const double ajj = sym_diag(uptr, uind, uval, j);
    x[j] = mul_rn(v, __ddiv_rn(omega, ajj));
  }
};

// RowSymSparse backward, first loop (:257-276): y_j = sum_{k<j} a_kj x_k (old x,
// increasing k); t_j = (((1-w)/w * ajj) * x_j + b_j) - y_j.
struct SymBwd1 {
  const int* fptr; const int* find; const double* fval;
  const int* uptr; const int* uind; const double* uval;
  const double* b; const double* x; double* t; double omega;
  __device__ void operator()(int j) const {
    double y = 0.0;
    for (int k = fptr[j]; k < fptr[j + 1]; k++) {
      const int c = find[k];
      if (c >= j) break;
      y = add_rn(y, mul_rn(fval[k], ldx(x + c)));
    }
    const double ajj = sym_diag(uptr, uind, uval, j);
    const double c0 = __ddiv_rn(__dsub_rn(1.0, omega), omega);
    t[j] = __dsub_rn(add_rn(mul_rn(mul_rn(c0, ajj), ldx(x + j)), b[j]), y);
  }
};

// RowSymSparse backward, second loop (:278-294): x_j = ((t_j - sum_{p != j}
// a_jp x_p) * w) / ajj, rows decreasing, stored order.
struct SymBwd2 {
  const int* uptr; const int* uind; const double* uval;
  const double* t; double* x; double omega;
  __device__ void operator()(int j) const {
    double temp = 0.0, ajj = 0.0;
    for (int k = uptr[j]; k < uptr[j + 1]; k++) {
      const int p = uind[k];
      if (p == j) ajj = add_rn(ajj, uval[k]);
      else temp = add_rn(temp, mul_rn(uval[k], ldx(x + p)));
    }
    x[j] = __ddiv_rn(mul_rn(__dsub_rn(t[j], temp), omega), ajj);
  }
};

template <class Op>
__global__ void rows_kernel(int n, Op op) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) op(j);
}

template <class Op>
__global__ void level_kernel(int begin, int end, const int* __restrict__ rows, Op op) {
  int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (i < end) op(rows[i]);
}

// All levels in one CTA, separated by __syncthreads (small systems).
template <class Op>
__global__ void __launch_bounds__(1024) level_single_cta(int nlev, const int* __restrict__ lvl,
                                                         const int* __restrict__ rows, Op op) {
  for (int l = 0; l < nlev; l++) {
    for (int i = lvl[l] + threadIdx.x; i < lvl[l + 1]; i += blockDim.x) op(rows[i]);
    __syncthreads();
  }
}

// The same kernels for ops that take the position in level order.
template <class Op>
__global__ void level_kernel_pos(int begin, int end, Op op) {
  int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (i < end) op(i);
}

template <class Op>
__global__ void __launch_bounds__(1024) level_single_cta_pos(int nlev, const int* __restrict__ lvl,
                                                             Op op) {
  for (int l = 0; l < nlev; l++) {
    for (int i = lvl[l] + threadIdx.x; i < lvl[l + 1]; i += blockDim.x) op(i);
    __syncthreads();
  }
}

// x_j = (x_j * pre_j - v_1 x_{c1} - v_2 x_{c2} - ...) * post_j, the
// subtractions in the listed order (pre/post may be null), for a gather
// sweep whose update lists are stored in level order: position i
// holds row rows[i] and its list ptr[i]..ptr[i+1], so the row id, the list
// bounds and (through them) the entries load without waiting on each other.
struct GatherSubPacked {
  const int* rows; const int* ptr; const int* ind; const double* val;
  const double* pre; const double* post; double* x;
  __device__ void operator()(int i) const {
    const int j = rows[i];
    const int e = ptr[i + 1];
    double v = ldx(x + j);
    if (pre) v = mul_rn(v, pre[j]);
    for (int k = ptr[i]; k < e; k++) v = __dsub_rn(v, mul_rn(val[k], ldx(x + ind[k])));
    if (post) v = mul_rn(v, post[j]);
    x[j] = v;
  }
};


// One row of GetIlu0 (IlutPreconditioning.cxx:1115-1176) or, with
// `modified`, of GetMilu0 (:1178-1243), in place on the CSR values: rows
// sorted by column with the diagonal at dpos.  For each L entry (stored
// order) tl = a_ij / u_jj (1/u_jj is already stored), then a_ic -= tl * u_jc
// for the columns c of row j's U part that row i holds; MILU(0) sums the
// others into s and takes s off the diagonal.  Finally the diagonal is
// inverted.  A zero pivot is recorded in *status (row + 1) and left as it is.
struct Ilu0Row {
  const int* ptr; const int* ind; double* val; const int* dpos; int* status; int modified;
  __device__ void operator()(int i) const {
    const int d = dpos[i], e = ptr[i + 1];
    double s = 0.0;
    for (int j = ptr[i]; j < d; j++) {
      const int jr = ind[j];
      const double tl = mul_rn(ldx(val + j), ldx(val + dpos[jr]));
      val[j] = tl;
      int q = j + 1;
      for (int k = dpos[jr] + 1; k < ptr[jr + 1]; k++) {
        const int c = ind[k];
        while (q < e && ind[q] < c) q++;
        if (q < e && ind[q] == c)
          val[q] = __dsub_rn(ldx(val + q), mul_rn(tl, ldx(val + k)));
        else if (modified)
          s = add_rn(s, mul_rn(tl, ldx(val + k)));
        else if (q == e)
          break;  // ILU(0): no column of row i is left to update
      }
    }
    double piv = ldx(val + d);
    if (modified) {
      piv = __dsub_rn(piv, s);
      val[d] = piv;
    }
    if (piv == 0.0) {
      atomicCAS(status, 0, i + 1);
      return;
    }
    val[d] = __ddiv_rn(1.0, piv);
  }
};

// out[idx[i]] = in[i]
__global__ void perm_scatter_kernel(int n, const int* __restrict__ idx,
                                    const double* __restrict__ in, double* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[idx[i]] = in[i];
}

// out[i] = in[idx[i]]
__global__ void perm_gather_kernel(int n, const int* __restrict__ idx,
                                   const double* __restrict__ in, double* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = in[idx[i]];
}

__global__ void jacobi_kernel(int n, const double* __restrict__ r,
                              const double* __restrict__ d, double* __restrict__ z) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    z[i] = __ddiv_rn(r[i], d[i]);
}
#endif

constexpr int kSorSingleCtaMaxN = 65536;

template <class Op>
static int run_levels(const LevelPlan& P, int n, const Op& op, cudaStream_t s) {
  if (n == 0 || P.nlev == 0) return SB2_OK;
  if (n <= kSorSingleCtaMaxN) {
    level_single_cta<Op><<<1, 1024, 0, s>>>(P.nlev, P.d_lvl, P.d_rows, op);
  } else {
    for (int l = 0; l < P.nlev; l++) {
      const int cnt = P.h_lvl[l + 1] - P.h_lvl[l];
      level_kernel<Op><<<(cnt + 255) / 256, 256, 0, s>>>(P.h_lvl[l], P.h_lvl[l + 1], P.d_rows, op);
    }
  }
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

template <class Op>
static int run_levels_pos(const LevelPlan& P, int n, const Op& op, cudaStream_t s) {
  if (n == 0 || P.nlev == 0) return SB2_OK;
  if (n <= kSorSingleCtaMaxN) {
    level_single_cta_pos<Op><<<1, 1024, 0, s>>>(P.nlev, P.d_lvl, op);
  } else {
    for (int l = 0; l < P.nlev; l++) {
      const int cnt = P.h_lvl[l + 1] - P.h_lvl[l];
      level_kernel_pos<Op><<<(cnt + 255) / 256, 256, 0, s>>>(P.h_lvl[l], P.h_lvl[l + 1], op);
    }
  }
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

template <class Op>
static int run_rows(int n, const Op& op, cudaStream_t s) {
  if (n == 0) return SB2_OK;
  rows_kernel<Op><<<(n + 255) / 256, 256, 0, s>>>(n, op);
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

}  // namespace sb2

namespace sb2 {
// One triangular sweep in gather form: the rows' update lists, stored in
// level order (list i belongs to row lv.d_rows[i]), and the levels.
struct GatherSweep {
  int* d_ptr = nullptr;
  int* d_ind = nullptr;
  double* d_val = nullptr;
  LevelPlan lv;
  void release() {
    cudaFree(d_ptr);
    cudaFree(d_ind);
    cudaFree(d_val);
    d_ptr = d_ind = nullptr;
    d_val = nullptr;
    lv.release();
  }
};
}  // namespace sb2

struct sb2_precond {
  const sb2_csr* A = nullptr;
  int kind = 0;
  double omega = 1.0;
  int nb_iter = 1;
  int symmetric = 1;
  // SOR schedules: general forward/backward sweeps, or for symmetric storage
  // the lower (forward) and upper (backward) triangular solves.
  sb2::LevelPlan fwd, bwd;
  double* d_t = nullptr;  // scratch of the symmetric sweeps and of ILUT
  std::mutex mu;
  bool planned = false;
  // ILUT: order, storage, permutations, 1/U(i,i) or 1/D(i), and the sweeps
  // (unsymmetric: L forward, U backward, U^T forward, L^T backward;
  // symmetric: L forward through the transposed rows, L^T backward)
  int n_ilu = 0;
  int ilu_sym = 0;
  int* d_prow = nullptr;
  int* d_pcol = nullptr;
  double* d_dinv = nullptr;
  sb2::GatherSweep s_lf, s_ub, s_utf, s_ltb;
  // Applies with one launch per level, recorded once per (r, z, direction)
  // as CUDA graphs and replayed (the Krylov drivers reuse their buffers).
  struct Recorded {
    const double* r;
    double* z;
    bool trans;
    cudaGraphExec_t exec;
  };
  std::vector<Recorded> graphs;
  cudaStream_t cap_stream = nullptr;
};

namespace sb2 {

static int plan_sor(sb2_precond* M) {
  std::lock_guard<std::mutex> g(M->mu);
  if (M->planned) return SB2_OK;
  const sb2_csr* A = M->A;
  const int n = A->m;
  const CsrArrays& src = A->sym ? A->upper : A->full;
  std::vector<int> ptr(n + 1), ind(src.nnz);
  SB2_CUDA_TRY(cudaMemcpy(ptr.data(), src.d_ptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
  if (src.nnz) SB2_CUDA_TRY(cudaMemcpy(ind.data(), src.d_ind, sizeof(int) * src.nnz, cudaMemcpyDeviceToHost));
  std::vector<int> level;
  if (!A->sym) {
    sweep_levels(n, ptr.data(), ind.data(), true, level);
    SB2_TRY(upload_plan(level, n, &M->fwd));
    sweep_levels(n, ptr.data(), ind.data(), false, level);
    SB2_TRY(upload_plan(level, n, &M->bwd));
  } else {
    // forward second loop = lower solve (dependencies c < j of the full
    // pattern); backward second loop = upper solve on the stored rows.
    const CsrArrays& f = A->full;
    std::vector<int> fptr(n + 1), find(f.nnz);
    SB2_CUDA_TRY(cudaMemcpy(fptr.data(), f.d_ptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
    if (f.nnz) SB2_CUDA_TRY(cudaMemcpy(find.data(), f.d_ind, sizeof(int) * f.nnz, cudaMemcpyDeviceToHost));
    tri_levels(n, fptr.data(), find.data(), true, level);
    SB2_TRY(upload_plan(level, n, &M->fwd));
    tri_levels(n, ptr.data(), ind.data(), false, level);
    SB2_TRY(upload_plan(level, n, &M->bwd));
    SB2_CUDA_TRY(cudaMalloc(&M->d_t, sizeof(double) * std::max(n, 1)));
  }
  M->planned = true;
  return SB2_OK;
}

// SOR(A, X, B, omega, iter, type_ssor) on device, in place on x, once the
// level plans and the diagonal exist (sor_apply makes them).
static int sor_run(sb2_precond* M, double* x, const double* b, double omega,
                   int iter, int type_ssor, cudaStream_t s) {
  const sb2_csr* A = M->A;
  const int n = A->m;
  if (!A->sym) {
    SB2_TRY(ensure_diag(A));
    RowSparseSor op{A->full.d_ptr, A->full.d_ind, A->full.d_val, A->d_diag, b, x, omega};
    if (type_ssor % 2 == 0)
      for (int i = 0; i < iter; i++) SB2_TRY(run_levels(M->fwd, n, op, s));
    if (type_ssor % 3 == 0)
      for (int i = 0; i < iter; i++) SB2_TRY(run_levels(M->bwd, n, op, s));
    return SB2_OK;
  }
  const CsrArrays& u = A->upper;
  const CsrArrays& f = A->full;
  if (type_ssor % 2 == 0)
    for (int i = 0; i < iter; i++) {
      SB2_TRY(run_rows(n, SymFwd1{u.d_ptr, u.d_ind, u.d_val, b, x, M->d_t, omega}, s));
      SB2_TRY(run_levels(M->fwd, n,
                         SymFwd2{f.d_ptr, f.d_ind, f.d_val, u.d_ptr, u.d_ind, u.d_val, M->d_t, x, omega}, s));
    }
  if (type_ssor % 3 == 0)
    for (int i = 0; i < iter; i++) {
      SB2_TRY(run_rows(n, SymBwd1{f.d_ptr, f.d_ind, f.d_val, u.d_ptr, u.d_ind, u.d_val, b, x, M->d_t, omega}, s));
      SB2_TRY(run_levels(M->bwd, n, SymBwd2{u.d_ptr, u.d_ind, u.d_val, M->d_t, x, omega}, s));
    }
  return SB2_OK;
}

static int sor_apply(sb2_precond* M, double* x, const double* b, double omega,
                     int iter, int type_ssor, cudaStream_t s) {
  SB2_TRY(plan_sor(M));
  if (!M->A->sym) SB2_TRY(ensure_diag(M->A));
  return sor_run(M, x, b, omega, iter, type_ssor, s);
}

// Levels of a gather sweep: row j waits for every row it reads; rows are
// visited in dependency order (increasing j when reads are of smaller
// rows, decreasing otherwise).
static void gather_levels(int n, const std::vector<int>& ptr, const std::vector<int>& ind,
                          bool ascending, std::vector<int>& level) {
  level.assign(n, 0);
  for (int s = 0; s < n; s++) {
    const int j = ascending ? s : n - 1 - s;
    int lev = 0;
    for (int k = ptr[j]; k < ptr[j + 1]; k++) lev = std::max(lev, level[ind[k]] + 1);
    level[j] = lev;
  }
}

static int upload_sweep(int n, const std::vector<int>& ptr, const std::vector<int>& ind,
                        const std::vector<double>& val, bool ascending, GatherSweep* S) {
  std::vector<int> level, order;
  gather_levels(n, ptr, ind, ascending, level);
  SB2_TRY(upload_plan(level, n, &S->lv, &order));
  // the lists in level order
  std::vector<int> pptr(n + 1, 0), pind;
  std::vector<double> pval;
  pind.reserve(ind.size());
  pval.reserve(val.size());
  for (int i = 0; i < n; i++) {
    const int j = order[i];
    pind.insert(pind.end(), ind.begin() + ptr[j], ind.begin() + ptr[j + 1]);
    pval.insert(pval.end(), val.begin() + ptr[j], val.begin() + ptr[j + 1]);
    pptr[i + 1] = (int)pind.size();
  }
  const size_t nz = pind.size();
  SB2_CUDA_TRY(cudaMalloc(&S->d_ptr, sizeof(int) * (n + 1)));
  SB2_CUDA_TRY(cudaMalloc(&S->d_ind, sizeof(int) * std::max<size_t>(nz, 1)));
  SB2_CUDA_TRY(cudaMalloc(&S->d_val, sizeof(double) * std::max<size_t>(nz, 1)));
  SB2_CUDA_TRY(cudaMemcpy(S->d_ptr, pptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
  if (nz) {
    SB2_CUDA_TRY(cudaMemcpy(S->d_ind, pind.data(), sizeof(int) * nz, cudaMemcpyHostToDevice));
    SB2_CUDA_TRY(cudaMemcpy(S->d_val, pval.data(), sizeof(double) * nz, cudaMemcpyHostToDevice));
  }
  return SB2_OK;
}

// Update lists of a column scatter: entry (i -> c, v) for the rows i in the
// order the sequential loop visits them, each row's entries in stored order.
struct ListBuilder {
  std::vector<std::vector<int>> src;
  std::vector<std::vector<double>> v;
  explicit ListBuilder(int n) : src(n), v(n) {}
  void add(int target, int source, double value) {
    src[target].push_back(source);
    v[target].push_back(value);
  }
  void flatten(std::vector<int>& ptr, std::vector<int>& ind, std::vector<double>& val) const {
    const int n = (int)src.size();
    ptr.assign(n + 1, 0);
    for (int j = 0; j < n; j++) ptr[j + 1] = ptr[j] + (int)src[j].size();
    ind.clear();
    val.clear();
    ind.reserve(ptr[n]);
    val.reserve(ptr[n]);
    for (int j = 0; j < n; j++) {
      ind.insert(ind.end(), src[j].begin(), src[j].end());
      val.insert(val.end(), v[j].begin(), v[j].end());
    }
  }
};

static bool is_permutation(int n, const int* p) {
  std::vector<char> seen(n, 0);
  for (int i = 0; i < n; i++) {
    if (p[i] < 0 || p[i] >= n || seen[p[i]]) return false;
    seen[p[i]] = 1;
  }
  return true;
}

// Builds every sweep of the factor (host arrays in Seldon's stored order).
static int plan_ilut(sb2_precond* M, int n, const int* fp, const int* fi, const double* fv,
                     const int* prow, const int* pcol) {
  if (fp[0] != 0) return SB2_ERR_INVALID_CSR;
  for (int i = 0; i < n; i++)
    if (fp[i + 1] < fp[i]) return SB2_ERR_INVALID_CSR;
  if (!is_permutation(n, prow) || (!M->ilu_sym && !is_permutation(n, pcol)))
    return SB2_ERR_INVALID_VALUE;
  std::vector<double> dinv(n);
  std::vector<int> ptr, ind;
  std::vector<double> val;
  if (M->ilu_sym) {
    // row i: 1/D(i) at the first position, then row i of L^T (columns > i)
    ListBuilder fwd(n);
    std::vector<int> bptr(n + 1, 0), bind;
    std::vector<double> bval;
    for (int i = 0; i < n; i++) {
      if (fp[i + 1] <= fp[i]) return SB2_ERR_INVALID_CSR;
      dinv[i] = fv[fp[i]];
      for (int k = fp[i] + 1; k < fp[i + 1]; k++) {
        if (fi[k] <= i || fi[k] >= n) return SB2_ERR_INVALID_CSR;
        fwd.add(fi[k], i, fv[k]);  // L y = b: x(j) -= A(i,k) x(i), i increasing
        bind.push_back(fi[k]);
        bval.push_back(fv[k]);
      }
      bptr[i + 1] = (int)bind.size();
    }
    fwd.flatten(ptr, ind, val);
    SB2_TRY(upload_sweep(n, ptr, ind, val, true, &M->s_lf));
    SB2_TRY(upload_sweep(n, bptr, bind, bval, false, &M->s_ub));
  } else {
    // row i: L part (columns < i), then 1/U(i,i), then the U part
    std::vector<int> lptr(n + 1, 0), lind, uptr(n + 1, 0), uind;
    std::vector<double> lval, uval;
    ListBuilder utf(n), ltb(n);
    std::vector<int> dpos(n);
    for (int i = 0; i < n; i++) {
      int k = fp[i];
      while (k < fp[i + 1] && fi[k] < i) {
        if (fi[k] < 0) return SB2_ERR_INVALID_CSR;
        lind.push_back(fi[k]);
        lval.push_back(fv[k]);
        k++;
      }
      if (k == fp[i + 1]) return SB2_ERR_INVALID_CSR;  // no diagonal position
      dpos[i] = k;
      dinv[i] = fv[k];
      for (int q = k + 1; q < fp[i + 1]; q++) {
        if (fi[q] <= i || fi[q] >= n) return SB2_ERR_INVALID_CSR;
        uind.push_back(fi[q]);
        uval.push_back(fv[q]);
        utf.add(fi[q], i, fv[q]);  // U^T: x(c) -= U(i,c) x(i), i increasing
      }
      lptr[i + 1] = (int)lind.size();
      uptr[i + 1] = (int)uind.size();
    }
    for (int i = n - 1; i >= 0; i--)  // L^T: x(k) -= L(i,k) x(i), i decreasing
      for (int k = fp[i]; k < dpos[i]; k++) ltb.add(fi[k], i, fv[k]);
    SB2_TRY(upload_sweep(n, lptr, lind, lval, true, &M->s_lf));
    SB2_TRY(upload_sweep(n, uptr, uind, uval, false, &M->s_ub));
    utf.flatten(ptr, ind, val);
    SB2_TRY(upload_sweep(n, ptr, ind, val, true, &M->s_utf));
    ltb.flatten(ptr, ind, val);
    SB2_TRY(upload_sweep(n, ptr, ind, val, false, &M->s_ltb));
  }
  SB2_CUDA_TRY(cudaMalloc(&M->d_dinv, sizeof(double) * std::max(n, 1)));
  SB2_CUDA_TRY(cudaMalloc(&M->d_prow, sizeof(int) * std::max(n, 1)));
  SB2_CUDA_TRY(cudaMalloc(&M->d_pcol, sizeof(int) * std::max(n, 1)));
  SB2_CUDA_TRY(cudaMalloc(&M->d_t, sizeof(double) * std::max(n, 1)));
  SB2_CUDA_TRY(cudaMemcpy(M->d_dinv, dinv.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  SB2_CUDA_TRY(cudaMemcpy(M->d_prow, prow, sizeof(int) * n, cudaMemcpyHostToDevice));
  SB2_CUDA_TRY(cudaMemcpy(M->d_pcol, M->ilu_sym ? prow : pcol, sizeof(int) * n,
                          cudaMemcpyHostToDevice));
  return SB2_OK;
}

// GetIlu0 on the device: rows in levels of their L dependencies, each row
// factored by one thread in the reference's operation order.  The factor
// (A's pattern, Seldon's ArrayRowSparse layout) is returned on the host.
static int ilu0_factor(const sb2_csr* A, int modified, std::vector<int>& ptr,
                       std::vector<int>& ind, std::vector<double>& val, cudaStream_t s) {
  const int n = A->m;
  const CsrArrays& f = A->full;
  ptr.resize(n + 1);
  ind.resize(f.nnz);
  val.resize(f.nnz);
  SB2_CUDA_TRY(cudaMemcpy(ptr.data(), f.d_ptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
  if (f.nnz) {
    SB2_CUDA_TRY(cudaMemcpy(ind.data(), f.d_ind, sizeof(int) * f.nnz, cudaMemcpyDeviceToHost));
  }
  // GetIlu0 reads the row prefix before the diagonal as L and needs every
  // row sorted, with its diagonal, and no repeated column
  std::vector<int> dpos(n, -1), lptr(n + 1, 0), lind;
  for (int i = 0; i < n; i++) {
    for (int k = ptr[i]; k < ptr[i + 1]; k++) {
      if (ind[k] < 0 || ind[k] >= n) return SB2_ERR_INVALID_CSR;
      if (k > ptr[i] && ind[k] <= ind[k - 1]) return SB2_ERR_INVALID_CSR;
      if (ind[k] == i) dpos[i] = k;
      if (ind[k] < i) lind.push_back(ind[k]);
    }
    if (dpos[i] < 0) return SB2_ERR_INVALID_CSR;
    lptr[i + 1] = (int)lind.size();
  }
  std::vector<int> level;
  gather_levels(n, lptr, lind, true, level);
  LevelPlan plan;
  int st = upload_plan(level, n, &plan);
  double* d_val = nullptr;
  int *d_dpos = nullptr, *d_status = nullptr;
  cudaError_t e = cudaMalloc(&d_val, sizeof(double) * std::max<long long>(f.nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_dpos, sizeof(int) * std::max(n, 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_status, sizeof(int));
  if (e == cudaSuccess && f.nnz)
    e = cudaMemcpyAsync(d_val, f.d_val, sizeof(double) * f.nnz, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_dpos, dpos.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_status, 0, sizeof(int), s);
  if (st == SB2_OK) st = map_cuda_error(e);
  int status = 0;
  if (st == SB2_OK)
    st = run_levels(plan, n, Ilu0Row{f.d_ptr, f.d_ind, d_val, d_dpos, d_status, modified}, s);
  if (st == SB2_OK) {
    e = cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && f.nnz)
      e = cudaMemcpyAsync(val.data(), d_val, sizeof(double) * f.nnz, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    st = map_cuda_error(e);
  }
  if (st == SB2_OK && status != 0) st = SB2_ERR_INVALID_VALUE;  // zero pivot
  cudaFree(d_val);
  cudaFree(d_dpos);
  cudaFree(d_status);
  plan.release();
  return st;
}

static GatherSubPacked sweep_op(const GatherSweep& S, const double* pre, const double* post,
                                double* x) {
  return GatherSubPacked{S.lv.d_rows, S.d_ptr, S.d_ind, S.d_val, pre, post, x};
}

// IlutPreconditioning::Solve / TransSolve (IlutPreconditioning.cxx:329-374):
// the launches.
static int ilut_launch(const sb2_precond* M, bool trans, const double* r, double* z,
                       cudaStream_t s) {
  const int n = M->n_ilu;
  double* t = M->d_t;
  const int g = std::min((n + 255) / 256, num_sms(current_device()) * 8);
  if (M->ilu_sym) {
    perm_scatter_kernel<<<g, 256, 0, s>>>(n, M->d_prow, r, t);
    SB2_TRY(run_levels_pos(M->s_lf.lv, n, sweep_op(M->s_lf, nullptr, nullptr, t), s));
    SB2_TRY(run_levels_pos(M->s_ub.lv, n, sweep_op(M->s_ub, M->d_dinv, nullptr, t), s));
    perm_gather_kernel<<<g, 256, 0, s>>>(n, M->d_prow, t, z);
  } else if (!trans) {
    perm_scatter_kernel<<<g, 256, 0, s>>>(n, M->d_prow, r, t);
    SB2_TRY(run_levels_pos(M->s_lf.lv, n, sweep_op(M->s_lf, nullptr, nullptr, t), s));
    SB2_TRY(run_levels_pos(M->s_ub.lv, n, sweep_op(M->s_ub, nullptr, M->d_dinv, t), s));
    perm_scatter_kernel<<<g, 256, 0, s>>>(n, M->d_pcol, t, z);
  } else {
    perm_gather_kernel<<<g, 256, 0, s>>>(n, M->d_pcol, r, t);
    SB2_TRY(run_levels_pos(M->s_utf.lv, n, sweep_op(M->s_utf, nullptr, M->d_dinv, t), s));
    SB2_TRY(run_levels_pos(M->s_ltb.lv, n, sweep_op(M->s_ltb, nullptr, nullptr, t), s));
    perm_gather_kernel<<<g, 256, 0, s>>>(n, M->d_prow, t, z);
  }
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

constexpr int kIluGraphs = 8;  // recorded applies kept per preconditioner

// Applies of large systems launch once per level: they are recorded once per
// (r, z, direction) as a CUDA graph and replayed, so the launches cost the
// device's dependency resolution only, not a host call each.  `launch`
// enqueues the apply on the stream it is given.
template <class Launch>
static int replay_recorded(sb2_precond* M, bool trans, const double* r, double* z,
                           cudaStream_t s, const Launch& launch) {
  std::lock_guard<std::mutex> g(M->mu);
  for (const auto& e : M->graphs)
    if (e.r == r && e.z == z && e.trans == trans) {
      SB2_CUDA_TRY(cudaGraphLaunch(e.exec, s));
      return SB2_OK;
    }
  if (!M->cap_stream)
    SB2_CUDA_TRY(cudaStreamCreateWithFlags(&M->cap_stream, cudaStreamNonBlocking));
  SB2_CUDA_TRY(cudaStreamBeginCapture(M->cap_stream, cudaStreamCaptureModeThreadLocal));
  int st = launch(M->cap_stream);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(M->cap_stream, &graph);
  if (st != SB2_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  SB2_CUDA_TRY(e);
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  SB2_CUDA_TRY(e);
  if ((int)M->graphs.size() >= kIluGraphs) {
    // the oldest recording goes once the stream has no launch of it pending
    cudaStreamSynchronize(s);
    cudaGraphExecDestroy(M->graphs.front().exec);
    M->graphs.erase(M->graphs.begin());
  }
  M->graphs.push_back({r, z, trans, exec});
  SB2_CUDA_TRY(cudaGraphLaunch(exec, s));
  return SB2_OK;
}

// Small systems run every level in one CTA (one launch); larger ones replay
// a recorded graph of the per-level launches.
static int ilut_apply(sb2_precond* M, bool trans, const double* r, double* z, cudaStream_t s) {
  if (M->n_ilu <= kSorSingleCtaMaxN) return ilut_launch(M, trans, r, z, s);
  return replay_recorded(M, trans, r, z, s, [&](cudaStream_t cs) {
    return ilut_launch(M, trans, r, z, cs);
  });
}

int precond_kind(const sb2_precond* M) { return M->kind; }
int precond_n(const sb2_precond* M) { return M->kind == SB2_PRECOND_ILUT ? M->n_ilu : M->A->m; }
const sb2_csr* precond_matrix(const sb2_precond* M) { return M->A; }

int precond_apply(const sb2_precond* cM, bool trans, const double* r, double* z,
                  cudaStream_t s) {
  sb2_precond* M = const_cast<sb2_precond*>(cM);
  if (M->kind == SB2_PRECOND_ILUT) return M->n_ilu ? ilut_apply(M, trans, r, z, s) : SB2_OK;
  const int n = M->A->m;
  if (n == 0) return SB2_OK;
  if (M->kind == SB2_PRECOND_IDENTITY) {
    SB2_CUDA_TRY(cudaMemcpyAsync(z, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    return SB2_OK;
  }
  if (M->kind == SB2_PRECOND_JACOBI) {
    SB2_TRY(ensure_diag(M->A));
    int g = std::min((n + 255) / 256, num_sms(current_device()) * 8);
    jacobi_kernel<<<g, 256, 0, s>>>(n, r, M->A->d_diag, z);
    SB2_CUDA_TRY(cudaGetLastError());
    return SB2_OK;
  }
  // SorPreconditioner::Solve / TransSolve (Precond_Ssor.cxx:62-90)
  const int type = M->symmetric ? 0 : (trans ? 3 : 2);
  SB2_TRY(plan_sor(M));
  if (!M->A->sym) SB2_TRY(ensure_diag(M->A));
  auto launch = [&](cudaStream_t cs) -> int {
    SB2_CUDA_TRY(cudaMemsetAsync(z, 0, sizeof(double) * n, cs));
    return sor_run(M, z, r, M->omega, M->nb_iter, type, cs);
  };
  if (n <= kSorSingleCtaMaxN) return launch(s);
  // the symmetric sweeps' trans flag does not change the launches
  return replay_recorded(M, M->symmetric ? false : trans, r, z, s, launch);
}

}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_precond_create(const sb2_csr* A, int kind, double omega, int nb_iter,
                       int symmetric, sb2_precond** out) try {
  if (!out || !A) return SB2_ERR_INVALID_VALUE;
  *out = nullptr;
  if (kind < SB2_PRECOND_IDENTITY || kind > SB2_PRECOND_SOR) return SB2_ERR_INVALID_VALUE;
  if (A->m != A->n) return SB2_ERR_INVALID_VALUE;
  std::unique_ptr<sb2_precond, int (*)(sb2_precond*)> M(new sb2_precond(),
                                                         sb2_precond_destroy);
  M->A = A;
  M->kind = kind;
  M->omega = omega;
  M->nb_iter = nb_iter;
  M->symmetric = symmetric ? 1 : 0;
  if (kind == SB2_PRECOND_JACOBI) SB2_TRY(ensure_diag(A));
  *out = M.release();
  return SB2_OK;
} SB2_CATCH

int sb2_precond_create_ilut(const sb2_csr* A, int n, const int* fptr, const int* find,
                            const double* fval, const int* perm_row, const int* perm_col,
                            int symmetric, sb2_precond** out) try {
  SB2_TRACE("sb2_precond_create_ilut");
  if (!out || n < 0 || (n > 0 && (!fptr || !perm_row || (!symmetric && !perm_col))))
    return SB2_ERR_INVALID_VALUE;
  *out = nullptr;
  if (A && (A->m != n || A->n != n)) return SB2_ERR_INVALID_VALUE;
  if (n > 0 && fptr[n] > 0 && (!find || !fval)) return SB2_ERR_INVALID_VALUE;
  // every index the sweeps read is checked while they are built
  std::unique_ptr<sb2_precond, int (*)(sb2_precond*)> M(new sb2_precond(),
                                                         sb2_precond_destroy);
  M->A = A;
  M->kind = SB2_PRECOND_ILUT;
  M->n_ilu = n;
  M->ilu_sym = symmetric ? 1 : 0;
  if (n > 0) SB2_TRY(plan_ilut(M.get(), n, fptr, find, fval, perm_row, perm_col));
  *out = M.release();
  return SB2_OK;
} SB2_CATCH

int sb2_precond_create_ilu0(const sb2_csr* A, int modified, void* stream, sb2_precond** out) try {
  SB2_TRACE("sb2_precond_create_ilu0");
  if (!out || !A || A->m != A->n || A->sym) return SB2_ERR_INVALID_VALUE;
  *out = nullptr;
  const int n = A->m;
  std::vector<int> ptr, ind;
  std::vector<double> val;
  if (n > 0) SB2_TRY(ilu0_factor(A, modified ? 1 : 0, ptr, ind, val, (cudaStream_t)stream));
  std::vector<int> ident(std::max(n, 1));
  for (int i = 0; i < n; i++) ident[i] = i;
  if (ptr.empty()) ptr.assign(1, 0);
  // the factor no longer needs A: like the reference's preconditioner, it
  // applies to whichever matrix of order n the solver is given
  return sb2_precond_create_ilut(nullptr, n, ptr.data(), ind.empty() ? nullptr : ind.data(),
                                 val.empty() ? nullptr : val.data(), ident.data(), ident.data(), 0,
                                 out);
} SB2_CATCH

int sb2_precond_destroy(sb2_precond* M) try {
  if (!M) return SB2_OK;
  if (!M->graphs.empty()) cudaDeviceSynchronize();  // no replay may be in flight
  for (auto& e : M->graphs) cudaGraphExecDestroy(e.exec);
  if (M->cap_stream) cudaStreamDestroy(M->cap_stream);
  M->fwd.release();
  M->bwd.release();
  cudaFree(M->d_t);
  M->s_lf.release();
  M->s_ub.release();
  M->s_utf.release();
  M->s_ltb.release();
  cudaFree(M->d_prow);
  cudaFree(M->d_pcol);
  cudaFree(M->d_dinv);
  delete M;
  return SB2_OK;
} SB2_CATCH

int sb2_precond_solve(const sb2_precond* M, const double* r, double* z, void* stream) try {
  SB2_TRACE("sb2_precond_solve");
  if (!M || (precond_n(M) > 0 && (!r || !z)) || (r == z && precond_n(M) > 0))
    return SB2_ERR_INVALID_VALUE;
  return precond_apply(M, false, r, z, (cudaStream_t)stream);
} SB2_CATCH

int sb2_precond_trans_solve(const sb2_precond* M, const double* r, double* z, void* stream) try {
  SB2_TRACE("sb2_precond_trans_solve");
  if (!M || (precond_n(M) > 0 && (!r || !z)) || (r == z && precond_n(M) > 0))
    return SB2_ERR_INVALID_VALUE;
  return precond_apply(M, true, r, z, (cudaStream_t)stream);
} SB2_CATCH

int sb2_sor(const sb2_csr* A, double* x, const double* b, double omega, int iter,
            int type_ssor, void* stream) try {
  SB2_TRACE("sb2_sor");
  if (!A || A->m != A->n || (A->m > 0 && (!x || !b)) || x == b) return SB2_ERR_INVALID_VALUE;
  sb2_precond tmp;
  tmp.A = A;
  tmp.kind = SB2_PRECOND_SOR;
  int st = sor_apply(&tmp, x, b, omega, iter, type_ssor, (cudaStream_t)stream);
  // the plan is released after the stream has consumed it
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  tmp.fwd.release();
  tmp.bwd.release();
  cudaFree(tmp.d_t);
  if (st == SB2_OK && e != cudaSuccess) st = map_cuda_error(e);
  return st;
} SB2_CATCH

}  // extern "C"
