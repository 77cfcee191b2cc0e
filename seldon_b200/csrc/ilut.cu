// ILUT factorization on the host, as IlutPreconditioning::FactorizeMatrix
// computes it for a RowSparse matrix with the unsymmetric algorithm
// (computation/solver/preconditioner/IlutPreconditioning.cxx:266-323 and
// GetIlut, :503-878): the factor and the two permutations that the device
// apply (sb2_precond_create_ilut) takes.
//
// The factorization is Saad's ILUT with column pivoting (ILUTP), with the
// reference's variants: ILUT (the lfil largest entries of each part kept,
// chosen by quick-split), ILU_D (entries dropped against the row norm,
// their sum added back to the pivot with weight alpha) and ILUT_K (lfil =
// row length + additional_fill).  Every step is taken in the reference's
// order, so the factor is the reference's bit for bit: the row scan order,
// the choice of the smallest remaining column at each elimination, the
// fill-in append order, the quick-split, the pivot search within blocks of
// mbloc columns, and the replacement of a zero pivot.
#include <algorithm>
#include <climits>
#include <cmath>
#include <memory>
#include <utility>
#include <vector>

#include "sb2_internal.cuh"

struct sb2_ilut {
  int n = 0;
  std::vector<int> fptr, find, perm_row, perm_col;
  std::vector<double> fval;
};

namespace sb2 {
namespace {

// Quick-split of a[first..n-1] (with ind): afterwards |a(i)| >= |a(ncut-1)|
// for i < ncut-1 and |a(i)| <= |a(ncut-1)| beyond (qsplit_ilut,
// IlutPreconditioning.cxx:436-497).
void quick_split(std::vector<double>& a, std::vector<int>& ind, int first, int n, int ncut) {
  int last = n - 1;
  const int cut = ncut - 1;
  if (cut < first || cut > last) return;
  for (;;) {
    int mid = first;
    const double key = std::fabs(a[mid]);
    for (int j = first + 1; j <= last; j++)
      if (std::fabs(a[j]) > key) {
        ++mid;
        std::swap(a[mid], a[j]);
        std::swap(ind[mid], ind[j]);
      }
    std::swap(a[mid], a[first]);
    std::swap(ind[mid], ind[first]);
    if (mid == cut) return;
    if (mid > cut) last = mid - 1;
    else first = mid + 1;
  }
}

// Rows in one flat CSR: the input rows, and the factor, whose rows are
// appended in order (the elimination of row i reads only rows before i).
struct Csr {
  std::vector<int> ptr{0}, idx;
  std::vector<double> val;
  int begin(int i) const { return ptr[i]; }
  int end(int i) const { return ptr[i + 1]; }
  // closes the row just appended; the factor's indices are int32
  bool close_row() {
    if (idx.size() > (size_t)INT_MAX) return false;
    ptr.push_back((int)idx.size());
    return true;
  }
};

int factor(int n, const Csr& A0, const sb2_ilut_params& p, Csr& F, std::vector<int>& iperm,
           std::vector<int>& rperm) {
  const bool variable_fill = (p.type == SB2_ILUT_K);
  const bool standard_dropping = (p.type == SB2_ILU_D);
  int lfil = p.fill_level;
  if (lfil < 0) return SB2_ERR_INVALID_VALUE;
  F = Csr();
  F.ptr.reserve((size_t)n + 1);
  std::vector<double> w(n, 0.0);
  std::vector<int> wi(n, -1), where(n, -1), diag_at(n, -1);
  iperm.resize(n);
  rperm.resize(n);
  for (int i = 0; i < n; i++) iperm[i] = rperm[i] = i;
  for (int i = 0; i < n; i++) {
    const int a0 = A0.begin(i);
    const int size_row = A0.end(i) - a0;
    const int* a_idx = A0.idx.data() + a0;
    const double* a_val = A0.val.data() + a0;
    double tnorm = 0.0;
    for (int k = 0; k < size_row; k++)
      if (a_val[k] != 0.0) tnorm += std::fabs(a_val[k]);
    if (tnorm == 0.0) return SB2_ERR_INVALID_VALUE;  // structurally singular row
    tnorm /= (double)size_row;
    if (variable_fill) lfil = size_row + p.additional_fill;
    // A fill below 1 keeps no U entry, not even the pivot: the reference then
    // stores 1/U(i,i) one position past the row it resized, so it is refused.
    if (!standard_dropping && lfil < 1) return SB2_ERR_INVALID_VALUE;
    double dropsum = 0.0;
    // the row's L part at w[0..nl), its diagonal at w[i], its U part after
    int nl = 0, nu = 1;
    wi[i] = i;
    w[i] = 0.0;
    where[i] = i;
    for (int k = 0; k < size_row; k++) {
      const int c = rperm[a_idx[k]];
      const double t = a_val[k];
      if (c < i) {
        wi[nl] = c;
        w[nl] = t;
        where[c] = nl;
        ++nl;
      } else if (c == i) {
        w[i] = t;
      } else {
        const int at = i + nu;
        wi[at] = c;
        w[at] = t;
        where[c] = at;
        nu++;
      }
    }
    // eliminate with the previous rows, smallest column first
    int kept = 0;
    for (int jc = 0; jc < nl; jc++) {
      int jrow = wi[jc], kmin = jc;
      for (int j = jc + 1; j < nl; j++)
        if (wi[j] < jrow) {
          jrow = wi[j];
          kmin = j;
        }
      if (kmin != jc) {
        const int other = wi[jc];
        wi[jc] = wi[kmin];
        wi[kmin] = other;
        where[jrow] = jc;
        where[other] = kmin;
        std::swap(w[jc], w[kmin]);
      }
      where[jrow] = -1;
      bool dropped = false;
      if (standard_dropping && std::fabs(w[jc]) <= p.droptol * tnorm) {
        dropsum += w[jc];
        dropped = true;
      }
      double fact = 0.0;
      if (!dropped) {
        fact = w[jc] * F.val[F.begin(jrow) + diag_at[jrow]];
        if (!standard_dropping && std::fabs(fact) <= p.droptol) dropped = true;
      }
      if (!dropped) {
        for (int k = F.begin(jrow) + diag_at[jrow] + 1; k < F.end(jrow); k++) {
          const double s = fact * F.val[k];
          const int c = rperm[F.idx[k]];
          const int at = where[c];
          if (c >= i) {
            if (at == -1) {
              const int slot = i + nu;
              wi[slot] = c;
              where[c] = slot;
              w[slot] = -s;
              ++nu;
            } else {
              w[at] -= s;
            }
          } else {
            if (at == -1) {
              wi[nl] = c;
              where[c] = nl;
              w[nl] = -s;
              ++nl;
            } else {
              w[at] -= s;
            }
          }
        }
        // the multiplier is kept in the L part, left to right
        w[kept] = fact;
        wi[kept] = jrow;
        ++kept;
      }
    }
    for (int k = 0; k < nu; k++) where[wi[i + k]] = -1;
    // L part: keep the lfil largest (quick-split) unless dropping by norm
    int len = kept;
    if (!standard_dropping) {
      len = std::min(kept, lfil);
      quick_split(w, wi, 0, kept, len);
    }
    const size_t row0 = F.idx.size();
    for (int k = 0; k < len; k++) {
      F.val.push_back(w[k]);
      F.idx.push_back(iperm[wi[k]]);
    }
    const int index_diag = len;
    diag_at[i] = index_diag;
    // U part: drop against the row norm, then keep the lfil largest
    int lu = 0;
    for (int k = 1; k <= nu - 1; k++) {
      if (std::fabs(w[i + k]) > p.droptol * tnorm) {
        ++lu;
        w[i + lu] = w[i + k];
        wi[i + lu] = wi[i + k];
      } else {
        dropsum += w[i + k];
      }
    }
    if (!standard_dropping) {
      const int nup = lu + 1;
      lu = std::min(nup, lfil);
      quick_split(w, wi, i + 1, i + nup, i + lu + 1);
    } else {
      lu++;
    }
    // pivot: the largest entry within this block of mbloc columns that beats
    // the diagonal by the threshold
    int imax = i;
    double xmax = std::fabs(w[imax]);
    const double xmax0 = xmax;
    const int icut = i + p.mbloc - 1 - i % p.mbloc;
    for (int k = i + 1; k <= i + lu - 1; k++) {
      tnorm = std::fabs(w[k]);  // the reference reuses the row norm's variable
      if (tnorm > xmax && tnorm * p.permtol > xmax0 && wi[k] <= icut) {
        imax = k;
        xmax = tnorm;
      }
    }
    std::swap(w[i], w[imax]);
    const int jcol = wi[imax];
    const int old = iperm[i];
    iperm[i] = iperm[jcol];
    iperm[jcol] = old;
    rperm[iperm[i]] = i;
    rperm[iperm[jcol]] = jcol;
    for (int k = i; k <= i + lu - 1; k++) {
      F.idx.push_back(iperm[wi[k]]);
      F.val.push_back(w[k]);
    }
    if (standard_dropping) w[i] += p.alpha * dropsum;
    if (w[i] == 0.0) w[i] = (p.droptol + 1e-4) * tnorm;
    F.val[row0 + index_diag] = 1.0 / w[i];
    if (!F.close_row()) return SB2_ERR_NOT_SUPPORTED;
  }
  for (int& c : F.idx) c = rperm[c];
  return SB2_OK;
}

// The symmetric algorithm (SymmetricIlutPreconditioning.cxx:27-346): B holds
// the full rows of the symmetric matrix, sorted by column; row i of the
// factor keeps 1/D(i) first and then its U part (no pivoting, no L part
// kept); at the end every U entry is scaled by its row's 1/D.
int factor_sym(int n, const Csr& B, const sb2_ilut_params& p, Csr& F) {
  const bool variable_fill = (p.type == SB2_ILUT_K);
  const bool standard_dropping = (p.type == SB2_ILU_D);
  int lfil = p.fill_level;
  if (lfil < 0) return SB2_ERR_INVALID_VALUE;
  F = Csr();
  F.ptr.reserve((size_t)n + 1);
  std::vector<double> w(n, 0.0);
  std::vector<int> wi(n, -1), where(n, -1);
  for (int i = 0; i < n; i++) {
    const int b0 = B.begin(i);
    const int size_row = B.end(i) - b0;
    const int* a_idx = B.idx.data() + b0;
    const double* a_val = B.val.data() + b0;
    double tnorm = 0.0;
    for (int k = 0; k < size_row; k++) tnorm += std::fabs(a_val[k]);
    if (tnorm == 0.0) return SB2_ERR_INVALID_VALUE;  // structurally singular row
    tnorm /= (double)size_row;
    if (variable_fill) lfil = size_row + p.additional_fill;
    // A fill below 1 leaves the row empty: the reference then stores 1/D(i)
    // in a row it reallocated to length 0, so it is refused.
    if (!standard_dropping && lfil < 1) return SB2_ERR_INVALID_VALUE;
    double dropsum = 0.0;
    int nl = 0, nu = 1;
    wi[i] = i;
    w[i] = 0.0;
    where[i] = i;
    for (int k = 0; k < size_row; k++) {
      const int c = a_idx[k];
      const double t = a_val[k];
      if (c < i) {
        wi[nl] = c;
        w[nl] = t;
        where[c] = nl;
        ++nl;
      } else if (c == i) {
        w[i] = t;
      } else {
        const int at = i + nu;
        wi[at] = c;
        w[at] = t;
        where[c] = at;
        nu++;
      }
    }
    int kept = 0;
    for (int jc = 0; jc < nl; jc++) {
      int jrow = wi[jc], kmin = jc;
      for (int j = jc + 1; j < nl; j++)
        if (wi[j] < jrow) {
          jrow = wi[j];
          kmin = j;
        }
      if (kmin != jc) {
        const int other = wi[jc];
        wi[jc] = wi[kmin];
        wi[kmin] = other;
        where[jrow] = jc;
        where[other] = kmin;
        std::swap(w[jc], w[kmin]);
      }
      where[jrow] = -1;
      bool dropped = false;
      if (standard_dropping && std::fabs(w[jc]) <= p.droptol * tnorm) {
        dropsum += w[jc];
        dropped = true;
      }
      double fact = 0.0;
      if (!dropped) {
        fact = w[jc] * F.val[F.begin(jrow)];
        if (!standard_dropping && std::fabs(fact) <= p.droptol) dropped = true;
      }
      if (!dropped) {
        for (int k = F.begin(jrow) + 1; k < F.end(jrow); k++) {
          const double s = fact * F.val[k];
          const int c = F.idx[k];
          const int at = where[c];
          if (c >= i) {
            if (at == -1) {
              const int slot = i + nu;
              wi[slot] = c;
              where[c] = slot;
              w[slot] = -s;
              ++nu;
            } else {
              w[at] -= s;
            }
          } else {
            if (at == -1) {
              wi[nl] = c;
              where[c] = nl;
              w[nl] = -s;
              ++nl;
            } else {
              w[at] -= s;
            }
          }
        }
        w[kept] = fact;
        wi[kept] = jrow;
        ++kept;
      }
    }
    for (int k = 0; k < nu; k++) where[wi[i + k]] = -1;
    int lu = 0;
    for (int k = 1; k <= nu - 1; k++) {
      if (std::fabs(w[i + k]) > p.droptol * tnorm) {
        ++lu;
        w[i + lu] = w[i + k];
        wi[i + lu] = wi[i + k];
      } else {
        dropsum += w[i + k];
      }
    }
    if (!standard_dropping) {
      const int nup = lu + 1;
      lu = std::min(nup, lfil);
      quick_split(w, wi, i + 1, i + nup, i + lu + 1);
    } else {
      lu++;
    }
    const size_t row0 = F.idx.size();
    F.idx.push_back(i);  // 1/D(i); the reference leaves this index unset
    F.val.push_back(0.0);
    for (int k = i + 1; k <= i + lu - 1; k++) {
      F.idx.push_back(wi[k]);
      F.val.push_back(w[k]);
    }
    if (standard_dropping) w[i] += p.alpha * dropsum;
    if (w[i] == 0.0) w[i] = (p.droptol + 1e-4) * tnorm;
    F.val[row0] = 1.0 / w[i];
    if (!F.close_row()) return SB2_ERR_NOT_SUPPORTED;
  }
  for (int i = 0; i < n; i++)
    for (int k = F.begin(i) + 1; k < F.end(i); k++) F.val[k] *= F.val[F.begin(i)];
  return SB2_OK;
}

int check_params(const sb2_ilut_params* params) {
  if (!params) return SB2_ERR_INVALID_VALUE;
  if (params->type != SB2_ILUT && params->type != SB2_ILU_D && params->type != SB2_ILUT_K)
    return SB2_ERR_NOT_SUPPORTED;
  if (params->mbloc < 1) return SB2_ERR_INVALID_VALUE;
  return SB2_OK;
}

int check_csr_perm(int n, const int* ptr, const int* ind, const double* val, const int* perm,
                   std::vector<int>& inv) {
  if (n < 0 || (n > 0 && (!ptr || !perm))) return SB2_ERR_INVALID_VALUE;
  if (ptr && ptr[0] != 0) return SB2_ERR_INVALID_CSR;
  for (int i = 0; i < n; i++)
    if (ptr[i + 1] < ptr[i]) return SB2_ERR_INVALID_CSR;
  if (n > 0 && ptr[n] > 0 && (!ind || !val)) return SB2_ERR_INVALID_VALUE;
  for (int i = 0; n > 0 && i < ptr[n]; i++)
    if (ind[i] < 0 || ind[i] >= n) return SB2_ERR_INVALID_CSR;
  // perm must be a permutation; inv(perm(i)) = i
  inv.assign(n, -1);
  for (int i = 0; i < n; i++) {
    if (perm[i] < 0 || perm[i] >= n || inv[perm[i]] != -1) return SB2_ERR_INVALID_VALUE;
    inv[perm[i]] = i;
  }
  return SB2_OK;
}

// The result handle, taking the factor's arrays.
std::unique_ptr<sb2_ilut> to_handle(int n, Csr& F) {
  std::unique_ptr<sb2_ilut> f(new sb2_ilut());
  f->n = n;
  f->fptr = std::move(F.ptr);
  f->find = std::move(F.idx);
  f->fval = std::move(F.val);
  return f;
}

// Input rows from (row, column, value) entries: a counting pass sizes the
// rows, a second pass places the entries, then each row is sorted by column
// and a repeated column is refused.
struct RowBuilder {
  int n;
  std::vector<long long> count;
  std::vector<int> fill;
  Csr out;
  explicit RowBuilder(int n_) : n(n_), count((size_t)n_ + 1, 0) {}
  void tally(int r) { count[r + 1]++; }
  int start() {
    for (int i = 0; i < n; i++) count[i + 1] += count[i];
    if (count[n] > INT_MAX) return SB2_ERR_NOT_SUPPORTED;  // int32 row offsets
    out.ptr.assign(count.begin(), count.end());
    fill.assign(out.ptr.begin(), out.ptr.end() - 1);
    out.idx.resize(count[n]);
    out.val.resize(count[n]);
    return SB2_OK;
  }
  void put(int r, int c, double v) {
    const int at = fill[r]++;
    out.idx[at] = c;
    out.val[at] = v;
  }
  int finish() {
    std::vector<std::pair<int, double>> e;
    for (int i = 0; i < n; i++) {
      const int b = out.begin(i), len = out.end(i) - b;
      e.resize(len);
      for (int k = 0; k < len; k++) e[k] = {out.idx[b + k], out.val[b + k]};
      std::sort(e.begin(), e.end(),
                [](const std::pair<int, double>& x, const std::pair<int, double>& y) {
                  return x.first < y.first;
                });
      for (int k = 0; k < len; k++) {
        if (k && e[k].first == e[k - 1].first) return SB2_ERR_NOT_SUPPORTED;
        out.idx[b + k] = e[k].first;
        out.val[b + k] = e[k].second;
      }
    }
    return SB2_OK;
  }
};

}  // namespace
}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_ilut_factor(int n, const int* ptr, const int* ind, const double* val, const int* perm,
                    const sb2_ilut_params* params, sb2_ilut** out) try {
  SB2_TRACE("sb2_ilut_factor");
  if (!out) return SB2_ERR_INVALID_VALUE;
  *out = nullptr;
  SB2_TRY(check_params(params));
  std::vector<int> inv;
  SB2_TRY(check_csr_perm(n, ptr, ind, val, perm, inv));
  // rows and columns permuted, each row sorted by its new columns
  // (ApplyInversePermutation, Permutation_ScalingMatrix.cxx:215-256, on the
  // ArrayRowSparse copy)
  RowBuilder rows(n);
  for (int i = 0; i < n; i++) rows.count[perm[i] + 1] += ptr[i + 1] - ptr[i];
  SB2_TRY(rows.start());
  for (int i = 0; i < n; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++) rows.put(perm[i], perm[ind[k]], val[k]);
  SB2_TRY(rows.finish());
  Csr F;
  std::vector<int> iperm, rperm;
  SB2_TRY(factor(n, rows.out, *params, F, iperm, rperm));
  std::unique_ptr<sb2_ilut> f = to_handle(n, F);
  // permutation_col(i) = inv(iperm(i)), permutation_row = perm
  // (IlutPreconditioning.cxx:315-322)
  f->perm_row.assign(perm, perm + n);
  f->perm_col.resize(n);
  for (int i = 0; i < n; i++) f->perm_col[i] = inv[iperm[i]];
  *out = f.release();
  return SB2_OK;
} SB2_CATCH

int sb2_ilut_factor_sym(int n, const int* ptr, const int* ind, const double* val,
                        const int* perm, const sb2_ilut_params* params, sb2_ilut** out) try {
  SB2_TRACE("sb2_ilut_factor_sym");
  if (!out) return SB2_ERR_INVALID_VALUE;
  *out = nullptr;
  SB2_TRY(check_params(params));
  std::vector<int> inv;
  SB2_TRY(check_csr_perm(n, ptr, ind, val, perm, inv));
  // the upper triangle permuted, each entry kept as (min, max)
  // (Permutation_ScalingMatrix.cxx:465-525), then both triangles of every
  // row sorted by column (Copy to ArrayRowSparse, Matrix_Conversions.cxx:
  // 4155-4200)
  RowBuilder rows(n);
  for (int i = 0; i < n; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++) {
      if (ind[k] < i) return SB2_ERR_INVALID_CSR;  // upper triangle only
      const int r = perm[i], c = perm[ind[k]];
      rows.tally(r);
      if (c != r) rows.tally(c);
    }
  SB2_TRY(rows.start());
  for (int i = 0; i < n; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++) {
      int r = perm[i], c = perm[ind[k]];
      if (c < r) std::swap(r, c);
      rows.put(r, c, val[k]);
      if (c != r) rows.put(c, r, val[k]);
    }
  SB2_TRY(rows.finish());
  Csr F;
  SB2_TRY(factor_sym(n, rows.out, *params, F));
  std::unique_ptr<sb2_ilut> f = to_handle(n, F);
  f->perm_row.assign(perm, perm + n);
  f->perm_col = f->perm_row;
  *out = f.release();
  return SB2_OK;
} SB2_CATCH

int sb2_ilut_size(const sb2_ilut* f, int* n, int* nnz) try {
  if (!f) return SB2_ERR_INVALID_VALUE;
  if (n) *n = f->n;
  if (nnz) *nnz = (int)f->find.size();
  return SB2_OK;
} SB2_CATCH

int sb2_ilut_arrays(const sb2_ilut* f, int* fptr, int* find, double* fval, int* perm_row,
                    int* perm_col) try {
  if (!f) return SB2_ERR_INVALID_VALUE;
  if (fptr) std::copy(f->fptr.begin(), f->fptr.end(), fptr);
  if (find) std::copy(f->find.begin(), f->find.end(), find);
  if (fval) std::copy(f->fval.begin(), f->fval.end(), fval);
  if (perm_row) std::copy(f->perm_row.begin(), f->perm_row.end(), perm_row);
  if (perm_col) std::copy(f->perm_col.begin(), f->perm_col.end(), perm_col);
  return SB2_OK;
} SB2_CATCH

int sb2_ilut_destroy(sb2_ilut* f) try {
  delete f;
  return SB2_OK;
} SB2_CATCH

}  // extern "C"
