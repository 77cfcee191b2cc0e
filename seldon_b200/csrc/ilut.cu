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

struct Row {
  std::vector<int> idx;
  std::vector<double> val;
};

int factor(int n, const std::vector<Row>& A0, const sb2_ilut_params& p, std::vector<Row>& F,
           std::vector<int>& iperm, std::vector<int>& rperm) {
  const bool variable_fill = (p.type == SB2_ILUT_K);
  const bool standard_dropping = (p.type == SB2_ILU_D);
  int lfil = p.fill_level;
  if (lfil < 0) return SB2_ERR_INVALID_VALUE;
  F.assign(n, Row());
  std::vector<double> w(n, 0.0);
  std::vector<int> wi(n, -1), where(n, -1), diag_at(n, -1);
  iperm.resize(n);
  rperm.resize(n);
  for (int i = 0; i < n; i++) iperm[i] = rperm[i] = i;
  for (int i = 0; i < n; i++) {
    const Row& a = A0[i];
    const int size_row = (int)a.idx.size();
    double tnorm = 0.0;
    for (int k = 0; k < size_row; k++)
      if (a.val[k] != 0.0) tnorm += std::fabs(a.val[k]);
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
      const int c = rperm[a.idx[k]];
      const double t = a.val[k];
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
        fact = w[jc] * F[jrow].val[diag_at[jrow]];
        if (!standard_dropping && std::fabs(fact) <= p.droptol) dropped = true;
      }
      if (!dropped) {
        const Row& u = F[jrow];
        for (int k = diag_at[jrow] + 1; k < (int)u.idx.size(); k++) {
          const double s = fact * u.val[k];
          const int c = rperm[u.idx[k]];
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
    Row& f = F[i];
    f.idx.clear();
    f.val.clear();
    for (int k = 0; k < len; k++) {
      f.val.push_back(w[k]);
      f.idx.push_back(iperm[wi[k]]);
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
      f.idx.push_back(iperm[wi[k]]);
      f.val.push_back(w[k]);
    }
    if (standard_dropping) w[i] += p.alpha * dropsum;
    if (w[i] == 0.0) w[i] = (p.droptol + 1e-4) * tnorm;
    f.val[index_diag] = 1.0 / w[i];
  }
  for (int i = 0; i < n; i++)
    for (int& c : F[i].idx) c = rperm[c];
  return SB2_OK;
}

// The symmetric algorithm (SymmetricIlutPreconditioning.cxx:27-346): B holds
// the full rows of the symmetric matrix, sorted by column; row i of the
// factor keeps 1/D(i) first and then its U part (no pivoting, no L part
// kept); at the end every U entry is scaled by its row's 1/D.
int factor_sym(int n, const std::vector<Row>& B, const sb2_ilut_params& p,
               std::vector<Row>& F) {
  const bool variable_fill = (p.type == SB2_ILUT_K);
  const bool standard_dropping = (p.type == SB2_ILU_D);
  int lfil = p.fill_level;
  if (lfil < 0) return SB2_ERR_INVALID_VALUE;
  F.assign(n, Row());
  std::vector<double> w(n, 0.0);
  std::vector<int> wi(n, -1), where(n, -1);
  for (int i = 0; i < n; i++) {
    const Row& a = B[i];
    const int size_row = (int)a.idx.size();
    double tnorm = 0.0;
    for (int k = 0; k < size_row; k++) tnorm += std::fabs(a.val[k]);
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
      const int c = a.idx[k];
      const double t = a.val[k];
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
        fact = w[jc] * F[jrow].val[0];
        if (!standard_dropping && std::fabs(fact) <= p.droptol) dropped = true;
      }
      if (!dropped) {
        const Row& u = F[jrow];
        for (int k = 1; k < (int)u.idx.size(); k++) {
          const double s = fact * u.val[k];
          const int c = u.idx[k];
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
    Row& f = F[i];
    f.idx.assign(1, i);  // 1/D(i); the reference leaves this index unset
    f.val.assign(1, 0.0);
    for (int k = i + 1; k <= i + lu - 1; k++) {
      f.idx.push_back(wi[k]);
      f.val.push_back(w[k]);
    }
    if (standard_dropping) w[i] += p.alpha * dropsum;
    if (w[i] == 0.0) w[i] = (p.droptol + 1e-4) * tnorm;
    f.val[0] = 1.0 / w[i];
  }
  for (int i = 0; i < n; i++)
    for (size_t j = 1; j < F[i].val.size(); j++) F[i].val[j] *= F[i].val[0];
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

sb2_ilut* flatten(int n, const std::vector<Row>& F) {
  sb2_ilut* f = new sb2_ilut();
  f->n = n;
  f->fptr.assign(n + 1, 0);
  for (int i = 0; i < n; i++) {
    f->find.insert(f->find.end(), F[i].idx.begin(), F[i].idx.end());
    f->fval.insert(f->fval.end(), F[i].val.begin(), F[i].val.end());
    f->fptr[i + 1] = (int)f->find.size();
  }
  return f;
}

// Rows sorted by column, a repeated column refused.
int sort_rows(std::vector<std::vector<std::pair<int, double>>>& rows, std::vector<Row>& out) {
  out.assign(rows.size(), Row());
  for (size_t i = 0; i < rows.size(); i++) {
    auto& e = rows[i];
    std::sort(e.begin(), e.end(),
              [](const std::pair<int, double>& x, const std::pair<int, double>& y) {
                return x.first < y.first;
              });
    for (size_t k = 1; k < e.size(); k++)
      if (e[k].first == e[k - 1].first) return SB2_ERR_NOT_SUPPORTED;
    for (const auto& q : e) {
      out[i].idx.push_back(q.first);
      out[i].val.push_back(q.second);
    }
  }
  return SB2_OK;
}

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
  std::vector<std::vector<std::pair<int, double>>> rows(n);
  for (int i = 0; i < n; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++) rows[perm[i]].emplace_back(perm[ind[k]], val[k]);
  std::vector<Row> A0;
  SB2_TRY(sort_rows(rows, A0));
  std::vector<Row> F;
  std::vector<int> iperm, rperm;
  SB2_TRY(factor(n, A0, *params, F, iperm, rperm));
  std::unique_ptr<sb2_ilut> f(flatten(n, F));
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
  std::vector<std::vector<std::pair<int, double>>> rows(n);
  for (int i = 0; i < n; i++)
    for (int k = ptr[i]; k < ptr[i + 1]; k++) {
      if (ind[k] < i) return SB2_ERR_INVALID_CSR;  // upper triangle only
      int r = perm[i], c = perm[ind[k]];
      if (c < r) std::swap(r, c);
      rows[r].emplace_back(c, val[k]);
      if (c != r) rows[c].emplace_back(r, val[k]);
    }
  std::vector<Row> B;
  SB2_TRY(sort_rows(rows, B));
  std::vector<Row> F;
  SB2_TRY(factor_sym(n, B, *params, F));
  std::unique_ptr<sb2_ilut> f(flatten(n, F));
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
