// Thin C entry points over the UNMODIFIED reference (Seldon) templates.
//
// This file is test infrastructure: it is compiled, by oracle/Makefile, against
// the Seldon headers where they lie in the reference tree, into
// oracle/_ref/libseldon_ref*.so.  Only the test-suite and the CPU-baseline leg
// of bench.py load it.  Every arithmetic step it runs is Seldon's own:
//   MltAdd RowSparse        computation/basic_functions/Functions_MatVect.cxx:398-431
//   MltAdd RowSymSparse     computation/basic_functions/Functions_MatVect.cxx:526-564
//   MltAdd Trans RowSparse  computation/basic_functions/Functions_MatVect.cxx:729-758
//   Cg / BiCgStab / Gmres   computation/solver/iterative/{Cg,BiCgStab,Gmres}.cxx
//   Cgs / TfQmr / MinRes    computation/solver/iterative/{Cgs,TfQmr,MinRes}.cxx
//   QCgs, BiCg              computation/solver/iterative/{QCgs,BiCg}.cxx
//   Gcr, BiCgStabl          computation/solver/iterative/{Gcr,BiCgStabl}.cxx
//                           (never with an input where they cannot return:
//                           see orc_gcr_impl, orc_bicgstabl_impl)
//   SOR                     matrix_sparse/Relaxation_MatVect.cxx:41-95, 176-298
//   SorPreconditioner       computation/solver/preconditioner/Precond_Ssor.cxx:24-90
//
// Two pieces are not in the reference and are supplied here:
//   * Solve(ColUpTriang) - Gmres.cxx:166 needs it and Seldon only provides it
//     through cblas (computation/interfaces/Blas_2.cxx:3226-3238).  The
//     overload below is the netlib DTRSV column sweep (UPLO=U, TRANS=N,
//     DIAG=N), the published reference-BLAS order.
//   * JacobiPreconditioner - z_i = r_i / A(i,i), with A(i,i) read through
//     Seldon's own Matrix_Sparse::operator() (Matrix_Sparse.cxx:1051-1083).
//
// Matrices and vectors wrap the caller's buffers through SetData/Nullify
// (Matrix_Sparse.cxx:397-412), so nothing is copied.

// The ILUT preconditioner (computation/solver/preconditioner/) is compiled
// in only with SELDON_WITH_PRECONDITIONING (SeldonSolver.hxx:49-51).  As
// shipped it does not compile: GetIlut calls param.GetFactorizationType()
// (IlutPreconditioning.cxx:509, SymmetricIlutPreconditioning.cxx:38) while
// the class declares GetFactorisationType() (IlutPreconditioning.hxx:70).
// The macro below maps the one misspelt name; nothing else is changed.
#define SELDON_WITH_PRECONDITIONING
#define GetFactorizationType GetFactorisationType

#include "Seldon.hxx"

namespace Seldon
{
  // Back-substitution for the (i x i) upper-triangular GMRES Hessenberg.
  template <class Prop0, class Allocator0, class Allocator1>
  void Solve(const Matrix<double, Prop0, ColUpTriang, Allocator0>& A,
             Vector<double, VectFull, Allocator1>& X)
  {
    int n = A.GetN();
    for (int j = n - 1; j >= 0; j--)
      if (X(j) != 0.0)
        {
          X(j) = X(j) / A(j, j);
          double t = X(j);
          for (int i = j - 1; i >= 0; i--)
            X(i) = X(i) - t * A(i, j);
        }
  }
}

#include "SeldonSolver.hxx"
// Harwell-Boeing files: Seldon.hxx does not include these (users do)
#include "matrix_sparse/IOMatrixMarket.cxx"

using namespace Seldon;

namespace
{
  typedef Matrix<double, General, RowSparse> GenMat;
  typedef Matrix<double, Symmetric, RowSymSparse> SymMat;
  typedef Vector<double> Vec;

  struct Wrap
  {
    GenMat G;
    SymMat S;
    bool sym;
    Wrap(int m, int n, int nnz, const int* ptr, const int* ind,
         const double* val, int sym_)
      : sym(sym_ != 0)
    {
      if (sym)
        S.SetData(m, n, nnz, const_cast<double*>(val),
                  const_cast<int*>(ptr), const_cast<int*>(ind));
      else
        G.SetData(m, n, nnz, const_cast<double*>(val),
                  const_cast<int*>(ptr), const_cast<int*>(ind));
    }
    ~Wrap() { G.Nullify(); S.Nullify(); }
  };

  struct VWrap
  {
    Vec v;
    VWrap(int n, const double* p) { v.SetData(n, const_cast<double*>(p)); }
    ~VWrap() { v.Nullify(); }
  };

  // Jacobi preconditioner: the reference has none; it is written here in the
  // shape of Preconditioner_Base (Iterative.hxx:24-39).
  class JacobiPreconditioner
  {
  public:
    Vec diag;
    template <class Mat>
    void Init(const Mat& A)
    {
      diag.Reallocate(A.GetM());
      for (int i = 0; i < A.GetM(); i++)
        diag(i) = A(i, i);
    }
    template <class Mat, class V>
    void Solve(const Mat&, const V& r, V& z)
    {
      for (int i = 0; i < r.GetM(); i++)
        z(i) = r(i) / diag(i);
    }
    template <class Mat, class V>
    void TransSolve(const Mat& A, const V& r, V& z) { Solve(A, r, z); }
  };

  template <class Mat, class Prec>
  int run_solver(int which, Mat& A, Vec& x, const Vec& b, Prec& M,
                 Iteration<double>& it)
  {
    switch (which)
      {
      case 0: return Cg(A, x, b, M, it);
      case 1: return BiCgStab(A, x, b, M, it);
      case 2: return Gmres(A, x, b, M, it);
      case 3: return Cgs(A, x, b, M, it);
      case 4: return TfQmr(A, x, b, M, it);
      case 5: return MinRes(A, x, b, M, it);
      case 6: return Gcr(A, x, b, M, it);
      case 7: return BiCgStabl(A, x, b, M, it);
      case 8: return QCgs(A, x, b, M, it);
      case 9: return BiCg(A, x, b, M, it);
      case 10: return CoCg(A, x, b, M, it);
      case 11: return Cgne(A, x, b, M, it);
      case 12: return BiCgcr(A, x, b, M, it);
      case 13: return Lsqr(A, x, b, M, it);
      case 14: return QmrSym(A, x, b, M, it);
      case 15: return Symmlq(A, x, b, M, it);
      default: return -100;
      }
  }

  template <class Mat>
  int solve_mat(int which, Mat& A, int precond, double omega, int sor_iter,
                int sor_sym, Vec& x, const Vec& b, double tol, int max_iter,
                int restart, int init_guess_null, int print_level,
                int* nb_iter)
  {
    Iteration<double> it(max_iter, tol);
    it.SetRestart(restart);
    it.SetInitGuess(init_guess_null != 0);
    if (print_level <= 0)
      it.HideMessages();
    else if (print_level >= 6)
      it.ShowFullHistory();
    else
      it.ShowMessages();
    int code;
    if (precond == 0)
      {
        Preconditioner_Base M;
        code = run_solver(which, A, x, b, M, it);
      }
    else if (precond == 1)
      {
        JacobiPreconditioner M;
        M.Init(A);
        code = run_solver(which, A, x, b, M, it);
      }
    else
      {
        SorPreconditioner<double> M;
        M.SetParameterRelaxation(omega);
        M.SetNumberIterations(sor_iter);
        if (sor_sym)
          M.InitSymmetricPreconditioning();
        else
          M.InitUnSymmetricPreconditioning();
        code = run_solver(which, A, x, b, M, it);
      }
    *nb_iter = it.GetNumberIteration();
    return code;
  }
}

extern "C"
{
  // Seldon's binary matrix format through its own Write/Read
  // (Matrix_Sparse.cxx:1531-1556, 1650-1680; Matrix_SymSparse.cxx:1440-1457).
  int ref_write_csr(const char* path, int m, int n, int nnz, const int* ptr,
                    const int* ind, const double* val, int sym)
  {
    Wrap A(m, n, nnz, ptr, ind, val, sym);
    if (sym)
      A.S.Write(std::string(path));
    else
      A.G.Write(std::string(path));
    return 0;
  }

  // Sizes of a binary matrix file read by Seldon (m, n, stored nonzeros).
  int ref_read_csr_sizes(const char* path, int sym, int* m, int* n, int* nnz)
  {
    if (sym)
      {
        SymMat S;
        S.Read(std::string(path));
        *m = S.GetM(); *n = S.GetN(); *nnz = S.GetNonZeros();
      }
    else
      {
        GenMat G;
        G.Read(std::string(path));
        *m = G.GetM(); *n = G.GetN(); *nnz = G.GetNonZeros();
      }
    return 0;
  }

  // Arrays of a binary matrix file read by Seldon (sizes from the above).
  int ref_read_csr(const char* path, int sym, int* ptr, int* ind, double* val)
  {
    GenMat G;
    SymMat S;
    int m, nnz;
    const int* p;
    const int* i;
    const double* v;
    if (sym)
      {
        S.Read(std::string(path));
        m = S.GetM(); nnz = S.GetNonZeros(); p = S.GetPtr(); i = S.GetInd(); v = S.GetData();
      }
    else
      {
        G.Read(std::string(path));
        m = G.GetM(); nnz = G.GetNonZeros(); p = G.GetPtr(); i = G.GetInd(); v = G.GetData();
      }
    for (int k = 0; k <= m; k++) ptr[k] = p[k];
    for (int k = 0; k < nnz; k++) { ind[k] = i[k]; val[k] = v[k]; }
    return 0;
  }

  // Seldon's text format (Matrix_Sparse.cxx:1568-1616, 1692-1724): one
  // "row column value" line per entry, 1-based.
  int ref_write_text(const char* path, int m, int n, int nnz, const int* ptr,
                     const int* ind, const double* val, int sym)
  {
    Wrap A(m, n, nnz, ptr, ind, val, sym);
    if (sym)
      A.S.WriteText(std::string(path));
    else
      A.G.WriteText(std::string(path));
    return 0;
  }

  // ReadText into a matrix; sizes first, then the arrays (two calls, each
  // reading the file).
  int ref_read_text_sizes(const char* path, int sym, int* m, int* n, int* nnz)
  {
    if (sym)
      {
        SymMat S;
        S.ReadText(std::string(path));
        *m = S.GetM(); *n = S.GetN(); *nnz = S.GetNonZeros();
      }
    else
      {
        GenMat G;
        G.ReadText(std::string(path));
        *m = G.GetM(); *n = G.GetN(); *nnz = G.GetNonZeros();
      }
    return 0;
  }

  int ref_read_text(const char* path, int sym, int* ptr, int* ind, double* val)
  {
    GenMat G;
    SymMat S;
    int m, nnz;
    const int* p;
    const int* i;
    const double* v;
    if (sym)
      {
        S.ReadText(std::string(path));
        m = S.GetM(); nnz = S.GetNonZeros(); p = S.GetPtr(); i = S.GetInd(); v = S.GetData();
      }
    else
      {
        G.ReadText(std::string(path));
        m = G.GetM(); nnz = G.GetNonZeros(); p = G.GetPtr(); i = G.GetInd(); v = G.GetData();
      }
    for (int k = 0; k <= m && p; k++) ptr[k] = p[k];
    for (int k = 0; k < nnz; k++) { ind[k] = i[k]; val[k] = v[k]; }
    return 0;
  }

  // WriteHarwellBoeing (IOMatrixMarket.cxx:394-511) of a RowSparse matrix.
  int ref_write_hb(const char* path, int m, int n, int nnz, const int* ptr,
                   const int* ind, const double* val)
  {
    Wrap A(m, n, nnz, ptr, ind, val, 0);
    WriteHarwellBoeing(A.G, std::string(path));
    return 0;
  }

  // ReadHarwellBoeing (IOMatrixMarket.cxx:45-329) into ColSparse: sizes,
  // then the arrays.  Returns -1 with *msg filled when Seldon throws.
  int ref_read_hb(const char* path, int* m, int* n, int* nnz, int cap_cols,
                  int cap_nnz, int* colptr, int* rowind, double* val,
                  char* msg, int msg_cap)
  {
    try
      {
        Matrix<double, General, ColSparse> C;
        ReadHarwellBoeing(std::string(path), C);
        *m = C.GetM(); *n = C.GetN(); *nnz = C.GetDataSize();
        if (*n > cap_cols || *nnz > cap_nnz) return -2;
        for (int k = 0; k <= *n; k++) colptr[k] = C.GetPtr()[k];
        for (int k = 0; k < *nnz; k++) { rowind[k] = C.GetInd()[k]; val[k] = C.GetData()[k]; }
        return 0;
      }
    catch (Error& e)
      {
        std::snprintf(msg, msg_cap, "%s", e.What().c_str());
        return -1;
      }
  }

  // Seldon's binary vector format (Vector.cxx:848-870): size, then values.
  int ref_write_vector(const char* path, int n, const double* x, int with_size)
  {
    VWrap v(n, x);
    v.v.Write(std::string(path), with_size != 0);
    return 0;
  }

  // Y = beta*Y + alpha*op(A)*X through Seldon's MltAdd.
  int ref_mltadd(int m, int n, int nnz, const int* ptr, const int* ind,
                 const double* val, int sym, int trans, double alpha,
                 const double* x, double beta, double* y)
  {
    Wrap A(m, n, nnz, ptr, ind, val, sym);
    int nx = trans ? m : n, ny = trans ? n : m;
    VWrap X(nx, x), Y(ny, y);
    if (sym)
      {
        if (trans)
          MltAdd(alpha, SeldonTrans, A.S, X.v, beta, Y.v);
        else
          MltAdd(alpha, A.S, X.v, beta, Y.v);
      }
    else
      {
        if (trans)
          MltAdd(alpha, SeldonTrans, A.G, X.v, beta, Y.v);
        else
          MltAdd(alpha, A.G, X.v, beta, Y.v);
      }
    return 0;
  }

  // Seldon's SOR sweeps (type 2 forward, 3 backward, 0 both).
  int ref_sor(int m, int nnz, const int* ptr, const int* ind, const double* val,
              int sym, double* x, const double* b, double omega, int iter,
              int type_ssor)
  {
    Wrap A(m, m, nnz, ptr, ind, val, sym);
    VWrap X(m, x), B(m, b);
    if (sym)
      SOR(A.S, X.v, B.v, omega, iter, type_ssor);
    else
      SOR(A.G, X.v, B.v, omega, iter, type_ssor);
    return 0;
  }

  // which: 0 Cg, 1 BiCgStab, 2 Gmres, 3 Cgs, 4 TfQmr, 5 MinRes, 6 Gcr,
  // 7 BiCgStabl, 8 QCgs, 9 BiCg, 10 CoCg, 11 Cgne.  precond: 0 identity,
  // 1 Jacobi, 2 SOR.
  // Returns Seldon's Iteration::ErrorCode(); *nb_iter the iteration count.
  int ref_solve(int which, int m, int nnz, const int* ptr, const int* ind,
                const double* val, int sym, int precond, double omega,
                int sor_iter, int sor_sym, double* x, const double* b,
                double tol, int max_iter, int restart, int init_guess_null,
                int print_level, int* nb_iter)
  {
    Wrap A(m, m, nnz, ptr, ind, val, sym);
    VWrap X(m, x), B(m, b);
    if (sym)
      return solve_mat(which, A.S, precond, omega, sor_iter, sor_sym, X.v,
                       B.v, tol, max_iter, restart, init_guess_null,
                       print_level, nb_iter);
    return solve_mat(which, A.G, precond, omega, sor_iter, sor_sym, X.v, B.v,
                     tol, max_iter, restart, init_guess_null, print_level,
                     nb_iter);
  }

  // Seldon's coordinate -> CSR assembly (ConvertMatrix_from_Coordinates,
  // Matrix_Conversions.cxx:1291-1334 RowSparse, 1397-1467 RowSymSparse) into
  // a matrix that starts as an empty m_min x n_min one.  The caller's
  // buffers hold at least cap_rows+1 row pointers and nnz entries; the
  // result's sizes go to *m, *n, *nnz_out (-1 when they would not fit).
  int ref_coo_to_csr(int nnz, const int* row, const int* col,
                     const double* val, int index, int m_min, int n_min,
                     int sym, int cap_rows, int* m, int* n, int* nnz_out,
                     int* ptr, int* ind, double* vout)
  {
    Vector<int> R(nnz), C(nnz);
    Vec V(nnz);
    for (int i = 0; i < nnz; i++)
      {
        R(i) = row[i];
        C(i) = col[i];
        V(i) = val[i];
      }
    const int *p, *q;
    const double* v;
    if (sym)
      {
        SymMat A;
        A.Reallocate(m_min, m_min);
        ConvertMatrix_from_Coordinates(R, C, V, A, index);
        *m = A.GetM();
        *n = A.GetN();
        *nnz_out = A.GetDataSize();
        p = A.GetPtr(); q = A.GetInd(); v = A.GetData();
        if (*m > cap_rows) return -1;
        for (int i = 0; i <= *m; i++) ptr[i] = p[i];
        for (int k = 0; k < *nnz_out; k++) { ind[k] = q[k]; vout[k] = v[k]; }
      }
    else
      {
        GenMat A;
        A.Reallocate(m_min, n_min);
        ConvertMatrix_from_Coordinates(R, C, V, A, index);
        *m = A.GetM();
        *n = A.GetN();
        *nnz_out = A.GetDataSize();
        p = A.GetPtr(); q = A.GetInd(); v = A.GetData();
        if (*m > cap_rows) return -1;
        for (int i = 0; i <= *m; i++) ptr[i] = p[i];
        for (int k = 0; k < *nnz_out; k++) { ind[k] = q[k]; vout[k] = v[k]; }
      }
    return 0;
  }

  // ------------------------------------------------------------ ILUT
  // IlutPreconditioning (IlutPreconditioning.cxx): Seldon factorizes with its
  // own GetIlut; the factor (ArrayRowSparse / ArrayRowSymSparse rows in
  // stored order) and the permutations are handed back as flat arrays.  One
  // factorization is held at a time (test infrastructure, one thread).
  typedef IlutPreconditioning<double, double> Ilut;

  // Reads the factor out of the protected members through pointers to
  // members named in a derived class.
  struct IlutAccess : Ilut
  {
    static const Matrix<double, General, ArrayRowSparse>& unsym(const Ilut& p)
    { return p.*(&IlutAccess::mat_unsym); }
    static const Matrix<double, Symmetric, ArrayRowSymSparse>& sym(const Ilut& p)
    { return p.*(&IlutAccess::mat_sym); }
    static const IVect& prow(const Ilut& p) { return p.*(&IlutAccess::permutation_row); }
    static const IVect& pcol(const Ilut& p) { return p.*(&IlutAccess::permutation_col); }
  };

  Ilut* g_ilut = 0;
  bool g_ilut_sym = false;

  // type_ilu: ILUT, ILU_D, ILUT_K, ILU_0, MILU_0, ILU_K (0..5).  sym selects
  // RowSymSparse input and the symmetric algorithm (FactorizeSymMatrix);
  // otherwise RowSparse and FactorizeMatrix.  perm may be NULL (identity).
  int ref_ilut_factor(int n, int nnz, const int* ptr, const int* ind,
                      const double* val, int sym, const int* perm, int type_ilu,
                      int fill_level, int additional_fill, int mbloc,
                      double alpha, double droptol, double permtol,
                      int* nnz_factor)
  {
    delete g_ilut;
    g_ilut = new Ilut();
    g_ilut->SetFactorisationType(type_ilu);
    g_ilut->SetFillLevel(fill_level);
    g_ilut->SetAdditionalFillNumber(additional_fill);
    g_ilut->SetPivotBlockInteger(mbloc);
    g_ilut->SetDiagonalCoefficient(alpha);
    g_ilut->SetDroppingThreshold(droptol);
    g_ilut->SetPivotThreshold(permtol);
    IVect P(n);
    for (int i = 0; i < n; i++)
      P(i) = perm ? perm[i] : i;
    Vector<int> p(n + 1), q(nnz);
    Vec v(nnz);
    for (int i = 0; i <= n; i++) p(i) = ptr[i];
    for (int k = 0; k < nnz; k++) { q(k) = ind[k]; v(k) = val[k]; }
    g_ilut_sym = sym != 0;
    int total = 0;
    if (g_ilut_sym)
      {
        SymMat S(n, n, v, p, q);
        g_ilut->SetSymmetricAlgorithm();
        g_ilut->FactorizeSymMatrix(P, S);
        const Matrix<double, Symmetric, ArrayRowSymSparse>& F = IlutAccess::sym(*g_ilut);
        for (int i = 0; i < n; i++) total += F.GetRowSize(i);
      }
    else
      {
        GenMat G(n, n, v, p, q);
        g_ilut->SetUnsymmetricAlgorithm();
        g_ilut->FactorizeMatrix(P, G);
        const Matrix<double, General, ArrayRowSparse>& F = IlutAccess::unsym(*g_ilut);
        for (int i = 0; i < n; i++) total += F.GetRowSize(i);
      }
    *nnz_factor = total;
    return 0;
  }

  // The held factor: fptr[n+1], find/fval[nnz_factor], permutation_row and
  // permutation_col (the row permutation again for the symmetric algorithm).
  int ref_ilut_get(int n, int* fptr, int* find, double* fval, int* perm_row,
                   int* perm_col)
  {
    if (!g_ilut) return -1;
    fptr[0] = 0;
    int t = 0;
    for (int i = 0; i < n; i++)
      {
        int len = g_ilut_sym ? IlutAccess::sym(*g_ilut).GetRowSize(i)
          : IlutAccess::unsym(*g_ilut).GetRowSize(i);
        for (int k = 0; k < len; k++, t++)
          {
            // the symmetric factor keeps 1/D in position 0, whose index
            // GetIlut leaves unset and SolveLU never reads: i is written
            find[t] = g_ilut_sym ? (k == 0 ? i : IlutAccess::sym(*g_ilut).Index(i, k))
              : IlutAccess::unsym(*g_ilut).Index(i, k);
            fval[t] = g_ilut_sym ? IlutAccess::sym(*g_ilut).Value(i, k)
              : IlutAccess::unsym(*g_ilut).Value(i, k);
          }
        fptr[i + 1] = t;
      }
    const IVect& pr = IlutAccess::prow(*g_ilut);
    const IVect& pc = g_ilut_sym ? pr : IlutAccess::pcol(*g_ilut);
    for (int i = 0; i < n; i++) { perm_row[i] = pr(i); perm_col[i] = pc(i); }
    return 0;
  }

  // z = M^{-1} r (Solve) or M^{-T} r (TransSolve) with the held factor.
  int ref_ilut_solve(int trans, int n, const double* r, double* z)
  {
    if (!g_ilut) return -1;
    Vec R(n), Z(n);
    for (int i = 0; i < n; i++) R(i) = r[i];
    Z.Zero();
    GenMat dummy;
    if (trans)
      g_ilut->TransSolve(dummy, R, Z);
    else
      g_ilut->Solve(dummy, R, Z);
    for (int i = 0; i < n; i++) z[i] = Z(i);
    return 0;
  }

  // Cg / BiCgStab / Gmres (which 0/1/2) preconditioned by the held factor.
  int ref_solve_ilut(int which, int m, int nnz, const int* ptr, const int* ind,
                     const double* val, int sym, double* x, const double* b,
                     double tol, int max_iter, int restart, int init_guess_null,
                     int* nb_iter)
  {
    if (!g_ilut) return -100;
    Wrap A(m, m, nnz, ptr, ind, val, sym);
    VWrap X(m, x), B(m, b);
    Iteration<double> it(max_iter, tol);
    it.SetRestart(restart);
    it.SetInitGuess(init_guess_null != 0);
    it.HideMessages();
    int code = sym ? run_solver(which, A.S, X.v, B.v, *g_ilut, it)
      : run_solver(which, A.G, X.v, B.v, *g_ilut, it);
    *nb_iter = it.GetNumberIteration();
    return code;
  }

  // Seldon's generic BLAS-1 loops (Functions_Vector.cxx), for pinning.
  double ref_dot(int n, const double* x, const double* y)
  {
    VWrap X(n, x), Y(n, y);
    return DotProd(X.v, Y.v);
  }
  double ref_norm2(int n, const double* x)
  {
    VWrap X(n, x);
    return Norm2(X.v);
  }
  void ref_genrot(double* a, double* b, double* c, double* s)
  {
    GenRot(*a, *b, *c, *s);
  }
}
