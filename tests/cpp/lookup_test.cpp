// Element access of the device matrix types (operator(), Print) reads the
// downloaded arrays with DeviceCsr::Lookup.  This host-only program checks
// Lookup against Seldon's own operator() (Matrix_Sparse.cxx:1054-1083,
// Matrix_SymSparse.cxx:1013-1053) on random RowSparse and RowSymSparse
// matrices, with unsorted and repeated columns and empty rows: no device
// call is made.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "Seldon.hxx"
#include "SeldonSolver.hxx"
#include "SeldonB200.hxx"

using namespace Seldon;

template <int Sym>
struct Probe: public b200::DeviceCsr<Sym>
{
  using b200::DeviceCsr<Sym>::Lookup;
};

template <int Sym, class HostMatrix>
int check(std::mt19937_64& g, int trials)
{
  int bad = 0;
  for (int t = 0; t < trials; t++)
    {
      const int m = 1 + g() % 12, n = Sym ? m : 1 + g() % 12;
      std::vector<int> ptr(1, 0), ind;
      std::vector<double> val;
      for (int i = 0; i < m; i++)
        {
          const int len = g() % 5;
          for (int k = 0; k < len; k++)
            {
              const int lo = Sym ? i : 0;
              ind.push_back(lo + g() % (n - lo));
              val.push_back(1.0 + g() % 100);
            }
          if (g() % 2)  // sorted rows, as well as unsorted ones
            std::sort(ind.begin() + ptr.back(), ind.end());
          ptr.push_back(ind.size());
        }
      Vector<double> v((int)val.size());
      Vector<int> p((int)ptr.size()), c((int)ind.size());
      for (size_t k = 0; k < val.size(); k++) { v(k) = val[k]; c(k) = ind[k]; }
      for (size_t k = 0; k < ptr.size(); k++) p(k) = ptr[k];
      HostMatrix A(m, n, v, p, c);
      for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++)
          if (Probe<Sym>::Lookup(ptr, ind, val, i, j) != A(i, j))
            bad++;
    }
  return bad;
}

int main()
{
  std::mt19937_64 g(5);
  const int bad_gen = check<0, Matrix<double, General, RowSparse> >(g, 2000);
  const int bad_sym = check<1, Matrix<double, Symmetric, RowSymSparse> >(g, 2000);
  std::printf("mismatches general %d symmetric %d\n", bad_gen, bad_sym);
  return bad_gen || bad_sym;
}
