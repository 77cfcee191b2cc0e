// Random matrices, orderings and option sets (ILUT, ILU_D, ILUT_K; both
// algorithms) through the host ILUT factorization (ilut.cu, compiled as
// C++), under AddressSanitizer and UBSan.  Argument: the number of
// factorizations.  Test infrastructure only.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#include <algorithm>
#include "seldon_b200.h"
int main(int argc, char** argv) {
  const int trials = argc > 1 ? atoi(argv[1]) : 20000;
  std::mt19937_64 g(1);
  int fails = 0, oks = 0;
  for (int trial = 0; trial < trials; trial++) {
    int n = 1 + g() % (trial % 10 == 0 ? 400 : 40);
    double dens = (g() % 100) / 100.0;
    std::vector<int> ptr(1, 0), ind;
    std::vector<double> val;
    bool sym = trial % 3 == 0;
    std::normal_distribution<double> N(0, 1);
    for (int i = 0; i < n; i++) {
      for (int j = sym ? i : 0; j < n; j++) {
        bool on = (j == i) ? (g() % 10 != 0) : (g() % 1000 < dens * 300);
        if (on) { ind.push_back(j); val.push_back(j == i ? 4 + N(g) : (g() % 7 == 0 ? 0.0 : N(g))); }
      }
      ptr.push_back(ind.size());
    }
    std::vector<int> perm(n);
    for (int i = 0; i < n; i++) perm[i] = i;
    if (g() % 2) std::shuffle(perm.begin(), perm.end(), g);
    sb2_ilut_params p{};
    p.type = g() % 3; p.fill_level = g() % 12; p.additional_fill = g() % 5;
    p.mbloc = 1 + g() % (n + 2); p.alpha = (g() % 3) * 0.5;
    p.droptol = (g() % 4) ? std::pow(10.0, -(double)(g() % 6)) : 0.0;
    p.permtol = (g() % 3) * 0.3;
    sb2_ilut* F = nullptr;
    int st = sym ? sb2_ilut_factor_sym(n, ptr.data(), ind.data(), val.data(), perm.data(), &p, &F)
                 : sb2_ilut_factor(n, ptr.data(), ind.data(), val.data(), perm.data(), &p, &F);
    if (st != SB2_OK) { fails++; continue; }
    oks++;
    int nn, nz;
    sb2_ilut_size(F, &nn, &nz);
    std::vector<int> fp(nn + 1), fi(std::max(nz, 1)), pr(nn), pc(nn);
    std::vector<double> fv(std::max(nz, 1));
    sb2_ilut_arrays(F, fp.data(), fi.data(), fv.data(), pr.data(), pc.data());
    sb2_ilut_destroy(F);
  }
  printf("ok %d rejected %d\n", oks, fails);
}
