// Random ILUT factors, well-formed and malformed, through
// sb2_precond_create_ilut's host planning and the host side of Solve and
// TransSolve (launches and graphs are stand-ins from cuda_stubs.cpp, so
// nothing is computed), under AddressSanitizer and UBSan.  Every factor the
// planner accepts is checked independently: each index the sweeps read lies
// in range and both permutations are permutations.  Argument: the number of
// factors.  Test infrastructure only.
#include "../../seldon_b200/csrc/precond.cu"
#include <cstdio>
#include <cstdlib>
#include <random>
int main(int argc, char** argv) {
  const int trials = argc > 1 ? atoi(argv[1]) : 3000;
  std::mt19937_64 g(3);
  int ok = 0, bad = 0;
  for (int trial = 0; trial < trials; trial++) {
    const bool sym = trial % 2 == 0;
    const int n = trial % 300 == 7 ? 70000 : 1 + (int)(g() % 120);
    std::vector<int> fptr(1, 0), find;
    std::vector<double> fval;
    for (int i = 0; i < n; i++) {
      const int nl = sym ? 0 : (i ? (int)(g() % std::min(i, 4) + (g() % 3 == 0)) : 0);
      for (int k = 0; k < nl && i > 0; k++) { find.push_back((int)(g() % i)); fval.push_back(0.1); }
      find.push_back(i);  // the pivot position
      fval.push_back(1.0);
      const int nu = i + 1 < n ? (int)(g() % 4) : 0;
      for (int k = 0; k < nu; k++) { find.push_back(i + 1 + (int)(g() % (n - i - 1))); fval.push_back(0.1); }
      fptr.push_back((int)find.size());
    }
    std::vector<int> prow(n), pcol(n);
    for (int i = 0; i < n; i++) prow[i] = pcol[i] = i;
    std::shuffle(prow.begin(), prow.end(), g);
    std::shuffle(pcol.begin(), pcol.end(), g);
    const int flaw = g() % 8;
    if (flaw == 1 && !find.empty()) find[g() % find.size()] = n + (int)(g() % 3);
    if (flaw == 2 && !find.empty()) find[g() % find.size()] = -1 - (int)(g() % 3);
    if (flaw == 3) prow[g() % n] = prow[(g() % n)];
    if (flaw == 4 && n > 1) std::swap(fptr[1], fptr[n]);
    if (flaw == 5 && !sym) {  // a row whose entries all lie below the row
      const int i = (int)(g() % n);
      for (int k = fptr[i]; k < fptr[i + 1]; k++) find[k] = i ? (int)(g() % i) : -1;
    }
    sb2_precond* M = nullptr;
    int st = sb2_precond_create_ilut(nullptr, n, fptr.data(), find.data(), fval.data(), prow.data(),
                                     pcol.data(), sym, &M);
    if (st != SB2_OK) { bad++; continue; }
    ok++;
    // independent check of what the sweeps read: L columns in [0, i), a
    // pivot position, U columns in (i, n), permutations
    bool valid = fptr[0] == 0;
    for (int i = 0; i < n && valid; i++) {
      if (fptr[i + 1] <= fptr[i]) { valid = false; break; }
      int k = fptr[i];
      if (sym) k++;
      else {
        while (k < fptr[i + 1] && find[k] < i) { if (find[k] < 0) valid = false; k++; }
        if (k == fptr[i + 1]) { valid = false; break; }
        k++;
      }
      for (; k < fptr[i + 1]; k++) if (find[k] <= i || find[k] >= n) valid = false;
    }
    std::vector<int> seen(n, 0), seen2(n, 0);
    for (int i = 0; i < n; i++) {
      if (prow[i] < 0 || prow[i] >= n || seen[prow[i]]++) valid = false;
      if (!sym && (pcol[i] < 0 || pcol[i] >= n || seen2[pcol[i]]++)) valid = false;
    }
    if (!valid) { printf("ACCEPTED AN INVALID FACTOR: trial %d\n", trial); return 1; }
    std::vector<double> r(n, 1.0), z(n, 0.0);
    for (int rep = 0; rep < 2; rep++) {
      sb2_precond_solve(M, r.data(), z.data(), nullptr);
      sb2_precond_trans_solve(M, r.data(), z.data(), nullptr);
    }
    sb2_precond_destroy(M);
  }
  printf("planned %d refused %d\n", ok, bad);
}
