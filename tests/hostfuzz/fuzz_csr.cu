// Random CSR matrices, well-formed and malformed, through sb2_csr_create's
// host work (the validator, the symmetric expansion, the stream-block, SELL
// and TMA layouts) and sb2_csr_destroy, under AddressSanitizer and UBSan,
// with cuda_stubs.cpp standing in for the device.  Argument: the number of
// matrices.  Test infrastructure only.
#include "../../seldon_b200/csrc/csr.cu"
#include <cstdio>
#include <cstdlib>
#include <random>
int main(int argc, char** argv) {
  const int trials = argc > 1 ? atoi(argv[1]) : 4000;
  std::mt19937_64 g(7);
  int ok = 0, bad = 0;
  for (int trial = 0; trial < trials; trial++) {
    const bool sym = trial % 3 == 0;
    const int m = trial % 500 == 1 ? 200000 : (int)(g() % (trial % 20 == 0 ? 3000 : 90));
    const int n = sym ? m : (trial % 13 == 5 ? 0 : (int)(g() % 90) + (m == 0 ? 0 : 1));
    std::vector<int> ptr(1, 0), ind;
    std::vector<double> val;
    const int shape = g() % 4;
    for (int i = 0; i < m; i++) {
      int len;
      if (shape == 0) len = g() % 6;
      else if (shape == 1) len = (g() % 50 == 0) ? 40 + g() % 5000 : g() % 3;  // a few long rows
      else if (shape == 2) len = g() % 40;
      else len = (i % 97 == 0) ? 600 : 0;
      const int lo = sym ? i : 0;
      const int span = (sym ? n - i : n);
      for (int k = 0; k < len && span > 0; k++) {
        ind.push_back(lo + (int)(g() % span));
        val.push_back(1.0);
      }
      ptr.push_back((int)ind.size());
    }
    if (trial % 7 == 0 && !ind.empty()) ind[g() % ind.size()] = (g() % 2) ? -1 : n + (int)(g() % 3);
    if (trial % 11 == 0 && m > 1) std::swap(ptr[1], ptr[m]);
    sb2_csr* A = nullptr;
    int st = sb2_csr_create(m, n, (int)ind.size(), ptr.data(), ind.data(), val.data(), sym, 1, &A);
    if (st == SB2_OK) { ok++; sb2_csr_destroy(A); } else bad++;
  }
  printf("created %d refused %d\n", ok, bad);
}
