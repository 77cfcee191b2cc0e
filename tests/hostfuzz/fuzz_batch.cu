// Random batches of systems, well-formed and malformed (system ranges that
// go backwards, row pointers that start off 0, fall or go negative, entries
// outside their own system), through sb2_batch_create's host validation and
// sb2_batch_destroy, under AddressSanitizer and UBSan, with cuda_stubs.cpp
// standing in for the device.  Every batch it accepts is checked
// independently.  Argument: the number of batches.  Test infrastructure only.
#include "../../seldon_b200/csrc/batch.cu"
#include <cstdio>
#include <cstdlib>
#include <random>
int main(int argc, char** argv) {
  const int trials = argc > 1 ? atoi(argv[1]) : 4000;
  std::mt19937_64 g(11);
  int ok = 0, bad = 0;
  for (int trial = 0; trial < trials; trial++) {
    const int nsys = (int)(g() % 6);
    std::vector<int> sys_row(1, 0), ptr(1, 0), ind;
    std::vector<double> val;
    for (int s = 0; s < nsys; s++) {
      const int rows = (int)(g() % 5);
      const int a = sys_row.back();
      for (int i = 0; i < rows; i++) {
        const int len = (int)(g() % 4);
        for (int k = 0; k < len; k++) { ind.push_back(a + (int)(g() % rows)); val.push_back(1.0); }
        ptr.push_back((int)ind.size());
      }
      sys_row.push_back(a + rows);
    }
    const int m = sys_row.back();
    const int flaw = (int)(g() % 7);
    if (flaw == 1 && nsys > 1) std::swap(sys_row[1], sys_row[nsys]);
    if (flaw == 2 && m > 0) ptr[1 + g() % m] = -1 - (int)(g() % 5);
    if (flaw == 3 && m > 0) ptr[1 + g() % m] += 10 + (int)(g() % 10);
    if (flaw == 4 && !ind.empty()) ind[g() % ind.size()] += (g() % 2) ? 7 : -7;
    if (flaw == 5) ptr[0] = (g() % 2) ? 3 : -3;
    // the arrays are padded so that a flawed header never sends the
    // validator past what this driver allocated
    std::vector<int> ptr_pad(ptr), ind_pad(ind);
    ptr_pad.resize(ptr.size() + 64, 0);
    ind_pad.resize(ind.size() + 64, 0);
    std::vector<double> val_pad(val);
    val_pad.resize(val.size() + 64, 0.0);
    sb2_batch* B = nullptr;
    int st = sb2_batch_create(nsys, sys_row.data(), ptr_pad.data(), ind_pad.data(),
                              val_pad.data(), &B);
    if (st != SB2_OK) { bad++; continue; }
    ok++;
    // (on the arrays the call saw, padding included)
    const std::vector<int>& P = ptr_pad;
    const std::vector<int>& I = ind_pad;
    bool valid = sys_row[0] == 0 && P[0] == 0;
    for (int s = 0; s < nsys; s++) valid = valid && sys_row[s + 1] >= sys_row[s];
    const int mm = sys_row[nsys];
    for (int i = 0; valid && i < mm; i++) valid = P[i + 1] >= P[i];
    valid = valid && P[mm] <= (int)I.size();
    for (int s = 0; valid && s < nsys; s++)
      for (int i = sys_row[s]; i < sys_row[s + 1]; i++)
        for (int k = P[i]; k < P[i + 1]; k++)
          valid = valid && I[k] >= sys_row[s] && I[k] < sys_row[s + 1];
    if (!valid) { printf("ACCEPTED AN INVALID BATCH: trial %d\n", trial); return 1; }
    sb2_batch_destroy(B);
  }
  printf("created %d refused %d\n", ok, bad);
}
