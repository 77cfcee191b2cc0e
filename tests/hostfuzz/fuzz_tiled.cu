// The x-tiled layout's host planning (build_tiled) under AddressSanitizer
// and UBSan, with cuda_stubs.cpp standing in for the device: random
// operators with long rows, sorted or not, through sb2_csr_create and
// build_tiled, and an independent check of every layout accepted: each long
// row is dealt to exactly one CTA, no CTA holds more rows than it has
// threads, chunks start on 8-entry boundaries and hold at most emax entries,
// every chunk's offsets rise to its size, the two stages fit the shared
// memory the kernel is given, and reading a row back tile by tile gives its
// columns and values in stored order within each tile.  Argument: the
// number of operators.  Test infrastructure only.
#include "../../seldon_b200/csrc/csr.cu"
#include "../../seldon_b200/csrc/tiled.cu"
#include <cstdio>
#include <cstdlib>
#include <random>
namespace sb2 {
std::atomic<long long> g_wait_limit_us{2000000};
// the product launches are never reached here
SellOp<double> sell_op(const CsrArrays&) { return SellOp<double>{}; }
template <int NT, bool O>
int launch_sell_warp_rows(const SellOp<double>&, double, const double*, double, double*,
                          cudaStream_t) {
  return 0;
}
template int launch_sell_warp_rows<256, true>(const SellOp<double>&, double, const double*, double,
                                              double*, cudaStream_t);
template int launch_sell_warp_rows<256, false>(const SellOp<double>&, double, const double*,
                                               double, double*, cudaStream_t);
}  // namespace sb2
static int fail(const char* what, int trial) {
  printf("layout error (%s) in trial %d\n", what, trial);
  return 1;
}
int main(int argc, char** argv) {
  const int trials = argc > 1 ? atoi(argv[1]) : 200;
  std::mt19937_64 g(11);
  int built = 0, skipped = 0;
  for (int trial = 0; trial < trials; trial++) {
    const int m = 1 + (int)(g() % 1200);
    const int n = 1000 + (int)(g() % 40000);
    const bool sorted = trial % 2 == 0;
    const int minlen = 33 + (int)(g() % 200);
    sb2_spmv_set_tiling(minlen, (long long)(g() % 3) * 1000);
    std::vector<int> ptr(1, 0), ind;
    std::vector<double> val;
    for (int i = 0; i < m; i++) {
      const int len = (g() % 4 == 0) ? (int)(g() % 1500) : (int)(g() % 40);
      std::vector<int> cols;
      for (int k = 0; k < len; k++) cols.push_back((int)(g() % n));
      if (sorted) std::sort(cols.begin(), cols.end());
      for (int c : cols) {
        ind.push_back(c);
        val.push_back((double)ind.size());  // values identify entries
      }
      ptr.push_back((int)ind.size());
    }
    sb2_csr* A = nullptr;
    if (sb2_csr_create(m, n, (int)ind.size(), ptr.data(), ind.data(), val.data(), 0, 1, &A) != SB2_OK)
      return fail("create", trial);
    if (sb2::build_tiled(&A->full) != SB2_OK) return fail("build", trial);
    const sb2::TiledArrays& t = A->full.tiled;
    if (t.ncta == 0) {
      skipped++;
      sb2_csr_destroy(A);
      continue;
    }
    built++;
    // the device arrays are host memory under the stubs
    std::vector<int> seen(m, 0);
    if (2 * ((size_t)t.T * 8 + (size_t)t.emax * 10 + (size_t)t.spmax * 2) > 220 * 1024)
      return fail("stages beyond shared memory", trial);
    for (int c = 0; c < t.ncta; c++) {
      const int r0 = t.d_rptr[c], R = t.d_rptr[c + 1] - r0;
      if (R < 0 || R > 512) return fail("rows per CTA", trial);
      const int SP = (R + 1 + 7) / 8 * 8;
      if (SP > t.spmax || t.d_sbase[c] % 8) return fail("offset blocks", trial);
      const unsigned short* seg = t.d_seg + t.d_sbase[c];
      for (int j = 0; j < R; j++) {
        const int row = t.d_rows[r0 + j];
        if (row < 0 || row >= m || seen[row]++) return fail("row dealt twice", trial);
        if (ptr[row + 1] - ptr[row] <= minlen) return fail("short row dealt", trial);
        // read the row back tile by tile
        std::vector<std::pair<int, double>> got;
        for (int tt = 0; tt < t.ntile; tt++) {
          const unsigned short* sg = seg + (size_t)tt * SP;
          const long long base = t.d_cbase[(size_t)c * t.ntile + tt];
          const long long cap = t.d_cbase[(size_t)c * t.ntile + tt + 1] - base;
          if (base % 8 || cap % 8 || cap > t.emax || sg[j] > sg[j + 1] || sg[R] > cap ||
              cap - sg[R] >= 8)
            return fail("offsets", trial);
          for (int k = sg[j]; k < sg[j + 1]; k++)
            got.emplace_back(tt * t.T + t.d_col[base + k], t.d_val[base + k]);
        }
        std::vector<std::pair<int, double>> want;
        for (int k = ptr[row]; k < ptr[row + 1]; k++) want.emplace_back(ind[k], val[k]);
        std::stable_sort(want.begin(), want.end(), [&](const std::pair<int, double>& a,
                                                       const std::pair<int, double>& b) {
          return a.first / t.T < b.first / t.T;
        });
        if (got != want) return fail("entries", trial);
      }
    }
    for (int i = 0; i < m; i++)
      if ((ptr[i + 1] - ptr[i] > minlen) != (seen[i] == 1)) return fail("long row missing", trial);
    sb2_csr_destroy(A);
  }
  printf("tiled %d skipped %d\n", built, skipped);
  return 0;
}
