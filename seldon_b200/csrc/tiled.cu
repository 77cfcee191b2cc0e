// x-tiled product of the long rows.
//
// In a matrix with many long rows and uniformly scattered columns (the Zipf
// workload: rows of 129..2000 entries hold 87% of its 68.8M entries), the
// binned product is bound by its gathers of x: each 8-byte read brings a
// 32-byte sector from L2, and the measured rate of such gathers is what the
// product reaches.  Here x moves instead as whole tiles of T consecutive
// entries, copied into shared memory by the bulk-copy engine (double
// buffered, completion on an mbarrier), and every gather is a shared-memory
// read.
//
// Layout (built once per operator, on its first standalone product): the
// long rows are dealt to CTAs by balancing their entries; a CTA's rows are
// sorted by length so the threads of a warp do similar work, and thread j
// owns row j of its CTA across all tiles.  Their entries are stored again,
// tile-major: for CTA c and tile t, the entries of row 0, then row 1, ... whose
// columns fall in tile t, each row's in stored order, with the column as a
// 2-byte offset into the tile.  A row summed tile after tile is then summed
// in stored order whenever its columns are sorted -- the reference's row
// loop (Functions_MatVect.cxx:423-428), bit for bit.
#include <algorithm>
#include <numeric>
#include <vector>

#include "sell.cuh"
#include "spmv_tma.cuh"

namespace sb2 {

constexpr int kTiledThreads = 512;   // threads (and rows at most) per CTA
constexpr int kTiledCols = 12288;    // columns per x tile (96 KB, two buffers)

// Rows longer than this go to the tiled product once the operator has at
// least kTiledMinEntries entries in such rows (sb2_spmv_set_tiling).
static std::atomic<int> g_tiled_min_len{128};
static std::atomic<long long> g_tiled_min_entries{1 << 20};

struct TiledView {
  int ncta, ntile, T, cols;
  const int* rows;                // [total rows] CTA-major
  const int* rptr;                // [ncta+1]
  const long long* cbase;         // [ncta*ntile+1] first entry of chunk (c, t)
  const unsigned short* seg;      // per (c, t): R_c+1 offsets into the chunk
  const unsigned short* col;      // column - t*T
  const double* val;
};

#ifdef __CUDACC__

template <int NT>
__global__ void __launch_bounds__(NT, 1)
    tiled_long_kernel(TiledView v, double alpha, const double* __restrict__ x, double beta,
                      double* __restrict__ y, bool overwrite, int* status,
                      unsigned long long limit_ns) {
  extern __shared__ __align__(128) unsigned char smem[];
  double* xs0 = reinterpret_cast<double*>(smem);
  double* xs1 = xs0 + v.T;
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ int s_abort;
  const int c = blockIdx.x, tid = threadIdx.x;
  const int r0 = v.rptr[c], R = v.rptr[c + 1] - r0;
  const unsigned short* seg = v.seg + (size_t)v.ntile * (r0 + c);
  // thread 0 copies tile t of x into buffer t & 1; the bytes up to the last
  // 16-byte boundary go by bulk copy, a trailing odd entry by a plain load
  auto issue = [&](int t) {
    const long long c0 = (long long)t * v.T;
    const long long cn = min((long long)v.T, (long long)v.cols - c0);
    const unsigned bytes = (unsigned)((cn * 8) & ~15ll);
    double* dst = (t & 1) ? xs1 : xs0;
    fence_proxy_async_smem();  // earlier reads of the buffer come first
    mbar_expect_tx(&bar[t & 1], bytes);
    if (bytes) bulk_g2s(dst, x + c0, bytes, &bar[t & 1]);
  };
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
    s_abort = 0;
  }
  __syncthreads();
  if (tid == 0) issue(0);
  double acc = 0.0;
  int t = 0;
  for (; t < v.ntile; t++) {
    if (tid == 0) {
      if (t + 1 < v.ntile) issue(t + 1);
      // bounded wait for tile t (phase t >> 1 of its buffer's barrier)
      if (!mbar_wait_bounded(&bar[t & 1], (unsigned)((t >> 1) & 1), limit_ns)) {
        atomicExch(status, 1);
        s_abort = 1;
      } else {
        const long long c0 = (long long)t * v.T;
        const long long cn = min((long long)v.T, (long long)v.cols - c0);
        if (cn & 1) ((t & 1) ? xs1 : xs0)[cn - 1] = __ldg(x + c0 + cn - 1);
      }
    }
    __syncthreads();
    if (s_abort) break;
    if (tid < R) {
      const double* xt = (t & 1) ? xs1 : xs0;
      const unsigned short* sg = seg + (size_t)t * (R + 1);
      const long long base = v.cbase[(size_t)c * v.ntile + t];
      const int k0 = sg[tid], k1 = sg[tid + 1];
#pragma unroll 4
      for (int k = k0; k < k1; k++)
        acc = add_rn(acc, mul_rn(__ldg(v.val + base + k), xt[__ldg(v.col + base + k)]));
    }
    __syncthreads();  // the buffer is read before tile t + 2 lands in it
  }
  if (s_abort) {
    // let the copies issued for tiles t and t + 1 land before the CTA exits
    if (tid == 0) {
      mbar_wait_bounded(&bar[t & 1], (unsigned)((t >> 1) & 1), limit_ns);
      if (t + 1 < v.ntile)
        mbar_wait_bounded(&bar[(t + 1) & 1], (unsigned)(((t + 1) >> 1) & 1), limit_ns);
    }
    return;
  }
  if (tid < R) {
    const int row = __ldg(v.rows + r0 + tid);
    double out = mul_rn(alpha, acc);
    if (!overwrite) out = add_rn(mul_rn(beta, y[row]), out);
    y[row] = out;
  }
}

#endif  // __CUDACC__

// Host plan.  Returns SB2_OK with a->tiled.ncta == 0 when the operator does
// not qualify (too few entries in long rows, x within one tile, or a chunk
// beyond 65535 entries).
int build_tiled(CsrArrays* a) {
  TiledArrays& tl = a->tiled;
  tl.built = true;
  const int m = a->rows, n = a->cols;
  const int min_len = g_tiled_min_len.load();
  if (m == 0 || n <= kTiledCols / 4 || a->max_row <= min_len) return SB2_OK;
  std::vector<int> ptr(m + 1);
  SB2_CUDA_TRY(cudaMemcpy(ptr.data(), a->d_ptr, sizeof(int) * (m + 1), cudaMemcpyDeviceToHost));
  std::vector<int> longr, shortw;
  long long lnnz = 0;
  for (int i = 0; i < m; i++) {
    const int len = ptr[i + 1] - ptr[i];
    if (len > min_len) {
      longr.push_back(i);
      lnnz += len;
    } else if (len > kSellMaxLen && len <= kSellCtaLen) {
      shortw.push_back(i);
    }
  }
  if (lnnz < g_tiled_min_entries.load()) return SB2_OK;
  // rows longer than kSellCtaLen but at most min_len (possible only when the
  // threshold is raised) would fall in neither list
  if (min_len > kSellCtaLen) return SB2_OK;
  const int T = kTiledCols;
  const int ntile = (int)((n + (long long)T - 1) / T);
  const int nsm = num_sms(current_device());
  const int G = std::max(nsm, (int)((longr.size() + kTiledThreads - 1) / kTiledThreads));
  // longest-processing-time deal of rows to CTAs (no CTA above kTiledThreads rows)
  std::sort(longr.begin(), longr.end(), [&](int p, int q) {
    const int lp = ptr[p + 1] - ptr[p], lq = ptr[q + 1] - ptr[q];
    return lp != lq ? lp > lq : p < q;
  });
  std::vector<std::vector<int>> deal(G);
  std::vector<long long> load(G, 0);
  {
    // a heap would do; G is small (one per SM), so a scan is cheap enough
    for (int r : longr) {
      int best = -1;
      for (int c = 0; c < G; c++)
        if ((int)deal[c].size() < kTiledThreads && (best < 0 || load[c] < load[best])) best = c;
      if (best < 0) return SB2_OK;  // cannot happen: G * kTiledThreads >= rows
      deal[best].push_back(r);
      load[best] += ptr[r + 1] - ptr[r];
    }
  }
  std::vector<int> ind(a->nnz);
  std::vector<double> val(a->nnz);
  if (a->nnz) {
    SB2_CUDA_TRY(cudaMemcpy(ind.data(), a->d_ind, sizeof(int) * a->nnz, cudaMemcpyDeviceToHost));
    SB2_CUDA_TRY(cudaMemcpy(val.data(), a->d_val, sizeof(double) * a->nnz, cudaMemcpyDeviceToHost));
  }
  // an operator created without validation may hold columns out of range:
  // it keeps the binned product
  for (int r : longr)
    for (int k = ptr[r]; k < ptr[r + 1]; k++)
      if (ind[k] < 0 || ind[k] >= n) return SB2_OK;
  std::vector<int> rows, rptr(G + 1, 0);
  std::vector<long long> cbase((size_t)G * ntile + 1, 0);
  std::vector<unsigned short> seg, col;
  std::vector<double> tval;
  seg.reserve((size_t)ntile * (longr.size() + G));
  col.reserve(lnnz);
  tval.reserve(lnnz);
  for (int c = 0; c < G; c++) {
    std::vector<int>& rs = deal[c];  // already by decreasing length
    rptr[c + 1] = rptr[c] + (int)rs.size();
    rows.insert(rows.end(), rs.begin(), rs.end());
    const int R = (int)rs.size();
    // entries of (row j, tile t)
    std::vector<int> cnt((size_t)R * ntile, 0);
    for (int j = 0; j < R; j++)
      for (int k = ptr[rs[j]]; k < ptr[rs[j] + 1]; k++) cnt[(size_t)j * ntile + ind[k] / T]++;
    // start of (row j, tile t) inside chunk t, and chunk sizes
    std::vector<int> off((size_t)R * ntile);
    for (int t = 0; t < ntile; t++) {
      long long s = 0;
      for (int j = 0; j < R; j++) {
        off[(size_t)j * ntile + t] = (int)s;
        s += cnt[(size_t)j * ntile + t];
      }
      if (s > 65535) {  // offsets are 2-byte
        tl = TiledArrays();
        tl.built = true;
        return SB2_OK;
      }
      cbase[(size_t)c * ntile + t + 1] = cbase[(size_t)c * ntile + t] + s;
      for (int j = 0; j < R; j++) seg.push_back((unsigned short)off[(size_t)j * ntile + t]);
      seg.push_back((unsigned short)s);
    }
    // chunk (c+1, 0) starts where (c, ntile-1) ends: the same cbase slot
    const long long cend = cbase[(size_t)c * ntile + ntile];
    col.resize(cend);
    tval.resize(cend);
    std::vector<int> fill(off);
    for (int j = 0; j < R; j++)
      for (int k = ptr[rs[j]]; k < ptr[rs[j] + 1]; k++) {
        const int t = ind[k] / T;
        const long long e = cbase[(size_t)c * ntile + t] + fill[(size_t)j * ntile + t]++;
        col[e] = (unsigned short)(ind[k] - t * T);
        tval[e] = val[k];
      }
  }
  // device copies
  auto up = [](void** d, const void* h, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMalloc(d, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess && bytes) e = cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice);
    return e;
  };
  TiledArrays out;
  out.built = true;
  cudaError_t e = up((void**)&out.d_rows, rows.data(), sizeof(int) * rows.size());
  if (e == cudaSuccess) e = up((void**)&out.d_rptr, rptr.data(), sizeof(int) * rptr.size());
  if (e == cudaSuccess) e = up((void**)&out.d_cbase, cbase.data(), sizeof(long long) * cbase.size());
  if (e == cudaSuccess) e = up((void**)&out.d_seg, seg.data(), sizeof(unsigned short) * seg.size());
  if (e == cudaSuccess) e = up((void**)&out.d_col, col.data(), sizeof(unsigned short) * col.size());
  if (e == cudaSuccess) e = up((void**)&out.d_val, tval.data(), sizeof(double) * tval.size());
  if (e == cudaSuccess) e = up((void**)&out.d_wshort, shortw.data(), sizeof(int) * shortw.size());
  if (e != cudaSuccess) {
    free_tiled(&out);
    return map_cuda_error(e);
  }
  out.ncta = G;
  out.ntile = ntile;
  out.T = T;
  out.nwshort = (int)shortw.size();
  out.entries = (long long)col.size();
  tl = out;
  return SB2_OK;
}

void free_tiled(TiledArrays* t) {
  cudaFree(t->d_rows);
  cudaFree(t->d_rptr);
  cudaFree(t->d_cbase);
  cudaFree(t->d_seg);
  cudaFree(t->d_col);
  cudaFree(t->d_val);
  cudaFree(t->d_wshort);
  *t = TiledArrays();
}

SellOp<double> sell_op(const CsrArrays& a);
template <int NT, bool OVERWRITE>
int launch_sell_warp_rows(const SellOp<double>& S, double alpha, const double* x, double beta,
                          double* y, cudaStream_t s);

// The standalone product through the tiled kernel: the slice kernel for
// rows of up to 32 entries, the warp kernel for rows of 33..min_len, the
// tiled kernel for the rest.  Returns SB2_ERR_NOT_SUPPORTED when the operator
// has no tiled layout or x is not 16-byte aligned (the caller then takes the
// binned product).
int launch_tiled_product(const CsrArrays& a, double alpha, const double* x, double beta,
                         double* y, bool overwrite, int* status, cudaStream_t s) {
  const TiledArrays& tl = a.tiled;
  if (!tl.built || tl.ncta == 0 || (reinterpret_cast<uintptr_t>(x) & 15u)) return SB2_ERR_NOT_SUPPORTED;
  SellOp<double> op = sell_op(a);
  op.nwarp_rows = tl.nwshort;
  op.wrows = tl.d_wshort;
  op.ncta_rows = 0;
  if (overwrite)
    SB2_TRY((launch_sell_warp_rows<256, true>(op, alpha, x, beta, y, s)));
  else
    SB2_TRY((launch_sell_warp_rows<256, false>(op, alpha, x, beta, y, s)));
  const size_t smem = sizeof(double) * 2 * (size_t)tl.T;
  static std::mutex mu;
  static std::vector<int> opted(64, 0);
  {
    std::lock_guard<std::mutex> g(mu);
    const int dev = current_device();
    if (dev >= 0 && dev < 64 && !opted[dev]) {
      SB2_CUDA_TRY(cudaFuncSetAttribute(tiled_long_kernel<kTiledThreads>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      opted[dev] = 1;
    }
  }
  TiledView v{tl.ncta, tl.ntile, tl.T, a.cols, tl.d_rows, tl.d_rptr, tl.d_cbase, tl.d_seg,
              tl.d_col, tl.d_val};
  tiled_long_kernel<kTiledThreads><<<tl.ncta, kTiledThreads, smem, s>>>(
      v, alpha, x, beta, y, overwrite, status, ring_wait_ns());
  SB2_CUDA_TRY(cudaGetLastError());
  return SB2_OK;
}

}  // namespace sb2

extern "C" int sb2_spmv_set_tiling(int min_row_len, long long min_entries) try {
  if (min_row_len < sb2::kSellMaxLen || min_row_len > sb2::kSellCtaLen || min_entries < 0)
    return SB2_ERR_INVALID_VALUE;
  sb2::g_tiled_min_len = min_row_len;
  sb2::g_tiled_min_entries = min_entries;
  return SB2_OK;
} SB2_CATCH
