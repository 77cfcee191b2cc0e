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
constexpr int kTiledCols = 6144;     // widest x tile (48 KB a stage)

// Rows longer than this go to the tiled product once the operator has at
// least kTiledMinEntries entries in such rows (sb2_spmv_set_tiling).
static std::atomic<int> g_tiled_min_len{128};
static std::atomic<long long> g_tiled_min_entries{1 << 20};

struct TiledView {
  int ncta, ntile, T, cols;
  int emax, spmax;                // largest chunk (entries) and offset block, both padded to 8
  const int* rows;                // [total rows] CTA-major
  const int* rptr;                // [ncta+1]
  const long long* cbase;         // [ncta*ntile+1] first entry of chunk (c, t), a multiple of 8
  const long long* sbase;         // [ncta] first row offset of CTA c's blocks
  const unsigned short* seg;      // per (c, t): R_c+1 offsets into the chunk, padded to 8
  const unsigned short* col;      // column - t*T
  const double* val;
};

#ifdef __CUDACC__

// Stage layout in shared memory (two stages): x tile (T doubles), the chunk's
// values (emax doubles), its 2-byte columns (emax), its row offsets (spmax).
template <int NT>
__global__ void __launch_bounds__(NT, 1)
    tiled_long_kernel(TiledView v, double alpha, const double* __restrict__ x, double beta,
                      double* __restrict__ y, bool overwrite, int* status,
                      unsigned long long limit_ns) {
  extern __shared__ __align__(128) unsigned char smem[];
  const size_t stage_bytes = (size_t)v.T * 8 + (size_t)v.emax * 10 + (size_t)v.spmax * 2;
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ int s_abort;
  const int c = blockIdx.x, tid = threadIdx.x;
  const int r0 = v.rptr[c], R = v.rptr[c + 1] - r0;
  const int SP = (R + 1 + 7) / 8 * 8;  // row offsets per tile, padded to 16 bytes
  auto xs_of = [&](int st) { return reinterpret_cast<double*>(smem + st * stage_bytes); };
  auto val_of = [&](int st) { return xs_of(st) + v.T; };
  auto col_of = [&](int st) {
    return reinterpret_cast<unsigned short*>(val_of(st) + v.emax);
  };
  auto seg_of = [&](int st) { return col_of(st) + v.emax; };
  // thread 0 copies what tile t needs into stage t & 1: the x tile (a
  // trailing odd entry by a plain load after the wait), the chunk's values
  // and columns and the row offsets, all with bulk copies.  A copy that would
  // not fit its stage is not issued: the status records it (3) and the CTA
  // stops.
  auto issue = [&](int t) {
    const int st = t & 1;
    const long long c0 = (long long)t * v.T;
    const long long cn = min((long long)v.T, (long long)v.cols - c0);
    const unsigned xb = (unsigned)((cn * 8) & ~15ll);
    const long long e0 = v.cbase[(size_t)c * v.ntile + t];
    const long long ne = v.cbase[(size_t)c * v.ntile + t + 1] - e0;  // a multiple of 8
    const unsigned short* sg = v.seg + v.sbase[c] + (long long)t * SP;
    fence_proxy_async_smem();  // earlier reads of the stage come first
    if (ne < 0 || ne > v.emax || SP > v.spmax || (e0 & 7) || (ne & 7) || cn <= 0) {
      atomicCAS(status, 0, 3);
      s_abort = 1;
      mbar_expect_tx(&bar[st], 0u);  // completes the phase: the wait below returns
      return;
    }
    mbar_expect_tx(&bar[st], xb + (unsigned)ne * 10u + (unsigned)SP * 2u);
    if (xb) bulk_g2s(xs_of(st), x + c0, xb, &bar[st]);
    if (ne) {
      bulk_g2s(val_of(st), v.val + e0, (unsigned)ne * 8u, &bar[st]);
      bulk_g2s(col_of(st), v.col + e0, (unsigned)ne * 2u, &bar[st]);
    }
    bulk_g2s(seg_of(st), sg, (unsigned)SP * 2u, &bar[st]);
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
    const int st = t & 1;
    if (tid == 0) {
      if (t + 1 < v.ntile) issue(t + 1);
      // bounded wait for tile t (phase t >> 1 of its stage's barrier)
      if (!mbar_wait_bounded(&bar[st], (unsigned)((t >> 1) & 1), limit_ns)) {
        atomicExch(status, 1);
        s_abort = 1;
      } else {
        const long long c0 = (long long)t * v.T;
        const long long cn = min((long long)v.T, (long long)v.cols - c0);
        if (cn & 1) xs_of(st)[cn - 1] = __ldg(x + c0 + cn - 1);
      }
    }
    __syncthreads();
    if (s_abort) break;
    if (tid < R) {
      // every index read from the stage is checked against the stage's own
      // extent (status 4 and the row's rest skipped): what the copies
      // delivered can never send a read outside the CTA's shared memory
      const long long c0 = (long long)t * v.T;
      const int cn = (int)min((long long)v.T, (long long)v.cols - c0);
      const int ne = (int)(v.cbase[(size_t)c * v.ntile + t + 1] - v.cbase[(size_t)c * v.ntile + t]);
      const double* xt = xs_of(st);
      const double* vt = val_of(st);
      const unsigned short* ct = col_of(st);
      const unsigned short* sg = seg_of(st);
      const int k0 = sg[tid], k1 = sg[tid + 1];
      if (k0 > k1 || k1 > ne) {
        atomicCAS(status, 0, 4);
      } else {
        for (int k = k0; k < k1; k++) {
          const int col = ct[k];
          if (col >= cn) {
            atomicCAS(status, 0, 4);
            break;
          }
          acc = add_rn(acc, mul_rn(vt[k], xt[col]));
        }
      }
    }
    __syncthreads();  // the stage is read before tile t + 2 lands in it
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
// not qualify (too few entries in long rows, x within a quarter of a tile,
// or no tile width whose two stages fit a CTA's shared memory).
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
  // the x tile: the widest whose two stages (x tile, largest chunk and its
  // row offsets) fit the shared memory of a CTA
  int T = 0, ntile = 0, emax = 0, spmax = 0;
  const size_t smem_cap = 220 * 1024;
  for (int Tc : {kTiledCols, kTiledCols * 2 / 3, kTiledCols / 3, kTiledCols / 6}) {
    const int nt = (int)((n + (long long)Tc - 1) / Tc);
    int em = 0, sp = 0;
    for (int c = 0; c < G; c++) {
      std::vector<int> chunk(nt, 0);
      for (int r : deal[c])
        for (int k = ptr[r]; k < ptr[r + 1]; k++) chunk[ind[k] / Tc]++;
      for (int t = 0; t < nt; t++) em = std::max(em, (chunk[t] + 7) / 8 * 8);
      sp = std::max(sp, ((int)deal[c].size() + 1 + 7) / 8 * 8);
    }
    const size_t need = 2 * ((size_t)Tc * 8 + (size_t)em * 10 + (size_t)sp * 2);
    if (em <= 65535 && need <= smem_cap) {
      T = Tc;
      ntile = nt;
      emax = em;
      spmax = sp;
      break;
    }
  }
  if (T == 0) return SB2_OK;  // some chunk too large for shared memory
  std::vector<int> rows, rptr(G + 1, 0);
  std::vector<long long> cbase((size_t)G * ntile + 1, 0), sbase(G, 0);
  std::vector<unsigned short> seg, col;
  std::vector<double> tval;
  col.reserve(lnnz + 8ll * G * ntile);
  tval.reserve(lnnz + 8ll * G * ntile);
  for (int c = 0; c < G; c++) {
    std::vector<int>& rs = deal[c];  // already by decreasing length
    rptr[c + 1] = rptr[c] + (int)rs.size();
    rows.insert(rows.end(), rs.begin(), rs.end());
    const int R = (int)rs.size();
    const int SP = (R + 1 + 7) / 8 * 8;
    sbase[c] = (long long)seg.size();
    // entries of (row j, tile t)
    std::vector<int> cnt((size_t)R * ntile, 0);
    for (int j = 0; j < R; j++)
      for (int k = ptr[rs[j]]; k < ptr[rs[j] + 1]; k++) cnt[(size_t)j * ntile + ind[k] / T]++;
    // start of (row j, tile t) inside chunk t; chunks padded to 8 entries
    // (16-byte bulk copies of the 2-byte columns), the padding never read
    std::vector<int> off((size_t)R * ntile);
    for (int t = 0; t < ntile; t++) {
      int sz = 0;
      for (int j = 0; j < R; j++) {
        off[(size_t)j * ntile + t] = sz;
        sz += cnt[(size_t)j * ntile + t];
      }
      cbase[(size_t)c * ntile + t + 1] = cbase[(size_t)c * ntile + t] + (sz + 7) / 8 * 8;
      for (int j = 0; j < R; j++) seg.push_back((unsigned short)off[(size_t)j * ntile + t]);
      seg.push_back((unsigned short)sz);
      for (int q = R + 1; q < SP; q++) seg.push_back((unsigned short)sz);
    }
    // chunk (c+1, 0) starts where (c, ntile-1) ends: the same cbase slot
    const long long cend = cbase[(size_t)c * ntile + ntile];
    col.resize(cend, 0);
    tval.resize(cend, 0.0);
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
  if (e == cudaSuccess) e = up((void**)&out.d_sbase, sbase.data(), sizeof(long long) * sbase.size());
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
  out.emax = emax;
  out.spmax = spmax;
  out.nwshort = (int)shortw.size();
  out.entries = (long long)col.size();
  tl = out;
  return SB2_OK;
}

void free_tiled(TiledArrays* t) {
  cudaFree(t->d_rows);
  cudaFree(t->d_rptr);
  cudaFree(t->d_cbase);
  cudaFree(t->d_sbase);
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
  const size_t smem = 2 * ((size_t)tl.T * 8 + (size_t)tl.emax * 10 + (size_t)tl.spmax * 2);
  static std::mutex mu;
  static std::vector<int> opted(64, 0);
  {
    // the opt-in covers the largest stage any plan may take
    std::lock_guard<std::mutex> g(mu);
    const int dev = current_device();
    if (dev >= 0 && dev < 64 && !opted[dev]) {
      SB2_CUDA_TRY(cudaFuncSetAttribute(tiled_long_kernel<kTiledThreads>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
      opted[dev] = 1;
    }
  }
  TiledView v{tl.ncta, tl.ntile, tl.T, a.cols, tl.emax, tl.spmax, tl.d_rows, tl.d_rptr,
              tl.d_cbase, tl.d_sbase, tl.d_seg, tl.d_col, tl.d_val};
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
