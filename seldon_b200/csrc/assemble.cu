// Device assembly of CSR matrices from coordinate triplets: Seldon's
// ConvertMatrix_from_Coordinates (matrix_sparse/Matrix_Conversions.cxx:
// 1291-1334 for RowSparse, 1397-1467 for RowSymSparse) on the GPU.
//
// Seldon sorts the triplets by row, then each row by column, both times with
// its bottom-up merge sort (vector/Functions_Arrays.cxx:412-500), which keeps
// equal keys in input order.  The result is the triplets in stable
// (row, column) order, duplicates kept as separate entries.  Here:
//
//   k_coo_stats       sizes: largest row and column, bad indices, kept count
//   k_row_count       entries per row (warp-aggregated atomics), scanned
//                     into ptr
//   k_row_scatter     each entry's key (column << ib | input position) to a
//                     free slot of its row (atomics: any order inside a row)
//   k_row_sort_short  rows of up to 32 entries, one thread each: an entry's
//                     place is the number of smaller keys in its row; the
//                     keys are distinct (they hold the input position), so
//                     the order is (column, input position) exactly
//   k_row_sort_cta    rows of 33..4096 entries, one CTA each: bitonic sort
//                     in shared memory
//   longer rows       the stable LSD radix sort below, on the row's keys
//   (the sorted keys give ind directly and val through the position)
//
// All of it is integer and byte movement bound by HBM bandwidth and L2
// atomics; the matrix comes out deterministic whatever order the atomics
// take, because every row is sorted on distinct keys afterwards.
#include <algorithm>
#include <climits>
#include <utility>

#include "sb2_internal.cuh"

namespace sb2 {
namespace {

constexpr int kAsmThreads = 256;
constexpr int kAsmWarps = kAsmThreads / 32;
constexpr int kChunks = 16;
constexpr int kTile = kAsmThreads * kChunks;  // triplets per tile
constexpr int kBins = 256;                     // 8-bit digits

struct CooStats {
  int row_max;  // largest row - index (0 when empty)
  int col_max;
  int bad;      // some index - index < 0 or too large
  int kept;     // entries with row <= col
};

__global__ void __launch_bounds__(kAsmThreads)
k_coo_stats(const int* __restrict__ row, const int* __restrict__ col, long long nnz, int index,
            CooStats* st) {
  int rmax = 0, cmax = 0, bad = 0, kept = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += stride) {
    const long long r = (long long)row[i] - index, c = (long long)col[i] - index;
    if (r < 0 || c < 0 || r >= INT_MAX || c >= INT_MAX) {
      bad = 1;
      continue;
    }
    rmax = max(rmax, (int)r);
    cmax = max(cmax, (int)c);
    kept += (r <= c);
  }
  rmax = __reduce_max_sync(0xffffffffu, rmax);
  cmax = __reduce_max_sync(0xffffffffu, cmax);
  bad = __reduce_or_sync(0xffffffffu, bad);
  kept = __reduce_add_sync(0xffffffffu, kept);
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&st->row_max, rmax);
    atomicMax(&st->col_max, cmax);
    if (bad) atomicOr(&st->bad, 1);
    atomicAdd(&st->kept, kept);
  }
}

// Digit counts of each tile, stored digit-major: hist[d * ntiles + tile].
template <typename K>
__global__ void __launch_bounds__(kAsmThreads)
k_radix_hist(const K* __restrict__ key, long long nnz, int ntiles, int shift,
             int* __restrict__ hist) {
  __shared__ int h[kBins];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long t0 = (long long)blockIdx.x * kTile;
  for (int c = 0; c < kChunks; ++c) {
    const long long i = t0 + c * kAsmThreads + threadIdx.x;
    if (i < nnz) atomicAdd(&h[(unsigned)(key[i] >> shift) & (kBins - 1)], 1);
  }
  __syncthreads();
  hist[(long long)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: entry i goes to the tile's first position for
// its digit plus the number of earlier entries of the tile with that digit.
template <typename K>
__global__ void __launch_bounds__(kAsmThreads)
k_radix_scatter(const K* __restrict__ kin, const int* __restrict__ pin, long long nnz,
                int ntiles, int shift, const int* __restrict__ off, K* __restrict__ kout,
                int* __restrict__ pout) {
  __shared__ int s_cnt[kAsmWarps][kBins];  // digit counts of each warp's 32 entries
  __shared__ int s_off[kAsmWarps][kBins];  // first position of each warp's run
  __shared__ int s_base[kBins];            // next free position of each digit
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int w = 0; w < kAsmWarps; ++w) s_cnt[w][tid] = 0;
  s_base[tid] = off[(long long)tid * ntiles + blockIdx.x];
  __syncthreads();
  const long long t0 = (long long)blockIdx.x * kTile;
  for (int c = 0; c < kChunks; ++c) {
    const long long c0 = t0 + c * kAsmThreads;
    if (c0 >= nnz) break;  // uniform across the block
    const long long i = c0 + tid;
    const bool valid = i < nnz;
    const K k = valid ? kin[i] : K(0);
    const int p = (valid && pin) ? pin[i] : 0;
    const unsigned d = valid ? ((unsigned)(k >> shift) & (kBins - 1)) : (unsigned)kBins;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned before = peers & ((1u << lane) - 1u);
    if (valid && before == 0) s_cnt[warp][d] = __popc(peers);
    __syncthreads();
    {
      int run = s_base[tid];
#pragma unroll
      for (int w = 0; w < kAsmWarps; ++w) {
        const int n = s_cnt[w][tid];
        s_off[w][tid] = run;
        run += n;
        s_cnt[w][tid] = 0;
      }
      s_base[tid] = run;
    }
    __syncthreads();
    if (valid) {
      const int q = s_off[warp][d] + __popc(before);
      kout[q] = k;
      if (pout) pout[q] = p;
    }
  }
}

// Exclusive scan of n ints in three launches: tile sums, a scan of the sums
// in one CTA, and the tiles rescanned from their base.
constexpr int kScanTile = kTile;

__device__ __forceinline__ int block_excl_scan(int v, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  int wbase = 0, sum = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    const int s = s_warp[w];
    if (w < warp) wbase += s;
    sum += s;
  }
  __syncthreads();
  *total = sum;
  return wbase + incl - v;
}

__global__ void __launch_bounds__(kAsmThreads)
k_scan_sums(const int* __restrict__ a, long long n, int* __restrict__ sums) {
  __shared__ int s_warp[kAsmWarps];
  const long long t0 = (long long)blockIdx.x * kScanTile;
  int v = 0;
  for (int c = 0; c < kChunks; ++c) {
    const long long i = t0 + c * kAsmThreads + threadIdx.x;
    if (i < n) v += a[i];
  }
  int total;
  block_excl_scan(v, s_warp, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_top(int* __restrict__ sums, int nb) {
  __shared__ int s_warp[32];
  const int per = (nb + 1023) / 1024;
  const int b0 = threadIdx.x * per;
  int v = 0;
  for (int j = 0; j < per; ++j)
    if (b0 + j < nb) v += sums[b0 + j];
  int total;
  int run = block_excl_scan(v, s_warp, &total);
  for (int j = 0; j < per; ++j)
    if (b0 + j < nb) {
      const int s = sums[b0 + j];
      sums[b0 + j] = run;
      run += s;
    }
}

__global__ void __launch_bounds__(kAsmThreads)
k_scan_tiles(int* __restrict__ a, long long n, const int* __restrict__ sums) {
  __shared__ int s_warp[kAsmWarps];
  const long long t0 = (long long)blockIdx.x * kScanTile;
  int base = sums[blockIdx.x];
  for (int c = 0; c < kChunks; ++c) {
    const long long c0 = t0 + c * kAsmThreads;
    if (c0 >= n) break;  // uniform
    const long long i = c0 + threadIdx.x;
    const int v = i < n ? a[i] : 0;
    int total;
    const int ex = block_excl_scan(v, s_warp, &total);
    if (i < n) a[i] = base + ex;
    base += total;
  }
}

// Entries per row.  Lanes of a warp that hit the same row add once.
__global__ void __launch_bounds__(kAsmThreads)
k_row_count(const int* __restrict__ row, const int* __restrict__ col, long long nnz, int index,
            int sym, int* __restrict__ cnt) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (long long i0 = (long long)blockIdx.x * blockDim.x; i0 < nnz; i0 += stride) {
    const long long i = i0 + threadIdx.x;
    int r = -1;
    if (i < nnz) {
      r = row[i] - index;
      if (sym && r > col[i] - index) r = -1;  // below the diagonal: dropped
    }
    const unsigned peers = __match_any_sync(0xffffffffu, r);
    if (r >= 0 && lane == __ffs(peers) - 1) atomicAdd(&cnt[r], __popc(peers));
  }
}

// Each kept entry's key to a free slot of its row.
__global__ void __launch_bounds__(kAsmThreads)
k_row_scatter(const int* __restrict__ row, const int* __restrict__ col, long long nnz, int index,
              int sym, int ib, int* __restrict__ fill, unsigned long long* __restrict__ key) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (long long i0 = (long long)blockIdx.x * blockDim.x; i0 < nnz; i0 += stride) {
    const long long i = i0 + threadIdx.x;
    int r = -1, c = 0;
    if (i < nnz) {
      r = row[i] - index;
      c = col[i] - index;
      if (sym && r > c) r = -1;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, r);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (r >= 0 && lane == leader) base = atomicAdd(&fill[r], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (r >= 0) {
      const int slot = base + __popc(peers & ((1u << lane) - 1u));
      key[slot] = ((unsigned long long)(unsigned)c << ib) | (unsigned long long)i;
    }
  }
}

__device__ __forceinline__ void emit(unsigned long long k, long long at, int ib,
                                     const double* __restrict__ val, int* __restrict__ ind,
                                     double* __restrict__ vout) {
  ind[at] = (int)(k >> ib);
  vout[at] = val[k & ((1ull << ib) - 1ull)];
}

constexpr int kShortRow = 32;
constexpr int kCtaRow = 4096;

// Rows of up to kShortRow entries; longer ones are listed for the CTA and
// segment sorts.
__global__ void __launch_bounds__(kAsmThreads)
k_row_sort_short(const int* __restrict__ ptr, int m, const unsigned long long* __restrict__ key,
                 int ib, const double* __restrict__ val, int* __restrict__ ind,
                 double* __restrict__ vout, int* __restrict__ long_rows, int* __restrict__ nlong) {
  const int stride = gridDim.x * blockDim.x;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += stride) {
    const int b = ptr[r], e = ptr[r + 1];
    if (e - b > kShortRow) {
      long_rows[atomicAdd(nlong, 1)] = r;
      continue;
    }
    for (int a = b; a < e; ++a) {
      const unsigned long long ka = key[a];
      int rank = 0;
      for (int c = b; c < e; ++c) rank += key[c] < ka;
      emit(ka, b + rank, ib, val, ind, vout);
    }
  }
}

// One CTA per listed row of kShortRow+1..kCtaRow entries: bitonic sort of the
// row's keys (padded with the largest key) in shared memory.
__global__ void __launch_bounds__(kAsmThreads)
k_row_sort_cta(const int* __restrict__ ptr, const int* __restrict__ rows,
               const unsigned long long* __restrict__ key, int ib,
               const double* __restrict__ val, int* __restrict__ ind,
               double* __restrict__ vout) {
  __shared__ unsigned long long s[kCtaRow];
  const int r = rows[blockIdx.x];
  const int b = ptr[r], L = ptr[r + 1] - b;
  if (L > kCtaRow) return;  // segment-sorted on its own
  int P = 1;
  while (P < L) P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x) s[i] = i < L ? key[b + i] : ~0ull;
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const int x = i ^ j;
        if (x > i) {
          const unsigned long long u = s[i], v = s[x];
          if ((u > v) == ((i & k) == 0)) {
            s[i] = v;
            s[x] = u;
          }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < L; i += blockDim.x) emit(s[i], b + i, ib, val, ind, vout);
}

// A sorted segment of keys written out.
__global__ void __launch_bounds__(kAsmThreads)
k_emit_segment(const unsigned long long* __restrict__ key, long long b, long long L, int ib,
               const double* __restrict__ val, int* __restrict__ ind, double* __restrict__ vout) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += stride)
    emit(key[b + i], b + i, ib, val, ind, vout);
}

int bits_for(long long v) {  // bits needed to store 0..v
  int b = 0;
  while (v > 0) {
    ++b;
    v >>= 1;
  }
  return b;
}

int excl_scan(int* a, long long n, cudaStream_t s) {
  if (n <= 0) return SB2_OK;
  const long long nb = (n + kScanTile - 1) / kScanTile;
  if (nb > INT_MAX) return SB2_ERR_INVALID_VALUE;
  int* sums = nullptr;
  SB2_CUDA_TRY(pool_malloc((void**)&sums, sizeof(int) * nb, s));
  k_scan_sums<<<(unsigned)nb, kAsmThreads, 0, s>>>(a, n, sums);
  k_scan_top<<<1, 1024, 0, s>>>(sums, (int)nb);
  k_scan_tiles<<<(unsigned)nb, kAsmThreads, 0, s>>>(a, n, sums);
  cudaFreeAsync(sums, s);
  return map_cuda_error(cudaGetLastError());
}

// Stable sort of keys (and positions, when pos is not null) in place over
// the low `bits` bits.
template <typename K>
int radix_sort(K* key, int* pos, long long nnz, int bits, cudaStream_t s) {
  if (nnz <= 1 || bits <= 0) return SB2_OK;
  const long long ntl = (nnz + kTile - 1) / kTile;
  const long long nh = ntl * kBins;
  K* k2 = nullptr;
  int *p2 = nullptr, *hist = nullptr;
  cudaError_t e = pool_malloc((void**)&k2, sizeof(K) * nnz, s);
  if (e == cudaSuccess && pos) e = pool_malloc((void**)&p2, sizeof(int) * nnz, s);
  if (e == cudaSuccess) e = pool_malloc((void**)&hist, sizeof(int) * nh, s);
  int st = map_cuda_error(e);
  K *ka = key, *kb = k2;
  int *pa = pos, *pb = p2;
  for (int shift = 0; st == SB2_OK && shift < bits; shift += 8) {
    k_radix_hist<K><<<(unsigned)ntl, kAsmThreads, 0, s>>>(ka, nnz, (int)ntl, shift, hist);
    st = excl_scan(hist, nh, s);
    if (st != SB2_OK) break;
    k_radix_scatter<K><<<(unsigned)ntl, kAsmThreads, 0, s>>>(ka, pa, nnz, (int)ntl, shift, hist,
                                                             kb, pb);
    std::swap(ka, kb);
    std::swap(pa, pb);
    st = map_cuda_error(cudaGetLastError());
  }
  if (st == SB2_OK && ka != key) {
    e = cudaMemcpyAsync(key, ka, sizeof(K) * nnz, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && pos)
      e = cudaMemcpyAsync(pos, pa, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s);
    st = map_cuda_error(e);
  }
  if (k2) cudaFreeAsync(k2, s);
  if (p2) cudaFreeAsync(p2, s);
  if (hist) cudaFreeAsync(hist, s);
  return st;
}

int assemble(long long nnz, const int* row, const int* col, const double* val, int index, int m,
             int cb, int sym, long long nout, int* ptr, int* ind, double* vout, cudaStream_t s) {
  const int grid = num_sms(current_device()) * 8;
  SB2_CUDA_TRY(cudaMemsetAsync(ptr, 0, sizeof(int) * ((size_t)m + 1), s));
  if (nout == 0) return SB2_OK;
  const int ib = bits_for(nnz - 1);  // input positions 0..nnz-1
  if (ib + cb > 64) return SB2_ERR_INVALID_VALUE;
  unsigned long long* key = nullptr;
  int *fill = nullptr, *long_rows = nullptr, *nlong = nullptr;
  cudaError_t e = pool_malloc((void**)&key, sizeof(unsigned long long) * nout, s);
  if (e == cudaSuccess) e = pool_malloc((void**)&fill, sizeof(int) * ((size_t)m + 1), s);
  if (e == cudaSuccess) e = pool_malloc((void**)&long_rows, sizeof(int) * ((size_t)m + 1), s);
  if (e == cudaSuccess) e = pool_malloc((void**)&nlong, sizeof(int), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(nlong, 0, sizeof(int), s);
  int st = map_cuda_error(e);
  int h_nlong = 0;
  std::vector<int> hrows, hptr;
  if (st == SB2_OK) {
    k_row_count<<<grid, kAsmThreads, 0, s>>>(row, col, nnz, index, sym, ptr);
    st = excl_scan(ptr, (long long)m + 1, s);
  }
  if (st == SB2_OK) {
    e = cudaMemcpyAsync(fill, ptr, sizeof(int) * ((size_t)m + 1), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) {
      k_row_scatter<<<grid, kAsmThreads, 0, s>>>(row, col, nnz, index, sym, ib, fill, key);
      k_row_sort_short<<<grid, kAsmThreads, 0, s>>>(ptr, m, key, ib, val, ind, vout, long_rows,
                                                    nlong);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_nlong, nlong, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    st = map_cuda_error(e);
  }
  if (st == SB2_OK && h_nlong > 0) {
    k_row_sort_cta<<<h_nlong, kAsmThreads, 0, s>>>(ptr, long_rows, key, ib, val, ind, vout);
    // rows past the CTA sort: each sorted on its own
    hrows.resize(h_nlong);
    hptr.resize((size_t)m + 1);
    e = cudaMemcpyAsync(hrows.data(), long_rows, sizeof(int) * h_nlong, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hptr.data(), ptr, sizeof(int) * ((size_t)m + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    st = map_cuda_error(e);
    for (int k = 0; st == SB2_OK && k < h_nlong; ++k) {
      const int r = hrows[k];
      const long long b = hptr[r], L = (long long)hptr[r + 1] - b;
      if (L <= kCtaRow) continue;
      st = radix_sort<unsigned long long>(key + b, nullptr, L, ib + cb, s);
      if (st == SB2_OK) {
        const int g = (int)std::min<long long>((L + kAsmThreads - 1) / kAsmThreads, grid);
        k_emit_segment<<<g, kAsmThreads, 0, s>>>(key, b, L, ib, val, ind, vout);
        st = map_cuda_error(cudaGetLastError());
      }
    }
  }
  if (st == SB2_OK) st = map_cuda_error(cudaGetLastError());
  cudaFreeAsync(key, s);
  cudaFreeAsync(fill, s);
  cudaFreeAsync(long_rows, s);
  cudaFreeAsync(nlong, s);
  return st;
}

}  // namespace
}  // namespace sb2

using namespace sb2;

extern "C" {

int sb2_coo_to_csr(int nnz, const int* row, const int* col, const double* val, int index,
                   int m_min, int n_min, int symmetric_upper, void* stream, int* m_out,
                   int* n_out, int* nnz_out, int** ptr, int** ind, double** val_out) try {
  SB2_TRACE("sb2_coo_to_csr");
  if (nnz < 0 || m_min < 0 || n_min < 0 || !m_out || !n_out || !nnz_out || !ptr || !ind ||
      !val_out)
    return SB2_ERR_INVALID_VALUE;
  if (nnz > 0 && (!row || !col || !val)) return SB2_ERR_INVALID_VALUE;
  *ptr = nullptr;
  *ind = nullptr;
  *val_out = nullptr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  CooStats h = {0, 0, 0, 0};
  if (nnz > 0) {
    CooStats* d = nullptr;
    SB2_CUDA_TRY(pool_malloc((void**)&d, sizeof(CooStats), s));
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(CooStats), s);
    if (e == cudaSuccess) {
      const long long want = (nnz + kAsmThreads - 1) / kAsmThreads;
      const int grid = (int)std::min<long long>(want, num_sms(current_device()) * 8LL);
      k_coo_stats<<<grid, kAsmThreads, 0, s>>>(row, col, nnz, index, d);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(CooStats), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    SB2_CUDA_TRY(e);
    if (h.bad) return SB2_ERR_INVALID_VALUE;
  }

  // Sizes as ConvertMatrix_from_Coordinates sets them: RowSparse takes
  // max(largest index + 1, current size) and is at least 1 x 1 (the norm of
  // an empty index vector is 0); RowSymSparse is (largest row + 1) square,
  // and an empty input leaves the m_min x m_min matrix unchanged.
  long long m, n, nout;
  if (symmetric_upper) {
    m = nnz > 0 ? (long long)h.row_max + 1 : m_min;
    n = m;
    nout = h.kept;
  } else {
    m = std::max<long long>((long long)h.row_max + 1, m_min);
    n = std::max<long long>((long long)h.col_max + 1, n_min);
    nout = nnz;
  }
  if (m >= INT_MAX || n >= INT_MAX) return SB2_ERR_INVALID_VALUE;
  const int cb = bits_for(nnz > 0 ? h.col_max : 0);  // columns 0..max(col)

  int *dp = nullptr, *di = nullptr;
  double* dv = nullptr;
  cudaError_t e = pool_malloc_owned((void**)&dp, sizeof(int) * (m + 1), s);
  if (e == cudaSuccess && nout > 0) e = pool_malloc_owned((void**)&di, sizeof(int) * nout, s);
  if (e == cudaSuccess && nout > 0) e = pool_malloc_owned((void**)&dv, sizeof(double) * nout, s);
  int st = map_cuda_error(e);
  if (st == SB2_OK)
    st = assemble(nnz, row, col, val, index, (int)m, cb, symmetric_upper, nout, dp, di, dv, s);
  if (st == SB2_OK) st = map_cuda_error(cudaStreamSynchronize(s));
  if (st != SB2_OK) {
    sb2_device_free(dp);
    sb2_device_free(di);
    sb2_device_free(dv);
    return st;
  }
  *m_out = (int)m;
  *n_out = (int)n;
  *nnz_out = (int)nout;
  *ptr = dp;
  *ind = di;
  *val_out = dv;
  return SB2_OK;
} SB2_CATCH

}  // extern "C"
