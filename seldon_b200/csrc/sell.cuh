// Row-length-binned SpMV over a sliced-ELLPACK copy of the short rows.
//
// Bins (chosen on the host from the row lengths):
//   thread bin  rows of <= kSellMaxLen nonzeros, packed into slices of 32
//               rows stored column-major (SELL-32): entry j of the 32 rows of
//               a slice sits in 32 consecutive words, so a warp reads its
//               values and column indices with fully coalesced loads and
//               each lane sums ONE row in stored order -- the reference's
//               sequential row sum (Functions_MatVect.cxx:423-428), bit for
//               bit.  Padding entries are skipped, never multiplied.
//   warp bin    rows of kSellMaxLen+1 .. kSellCtaLen nonzeros: one warp per
//               row over the original CSR arrays, shuffle reduction.
//   CTA bin     longer rows: one CTA per row, block reduction.
// Rows of the thread bin may be sorted by length (irregular matrices) so the
// slices carry little padding; the per-lane row id says where the result goes.
#pragma once

#include "sb2_internal.cuh"

namespace sb2 {

constexpr int kSellMaxLen = 32;    // longest row of the thread bin
constexpr int kSellCtaLen = 1024;  // longest row of the warp bin
constexpr int kSellRowBits = 26;   // row id bits in a lane descriptor
constexpr unsigned kSellRowMask = (1u << kSellRowBits) - 1u;

// Device view of the binned operator (value type VT).
template <typename VT>
struct SellOp {
  int nslice;            // thread-bin slices of 32 rows
  const long long* sptr; // [nslice+1] element offset of each slice (multiple of 32)
  const unsigned* rinfo; // [nslice*32] row | len << 26; padding lanes: row field = mask
  const int* scol;       // column indices, column-major per slice
  const VT* sval;        // values, same layout
  int nwarp_rows;        // warp bin
  const int* wrows;
  int ncta_rows;         // CTA bin
  const int* crows;
  const int* ptr;        // the CSR arrays the warp and CTA bins read
  const int* ind;
  const VT* val;
};

#ifdef __CUDACC__

// One slice: every lane sums its row (entries loaded U at a time, all
// gathers of a group in flight before the first product).
template <typename VT, typename AT, class XLoad, class Epi, int U = 4>
__device__ __forceinline__ void sell_slice(const SellOp<VT>& S, int slice, int lane,
                                           const XLoad& xl, Epi& epi) {
  const unsigned info = __ldg(S.rinfo + (size_t)slice * 32 + lane);
  const int len = (int)(info >> kSellRowBits);
  const long long base = __ldg(S.sptr + slice) + lane;
  AT t = AT(0);
  for (int j0 = 0; j0 < len; j0 += U) {
    AT vv[U], xv[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (j0 + u < len) {
        const long long e = base + (long long)(j0 + u) * 32;
        vv[u] = AT(__ldcs(S.sval + e));
        xv[u] = AT(xl(__ldcs(S.scol + e)));
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (j0 + u < len) t = add_rn(t, mul_rn(vv[u], xv[u]));
  }
  const unsigned row = info & kSellRowMask;
  if (row != kSellRowMask) epi((int)row, t);
}

// Sum of the entries k0, k0+STEP, ... < e of a CSR row, four loads in
// flight at a time.
template <int STEP, typename VT, typename AT, class XLoad>
__device__ __forceinline__ AT strided_row_sum(const SellOp<VT>& S, int k0, int e, const XLoad& xl) {
  AT t = AT(0);
  int k = k0;
  for (; k + 3 * STEP < e; k += 4 * STEP) {
    AT v[4], xv[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      v[u] = AT(__ldcs(S.val + k + u * STEP));
      xv[u] = AT(xl(__ldcs(S.ind + k + u * STEP)));
    }
#pragma unroll
    for (int u = 0; u < 4; u++) t = add_rn(t, mul_rn(v[u], xv[u]));
  }
  for (; k < e; k += STEP) t = add_rn(t, mul_rn(AT(__ldcs(S.val + k)), AT(xl(__ldcs(S.ind + k)))));
  return t;
}

template <typename VT, typename AT, class XLoad, class Epi>
__device__ __forceinline__ void sell_warp_row(const SellOp<VT>& S, int row, int lane,
                                              const XLoad& xl, Epi& epi) {
  const int a = __ldg(S.ptr + row), e = __ldg(S.ptr + row + 1);
  AT t = strided_row_sum<32, VT, AT>(S, a + lane, e, xl);
  t = warp_sum(t);
  if (lane == 0) epi(row, t);
}

template <int NT, typename VT, typename AT, class XLoad, class Epi>
__device__ __forceinline__ void sell_cta_row(const SellOp<VT>& S, int row, const XLoad& xl,
                                             Epi& epi, AT* s_red) {
  const int a = __ldg(S.ptr + row), e = __ldg(S.ptr + row + 1);
  AT t = strided_row_sum<NT, VT, AT>(S, a + (int)threadIdx.x, e, xl);
  t = block_sum<NT>(t, s_red);
  if (threadIdx.x == 0) epi(row, t);
}

// All bins of one product, work spread over the grid: warps take slices and
// warp-bin rows, CTAs take CTA-bin rows.  `cta`/`ncta` let a persistent
// kernel pass its own CTA index and grid size.
// The thread bin (slices), warps grid-strided from (cta, ncta).
template <int NT, typename VT, typename AT, class XLoad, class Epi, int U = 4>
__device__ __forceinline__ void sell_spmv_slices(const SellOp<VT>& S, const XLoad& xl, Epi& epi,
                                                 int cta, int ncta) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)cta * W + (threadIdx.x >> 5), nw = (long long)ncta * W;
  for (long long s = gw; s < S.nslice; s += nw) sell_slice<VT, AT, XLoad, Epi, U>(S, (int)s, lane, xl, epi);
}

// The warp and CTA bins.
template <int NT, typename VT, typename AT, class XLoad, class Epi>
__device__ __forceinline__ void sell_spmv_long(const SellOp<VT>& S, const XLoad& xl, Epi& epi,
                                               AT* s_red, int cta, int ncta) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)cta * W + (threadIdx.x >> 5), nw = (long long)ncta * W;
  for (long long r = gw; r < S.nwarp_rows; r += nw)
    sell_warp_row<VT, AT>(S, __ldg(S.wrows + r), lane, xl, epi);
  for (int r = cta; r < S.ncta_rows; r += ncta)
    sell_cta_row<NT, VT, AT>(S, __ldg(S.crows + r), xl, epi, s_red);
}

// All bins of one product, work spread over the grid: warps take slices and
// warp-bin rows, CTAs take CTA-bin rows.  `cta`/`ncta` let a persistent
// kernel pass its own CTA index and grid size.
template <int NT, typename VT, typename AT, class XLoad, class Epi, int U = 4>
__device__ __forceinline__ void sell_spmv(const SellOp<VT>& S, const XLoad& xl, Epi& epi,
                                          AT* s_red, int cta, int ncta) {
  sell_spmv_slices<NT, VT, AT, XLoad, Epi, U>(S, xl, epi, cta, ncta);
  sell_spmv_long<NT, VT, AT>(S, xl, epi, s_red, cta, ncta);
}

#endif  // __CUDACC__

}  // namespace sb2
