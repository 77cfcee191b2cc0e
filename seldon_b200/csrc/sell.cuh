// Row-length-binned SpMV over a sliced-ELLPACK copy of the short rows.
//
// Bins (chosen on the host from the row lengths):
//   thread bin  rows of <= kSellMaxLen nonzeros, packed into slices of 128
//               rows; lane l of the warp that takes a slice owns its rows
//               4l..4l+3 ("quad rows").  Group g of a slice holds entry k of
//               the four rows of one lane, so a lane reads the column
//               indices of its four rows with one 16-byte load and their
//               values with one (FP32) or two (FP64) 16-byte loads, and a
//               warp's loads are 512 contiguous bytes.  When the four
//               columns are consecutive and 16-byte aligned (banded and
//               stencil matrices) the four x values come with one vector
//               load too.  Each row is still summed alone, in stored order --
//               the reference's sequential row sum (Functions_MatVect.cxx:
//               423-428), bit for bit; padding entries are skipped, never
//               multiplied.
//   warp bin    rows of kSellMaxLen+1 .. kSellCtaLen nonzeros: one warp per
//               row over the original CSR arrays, shuffle reduction.
//   CTA bin     longer rows: one CTA per row, block reduction.
// Rows of the thread bin may be sorted by length (irregular matrices) so the
// slices carry little padding; lanes whose four rows are not consecutive
// read their row ids from a side table.
#pragma once

#include <cstdint>
#include <type_traits>
#include <utility>

#include "sb2_internal.cuh"

namespace sb2 {

constexpr int kSellMaxLen = 32;    // longest row of the thread bin
constexpr int kSellCtaLen = 1024;  // longest row of the warp bin
constexpr int kQuadRows = 128;     // rows of a slice: 32 lanes x 4 rows
constexpr unsigned kQuadScattered = 1u << 31;  // lane rows not row0..row0+3

// Device view of the binned operator (value type VT).
template <typename VT>
struct SellOp {
  int nslice;            // thread-bin slices of 128 rows
  const long long* sptr; // [nslice+1] first group of each slice (a group = 4 entries)
  const uint2* qinfo;    // [nslice*32] per lane: {row0 or kQuadScattered,
                         //  lengths of its 4 rows, 8 bits each}
  const int4* qrows;     // [nslice*32] row ids of scattered lanes (-1: none)
  const int* scol;       // [groups*4] column indices, group-major
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

// Epilogues may handle four consecutive rows at once: quad(row0, t[4]) is
// called for lanes whose rows are row0..row0+3 with row0 % 4 == 0; without
// it the scalar operator() runs for each row.
template <class E, typename AT, class = void>
struct HasQuad : std::false_type {};
template <class E, typename AT>
struct HasQuad<E, AT, std::void_t<decltype(std::declval<E&>().quad(0, std::declval<const AT*>()))>>
    : std::true_type {};

template <typename AT, class Epi>
__device__ __forceinline__ void epi_quad(Epi& epi, int row0, const AT* t) {
  if constexpr (HasQuad<Epi, AT>::value) {
    epi.quad(row0, t);
  } else {
    epi(row0, t[0]);
    epi(row0 + 1, t[1]);
    epi(row0 + 2, t[2]);
    epi(row0 + 3, t[3]);
  }
}

// One slice: lane `lane` sums its four rows (U groups loaded before the
// first product).
template <typename VT, typename AT, class XLoad, class Epi, int U = 1>
__device__ __forceinline__ void sell_slice(const SellOp<VT>& S, int slice, int lane,
                                           const XLoad& xl, Epi& epi) {
  const size_t q = (size_t)slice * 32 + lane;
  const uint2 inf = __ldg(S.qinfo + q);
  const int ln[4] = {(int)(inf.y & 255u), (int)((inf.y >> 8) & 255u),
                     (int)((inf.y >> 16) & 255u), (int)(inf.y >> 24)};
  const int L = max(max(ln[0], ln[1]), max(ln[2], ln[3]));
  const long long g0 = __ldg(S.sptr + slice) + lane;
  const int4* __restrict__ col4 = reinterpret_cast<const int4*>(S.scol);
  AT t[4] = {AT(0), AT(0), AT(0), AT(0)};
  for (int k0 = 0; k0 < L; k0 += U) {
    int4 c[U];
    VT v[U][4];
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (k0 + u < L) {
        const long long g = g0 + (long long)(k0 + u) * 32;
        c[u] = __ldcs(col4 + g);
        vld4_cs(S.sval + g * 4, v[u]);
      }
    }
    // every group's gathers are issued before the first product waits on one
    AT xv[U][4];
#pragma unroll
    for (int u = 0; u < U; u++)
      if (k0 + u < L) xl.gather4(c[u], xv[u]);
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (k0 + u < L) {
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (k0 + u < ln[j]) t[j] = add_rn(t[j], mul_rn(AT(v[u][j]), xv[u][j]));
      }
    }
  }
  if (!(inf.x & kQuadScattered)) {
    const int row0 = (int)inf.x;
    if ((row0 & 3) == 0) {
      epi_quad<AT>(epi, row0, t);
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) epi(row0 + j, t[j]);
    }
  } else {
    const int4 rr = __ldg(S.qrows + q);
    if (rr.x >= 0) epi(rr.x, t[0]);
    if (rr.y >= 0) epi(rr.y, t[1]);
    if (rr.z >= 0) epi(rr.z, t[2]);
    if (rr.w >= 0) epi(rr.w, t[3]);
  }
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
template <int NT, typename VT, typename AT, class XLoad, class Epi, int U = 1>
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
template <int NT, typename VT, typename AT, class XLoad, class Epi, int U = 1>
__device__ __forceinline__ void sell_spmv(const SellOp<VT>& S, const XLoad& xl, Epi& epi,
                                          AT* s_red, int cta, int ncta) {
  sell_spmv_slices<NT, VT, AT, XLoad, Epi, U>(S, xl, epi, cta, ncta);
  sell_spmv_long<NT, VT, AT>(S, xl, epi, s_red, cta, ncta);
}

#endif  // __CUDACC__

}  // namespace sb2
