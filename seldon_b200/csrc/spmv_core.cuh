// Row-block CSR SpMV, the building block of every product in the library.
//
// Computes, for each row r of one row block, t_r = sum_j A(r, j) * x(j) with
// the terms added in stored order (as the reference's inner loop
// `temp += data[j] * X(ind[j])`, Functions_MatVect.cxx:423-428), and hands
// (r, t_r) to an epilogue functor.
//
// Block kinds (chosen on the host from the row lengths):
//   kBlkThread  consecutive short rows: the block's nonzeros are streamed once
//               with 16-byte loads of ind/val into shared memory as products,
//               then each thread sums one row sequentially (bit-identical to
//               the reference's sequential row sum).
//   kBlkWarp    the same staging, one warp per row with a shuffle reduction.
//   kBlkLong    one long row: the whole CTA strides over it with 16-byte loads
//               and a block reduction.
#pragma once

#include "sb2_internal.cuh"

namespace sb2 {

template <typename XT>
struct XLoadLdg {
  const XT* __restrict__ x;
  __device__ __forceinline__ XT operator()(int j) const { return __ldg(x + j); }
  // x[c.x], x[c.y], x[c.z], x[c.w]: one vector load when they are adjacent
  template <typename O>
  __device__ __forceinline__ void gather4(const int4& c, O (&o)[4]) const {
    XT v[4];
    if (quad_contiguous(x, c)) {
      vld4_ldg(x + c.x, v);
    } else {
      v[0] = __ldg(x + c.x); v[1] = __ldg(x + c.y); v[2] = __ldg(x + c.z); v[3] = __ldg(x + c.w);
    }
    o[0] = O(v[0]); o[1] = O(v[1]); o[2] = O(v[2]); o[3] = O(v[3]);
  }
};

// VT: matrix value type; AT: product/accumulation type (VT and XT are
// converted to AT before the multiply).  s_prod: kNnzCap AT in shared memory;
// s_red: NT/32 AT in shared memory.
template <int NT, typename VT, typename AT, class XLoad, class Epi>
__device__ __forceinline__ void spmv_row_block(
    const int* __restrict__ ptr, const int* __restrict__ ind,
    const VT* __restrict__ val, int r0, int r1, int kind, const XLoad& xl,
    Epi& epi, AT* s_prod, AT* s_red) {
  const int tid = threadIdx.x;
  if (kind == kBlkLong) {
    const int k0 = ptr[r0], k1 = ptr[r0 + 1];
    AT acc = AT(0);
    for (int g = (k0 >> 2) + tid; g < ((k1 + 3) >> 2); g += NT) {
      const int k = g << 2;
      int4 c = ld_stream_int4(ind + k);
      VT v[4];
      ld_stream_val4(val + k, v);
      if (k >= k0 && k < k1) acc = add_rn(acc, mul_rn(AT(v[0]), AT(xl(c.x))));
      if (k + 1 >= k0 && k + 1 < k1) acc = add_rn(acc, mul_rn(AT(v[1]), AT(xl(c.y))));
      if (k + 2 >= k0 && k + 2 < k1) acc = add_rn(acc, mul_rn(AT(v[2]), AT(xl(c.z))));
      if (k + 3 >= k0 && k + 3 < k1) acc = add_rn(acc, mul_rn(AT(v[3]), AT(xl(c.w))));
    }
    acc = block_sum<NT>(acc, s_red);
    if (tid == 0) epi(r0, acc);
    return;
  }

  const int k0 = ptr[r0], k1 = ptr[r1];
  for (int g = (k0 >> 2) + tid; g < ((k1 + 3) >> 2); g += NT) {
    const int k = g << 2;
    int4 c = ld_stream_int4(ind + k);
    VT v[4];
    ld_stream_val4(val + k, v);
    // all four gathers issue before the first product is stored
    AT xv[4];
    xv[0] = (k >= k0 && k < k1) ? AT(xl(c.x)) : AT(0);
    xv[1] = (k + 1 >= k0 && k + 1 < k1) ? AT(xl(c.y)) : AT(0);
    xv[2] = (k + 2 >= k0 && k + 2 < k1) ? AT(xl(c.z)) : AT(0);
    xv[3] = (k + 3 >= k0 && k + 3 < k1) ? AT(xl(c.w)) : AT(0);
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (k + e >= k0 && k + e < k1) s_prod[k + e - k0] = mul_rn(AT(v[e]), xv[e]);
  }
  __syncthreads();
  if (kind == kBlkThread) {
    for (int r = r0 + tid; r < r1; r += NT) {
      const int a = ptr[r] - k0, b = ptr[r + 1] - k0;
      AT t = AT(0);
      for (int k = a; k < b; k++) t = add_rn(t, s_prod[k]);
      epi(r, t);
    }
  } else {
    const int warp = tid >> 5, lane = tid & 31;
    for (int r = r0 + warp; r < r1; r += NT / 32) {
      const int a = ptr[r] - k0, b = ptr[r + 1] - k0;
      AT t = AT(0);
      for (int k = a + lane; k < b; k += 32) t = add_rn(t, s_prod[k]);
      t = warp_sum(t);
      if (lane == 0) epi(r, t);
    }
  }
  __syncthreads();  // s_prod is reused by the caller's next block
}

}  // namespace sb2
