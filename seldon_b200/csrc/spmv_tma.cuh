// TMA-pipelined CSR SpMV engine (sm_100a).
//
// Each CTA owns a contiguous range of row blocks.  One elected thread streams
// every block's row pointers, column indices and values from HBM into a ring
// of S shared-memory stages with 1D bulk copies (cp.async.bulk, completion
// counted on an mbarrier per stage), running S-1 blocks ahead of the
// threads that consume them.  The consumers gather x, form the products in
// shared memory and reduce each row (thread-, warp- or CTA-per-row, chosen on
// the host from the row lengths).  Loading is thereby decoupled from the
// dependent gather/reduce chain that made the plain kernel latency-bound.
//
// The ring is perpetual: the producer wraps around the CTA's block range, so
// inside a persistent solver the matrix bytes of the NEXT product are already
// in flight while the grid waits at a barrier (the matrix does not depend on
// the vector being multiplied).
//
// Every wait is bounded (%globaltimer); a wait that runs out sets *status and
// the CTA unwinds after draining the copies it issued.
#pragma once

#include "sb2_internal.cuh"

namespace sb2 {

// Geometry of one stage.  kTmaCap nonzeros and kTmaRowCap rows at most per
// block; the copies start at 16-byte boundaries (4 indices), so each region
// carries up to 4 extra leading and trailing elements.
constexpr int kTmaCap = 2048;
constexpr int kTmaRowCap = 512;
constexpr int kTmaPad = 8;

template <typename VT>
struct TmaStageLayout {
  static constexpr int kIndBytes = (kTmaCap + kTmaPad) * 4;
  static constexpr int kValBytes = (kTmaCap + kTmaPad) * (int)sizeof(VT);
  static constexpr int kRpBytes = (kTmaRowCap + kTmaPad) * 4;
  static constexpr int kBytes = kIndBytes + kValBytes + kRpBytes;  // multiple of 16
};

// Block kinds of the TMA partition
enum TmaKind : unsigned char { kTmaThread = 0, kTmaWarp = 1, kTmaCta = 2 };

#ifdef __CUDACC__

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// 1D bulk copy global -> shared, completion counted on `bar`.  dst, src and
// bytes must be multiples of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Bounded wait on a stage barrier; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_timer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// Operator description consumed by the engine.
template <typename VT>
struct TmaOp {
  const int* ptr;    // [rows+1], padded
  const int* ind;    // padded
  const VT* val;     // padded
  const int4* desc;  // [nblk] {r0, r1 | kind << 30, k0, k1}
  int nblk;
  int rows;
};

// Shared-memory state of the engine (carved from dynamic shared memory).
//
// full[s]:  completes when stage s holds its block (producer arrive + bytes)
// empty[s]: completes when all W consumer warps are done with stage s
// Consumers are the W warps of the CTA, each working on its own slice of a
// block without any CTA-wide barrier; the producer is thread 0, which also
// consumes.  Products are formed in place over the staged values.
template <int S, typename VT, typename AT>
struct TmaRing {
  static_assert(sizeof(AT) == sizeof(VT), "products are stored over the staged values");
  unsigned char* stage;        // S * TmaStageLayout<VT>::kBytes
  unsigned long long* full;    // S
  unsigned long long* empty;   // S
  int4* sdesc;                 // S descriptors of the blocks in flight
  AT* part;                    // S * 32 per-warp partial sums (single-row blocks)
  int* cnt;                    // S arrival counters (single-row blocks)
  int b0, nb;                  // this CTA's block range
  unsigned issued, consumed;   // issued: thread 0; consumed: uniform per warp
  int4 pre;                    // thread 0: descriptor of the next block to issue

  static constexpr size_t smem_bytes() {
    return (size_t)S * TmaStageLayout<VT>::kBytes + 16 * S + 16 * S + sizeof(AT) * 32 * S +
           4 * S + 64;
  }

  __device__ __forceinline__ void carve(unsigned char* base) {
    stage = base;
    unsigned char* p = base + (size_t)S * TmaStageLayout<VT>::kBytes;
    full = reinterpret_cast<unsigned long long*>(p);
    empty = full + S;
    sdesc = reinterpret_cast<int4*>(p + 16 * S);
    part = reinterpret_cast<AT*>(p + 32 * S);
    cnt = reinterpret_cast<int*>(p + 32 * S + sizeof(AT) * 32 * S);
  }

  __device__ __forceinline__ int* s_ind(int s) const {
    return reinterpret_cast<int*>(stage + (size_t)s * TmaStageLayout<VT>::kBytes);
  }
  __device__ __forceinline__ VT* s_val(int s) const {
    return reinterpret_cast<VT*>(stage + (size_t)s * TmaStageLayout<VT>::kBytes +
                                 TmaStageLayout<VT>::kIndBytes);
  }
  __device__ __forceinline__ int* s_rp(int s) const {
    return reinterpret_cast<int*>(stage + (size_t)s * TmaStageLayout<VT>::kBytes +
                                  TmaStageLayout<VT>::kIndBytes + TmaStageLayout<VT>::kValBytes);
  }

  // Static contiguous share of the blocks for this CTA.
  __device__ __forceinline__ void init(const TmaOp<VT>& op) {
    const long long G = gridDim.x, c = blockIdx.x;
    b0 = (int)((op.nblk * c) / G);
    nb = (int)((op.nblk * (c + 1)) / G) - b0;
    issued = consumed = 0;
    const unsigned W = blockDim.x / 32;
    if (threadIdx.x == 0) {
      for (int s = 0; s < S; s++) {
        mbar_init(full + s, 1);
        mbar_init(empty + s, W);
        cnt[s] = 0;
      }
      mbar_fence_init();
      if (nb > 0) pre = op.desc[b0];
    }
    __syncthreads();
  }

  // Thread 0: copy block (b0 + issued mod nb) into stage issued mod S, after
  // every warp has released the stage's previous use.  The descriptor was
  // loaded one issue earlier; the next one is loaded now.
  __device__ __forceinline__ bool issue_one(const TmaOp<VT>& op, unsigned long long limit_ns) {
    const int s = (int)(issued % S);
    if (issued >= (unsigned)S &&
        !mbar_wait_bounded(empty + s, ((issued / S) - 1u) & 1u, limit_ns))
      return false;
    const int4 d = pre;
    pre = op.desc[b0 + (int)((issued + 1) % (unsigned)nb)];
    const int r0 = d.x, r1 = d.y & 0x3fffffff, k0 = d.z, k1 = d.w;
    const int kA = k0 & ~3, kE = (k1 + 3) & ~3;
    const int rA = r0 & ~3, rE = (r1 + 1 + 3) & ~3;
    const unsigned ib = (unsigned)(kE - kA) * 4u, vb = (unsigned)(kE - kA) * (unsigned)sizeof(VT);
    const unsigned rb = (unsigned)(rE - rA) * 4u;
    sdesc[s] = d;
    fence_proxy_async_smem();
    mbar_expect_tx(full + s, ib + vb + rb);
    if (ib) {
      bulk_g2s(s_ind(s), op.ind + kA, ib, full + s);
      bulk_g2s(s_val(s), op.val + kA, vb, full + s);
    }
    bulk_g2s(s_rp(s), op.ptr + rA, rb, full + s);
    issued++;
    return true;
  }

  // Thread 0 keeps up to S-1 blocks ahead of its own warp (never beyond
  // `horizon` issues in all).
  __device__ __forceinline__ bool top_up(const TmaOp<VT>& op, unsigned horizon,
                                         unsigned long long limit_ns) {
    if (threadIdx.x != 0 || nb == 0) return true;
    unsigned target = consumed + (S - 1);
    if (target > horizon) target = horizon;
    while (issued < target)
      if (!issue_one(op, limit_ns)) return false;
    return true;
  }

  // Thread 0 waits for the copies it issued that nobody consumed (end of a
  // persistent kernel, or after a wait ran out), so no copy outlives the CTA.
  __device__ __forceinline__ void drain(unsigned long long limit_ns) {
    if (threadIdx.x == 0) {
      unsigned c = consumed;
      while (c < issued) {
        const int s = (int)(c % S);
        mbar_wait_bounded(full + s, (c / S) & 1u, limit_ns);
        c++;
      }
    }
  }
};

// Process this CTA's blocks once (one product).  `horizon` = the total number
// of blocks the producer may issue over the kernel's life (a single product:
// nb; a persistent solver: unbounded, the ring wraps around).  Each warp
// returns when it has consumed every block; the caller synchronizes the CTA.
// Returns false when a wait ran out (*status set).
template <int NT, int S, typename VT, typename AT, class XLoad, class Epi>
__device__ __forceinline__ bool tma_spmv_pass(TmaRing<S, VT, AT>& R, const TmaOp<VT>& op,
                                              const XLoad& xl, Epi& epi, AT* s_red,
                                              unsigned horizon, unsigned long long limit_ns,
                                              int* status) {
  constexpr int W = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j = 0; j < R.nb; j++) {
    if (!R.top_up(op, horizon, limit_ns)) {
      atomicExch(status, 1);
      return false;
    }
    const int s = (int)(R.consumed % S);
    if (!mbar_wait_bounded(R.full + s, (R.consumed / S) & 1u, limit_ns)) {
      if (lane == 0) atomicExch(status, 1);
      return false;
    }
    const int4 d = R.sdesc[s];
    const int r0 = d.x, r1 = d.y & 0x3fffffff, kind = (unsigned)d.y >> 30, k0 = d.z, k1 = d.w;
    const int rA = r0 & ~3, kA = k0 & ~3;
    const int* rp = R.s_rp(s);
    const int* si = R.s_ind(s);
    VT* sv = R.s_val(s);
    if (kind == kTmaThread) {
      // this warp's slice of rows; products in place, then one lane per row
      // sums its row in stored order
      const int nr = r1 - r0, per = (nr + W - 1) / W;
      const int ra = r0 + min(nr, warp * per), rb = r0 + min(nr, (warp + 1) * per);
      const int ka = rp[ra - rA], kb = rp[rb - rA];
      for (int base = ka; base < kb; base += 32 * 8) {
        AT xv[8], vv[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int k = base + lane + 32 * u;
          if (k < kb) {
            vv[u] = AT(sv[k - kA]);
            xv[u] = AT(xl(si[k - kA]));
          }
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int k = base + lane + 32 * u;
          if (k < kb) sv[k - kA] = VT(mul_rn(vv[u], xv[u]));
        }
      }
      __syncwarp();
      for (int r = ra + lane; r < rb; r += 32) {
        const int a = rp[r - rA] - kA, e = rp[r + 1 - rA] - kA;
        AT t = AT(0);
        for (int k = a; k < e; k++) t = add_rn(t, AT(sv[k]));
        epi(r, t);
      }
    } else if (kind == kTmaWarp) {
      for (int r = r0 + warp; r < r1; r += W) {
        const int a = rp[r - rA], e = rp[r + 1 - rA];
        AT t = AT(0);
        for (int k = a + lane; k < e; k += 32)
          t = add_rn(t, mul_rn(AT(sv[k - kA]), AT(xl(si[k - kA]))));
        t = warp_sum(t);
        if (lane == 0) epi(r, t);
      }
    } else {
      // one long row: every warp sums a strided share, the last warp to
      // finish adds the W partial sums in warp order
      AT t = AT(0);
      for (int k = k0 + tid; k < k1; k += NT)
        t = add_rn(t, mul_rn(AT(sv[k - kA]), AT(xl(si[k - kA]))));
      t = warp_sum(t);
      if (lane == 0) {
        volatile AT* pv = R.part + s * 32;
        pv[warp] = t;
        __threadfence_block();
        const int old = atomicAdd(R.cnt + s, 1);
        if (old == W - 1) {
          __threadfence_block();
          AT acc = AT(0);
          for (int w = 0; w < W; w++) acc = add_rn(acc, pv[w]);
          R.cnt[s] = 0;
          epi(r0, acc);
        }
      }
    }
    __syncwarp();
    if (lane == 0) {
      fence_proxy_async_smem();  // our in-place writes precede the next copy
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(R.empty + s))
                   : "memory");
    }
    R.consumed++;
  }
  return true;
}

#endif  // __CUDACC__

}  // namespace sb2
